// Toy ensembles fitted together: every toy's likelihood over its own data window and the one shared
// MC sample, for fits that float the couplings (the lineshape parameters stay where the ensemble was
// set up).  No counterpart in the reference, which builds one PDF per toy and evaluates the MC
// normalisation integral anew at every call (src/RooDalitzAmplitude.cxx:1293-1628, gen_toys/).
//
// With the lineshapes fixed, each event's |A|^2 is a Hermitian form in the helicity couplings c (the
// "slots": c_{r,k,m} of Lambda* r, c_{q,k,m} of Pc entry q in group order, proton helicity k):
//   v(c) = sum_h [ |H_L|^2 + 2 wgt Re(conj(H_L) sum_q S1_q HZ_q) + c2 sum_qq' S2_qq' conj(HZ_q) HZ_q' ]
// with H_L[h] = sum c L_r DL A and HZ_q[h] = sum c DZ AZ the Lambda* and per-entry Pc amplitudes of
// helicity h = (dmu, lb, k), S1_q = sum_b w_b R_q(m_b) and S2_qq' = sum_b w_b conj(R_q) R_q' the
// moments of the Pc lineshapes over the event's resolution rows (one row at m(J/psi p) when the event
// is not smeared), and wgt, c2 the reference's weights of its smearing scheme (kernel_calEva.cu:
// 676-810; wgt = c2 = 1 for unsmeared events and the weighted grid).  Hence
//   * the MC normalisation is c^H M c with M = sum_MC w d^2 v / dc* dc, built once per ensemble
//     (the Gram matrix of the per-event basis, FP64; k_ens_gram), and the non-interference sum
//     likewise with Mn;
//   * the data term of toy t, sum_{e in t} sw ln v_e(c_t), and its gradient in the slots need per
//     event only the lineshape factors L_r, S1, S2, which are cached once (k_ens_factors); one
//     persistent launch per ensemble step evaluates every toy's data term and gradient (k_ens_data).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pwa_b200.h"
#include "pwa_device.cuh"
#include "pwa_kernels.cuh"

namespace pwa {
namespace ens {

// Event classes of the ensemble (the segment kinds of the single-point evaluator).
enum EnsKind : uint8_t { EK_NONE = 0, EK_S20 = 1, EK_S30 = 2, EK_S150 = 3, EK_GRID = 4 };

// Layout of one event's factor row (doubles): L_r (2 NR), S1w = wgt S1 (2 NZ), S2c = c2 S2 for q <= q'
// (NZ (NZ + 1) / 2 complex), and for the Gram pass Rn = R(m(J/psi p)) (2 NZ), the rows' lineshapes at
// the event's own mass (the non-interference sum).
struct FactorLayout {
  int NR, NZ;
  __host__ __device__ int l() const { return 0; }
  __host__ __device__ int s1() const { return 2 * NR; }
  __host__ __device__ int s2() const { return 2 * NR + 2 * NZ; }
  __host__ __device__ int rn() const { return 2 * NR + 2 * NZ + NZ * (NZ + 1); }
  __host__ __device__ int size(bool with_rn) const { return rn() + (with_rn ? 2 * NZ : 0); }
};
__host__ __device__ inline int tri(int q, int p, int NZ) {  // index of (q, p), q <= p, in the upper triangle
  return q * NZ - q * (q - 1) / 2 + (p - q);
}

// Resolution rows of an event of class kind: the masses, weights and the scheme's wgt, c2.
struct Rows {
  int n;        // number of rows
  double wgt, c2;
  const float* qoff;   // quantile offsets (units of the resolution) or null
  const double* grid;  // (offset, weight) pairs or null
  double mz, mres;
  __device__ double mass(int b) const {
    if (qoff) return mz + (double)qoff[b] * mres;
    if (grid) return mz + __ldg(grid + 2 * b);
    return mz;
  }
  __device__ double weight(int b) const { return grid ? __ldg(grid + 2 * b + 1) : 1.0; }
};

__device__ inline Rows rows_of(int kind, double mz, const double* grid, int grid_nb) {
  Rows R{1, 1.0, 1.0, nullptr, nullptr, mz, MRES0 + mz * (MRES1 + mz * MRES2)};
  int nb = 0;
  switch (kind) {
    case EK_S20: nb = 20; R.qoff = kSmear20; break;
    case EK_S30: nb = 30; R.qoff = kSmear30; break;
    case EK_S150: nb = 150; R.qoff = kSmear150; break;
    case EK_GRID: R.n = grid_nb; R.grid = grid; return R;
    default: return R;
  }
  // the reference's float weight w = float(1 / NB) and rescale float(1 / w) (k_smeared's wgt, c2)
  const float wf = (float)(1.0 / nb);
  R.n = nb;
  R.wgt = (double)wf;
  R.c2 = R.wgt * R.wgt * (double)(1.0f / wf);
  return R;
}

// One thread per event: the factor row of events list[i] (or begin + i) into out[f * ld + i].
__global__ void __launch_bounds__(128) k_ens_factors(const PointTable* __restrict__ gtab, EventSet ev,
                                                     const uint8_t* __restrict__ kind, int64_t begin, int64_t count,
                                                     const double* __restrict__ grid, int grid_nb, double* out,
                                                     int64_t ld, int with_rn) {
  extern __shared__ __align__(16) unsigned char sm[];
  PointTable& T = *reinterpret_cast<PointTable*>(sm);
  load_table<128>(gtab, &T);
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int64_t e = begin + i;
  const Ev E{ev.pp, ev.pp1, ev.pp2, ev.n_size, e};
  const FactorLayout F{T.NR, T.NZ};
  const double mkp = E.mkp(), mz = E.mz();
  const LstarKin lk = lstar_kin(T, mkp);
  for (int r = 0; r < T.NR; ++r) {
    const cplx L = lstar_lineshape(T, r, lk);
    out[(size_t)(F.l() + 2 * r) * ld + i] = L.re;
    out[(size_t)(F.l() + 2 * r + 1) * ld + i] = L.im;
  }
  const int NZ = T.NZ;
  if (NZ == 0) return;
  const Rows R = rows_of(kind[e], mz, grid, grid_nb);
  cplx s1[MAX_PC], s2[MAX_PC * (MAX_PC + 1) / 2], raw[MAX_PC];
  for (int q = 0; q < NZ; ++q) s1[q] = mk(0, 0);
  for (int j = 0; j < NZ * (NZ + 1) / 2; ++j) s2[j] = mk(0, 0);
  for (int b = 0; b < R.n; ++b) {
    const double wb = R.weight(b);
    lookup_entries(T, R.mass(b), raw);
    for (int q = 0; q < NZ; ++q) {
      s1[q] += raw[q] * wb;
      for (int p = q; p < NZ; ++p) s2[tri(q, p, NZ)] += (conj(raw[q]) * raw[p]) * wb;
    }
  }
  for (int q = 0; q < NZ; ++q) {
    out[(size_t)(F.s1() + 2 * q) * ld + i] = R.wgt * s1[q].re;
    out[(size_t)(F.s1() + 2 * q + 1) * ld + i] = R.wgt * s1[q].im;
  }
  for (int j = 0; j < NZ * (NZ + 1) / 2; ++j) {
    out[(size_t)(F.s2() + 2 * j) * ld + i] = R.c2 * s2[j].re;
    out[(size_t)(F.s2() + 2 * j + 1) * ld + i] = R.c2 * s2[j].im;
  }
  if (with_rn) {
    lookup_entries(T, mz, raw);
    for (int q = 0; q < NZ; ++q) {
      out[(size_t)(F.rn() + 2 * q) * ld + i] = raw[q].re;
      out[(size_t)(F.rn() + 2 * q + 1) * ld + i] = raw[q].im;
    }
  }
}

// ------------------------------------------------------------------ Gram matrices of the MC
// An entry of M (or of Mn's Pc part) for slots a <= b of one proton helicity: per event it adds
// conj(f[o1]) f[o2] f[o3] f[o4] over the event's complex factor buffer f (layout GramBuf).
struct GramEntry {
  int16_t o1, o2, o3, o4;
};

// Complex factors of one MC event in shared memory: [0] = 1; QL[k][r][m] = L_r DL(s_r, k, m);
// YZ[k][q][m] = wgt S1_q DZ(s_q, k, m); DZ[k][q][m]; PL[m][m'] = w sum_ij conj(A_ijm) A_ijm';
// PLZ[m][m'] = w sum_ij conj(A_ijm) AZ_ijm'; PZ[m][m'] = w sum_ij conj(AZ_ijm) AZ_ijm'; S2c[q][q']
// (full); RN2[q][q'] = conj(Rn_q) Rn_q'.
struct GramBuf {
  int NR, NZ;
  __host__ __device__ int one() const { return 0; }
  __host__ __device__ int ql(int k, int r, int m) const { return 1 + (k * NR + r) * 6 + m; }
  __host__ __device__ int yz(int k, int q, int m) const { return 1 + 12 * NR + (k * NZ + q) * 12 + m; }
  __host__ __device__ int dz(int k, int q, int m) const { return 1 + 12 * NR + 24 * NZ + (k * NZ + q) * 12 + m; }
  __host__ __device__ int pl(int m, int n) const { return 1 + 12 * NR + 48 * NZ + m * 6 + n; }
  __host__ __device__ int plz(int m, int n) const { return 1 + 12 * NR + 48 * NZ + 36 + m * 12 + n; }
  __host__ __device__ int pz(int m, int n) const { return 1 + 12 * NR + 48 * NZ + 108 + m * 12 + n; }
  __host__ __device__ int s2(int q, int p) const { return 1 + 12 * NR + 48 * NZ + 252 + q * NZ + p; }
  __host__ __device__ int rn2(int q, int p) const { return 1 + 12 * NR + 48 * NZ + 252 + NZ * NZ + q * NZ + p; }
  __host__ __device__ int size() const { return 1 + 12 * NR + 48 * NZ + 252 + 2 * NZ * NZ; }
};

constexpr int GRAM_THREADS = 256;
constexpr int GRAM_EPT = 8;   // entries per thread
constexpr int GRAM_EB = 4;    // events staged per round

// Fills the factor buffers of events [e0, e0 + ne) (ne <= GRAM_EB) of a chunk whose factor rows are
// fac[f * ld + i] (i = event - chunk_begin).
__device__ void gram_stage(const PointTable& T, const EventSet& ev, int64_t chunk_begin, int64_t i0, int ne,
                           const double* __restrict__ fac, int64_t ld, cplx* buf, int bsize) {
  const GramBuf G{T.NR, T.NZ};
  const FactorLayout F{T.NR, T.NZ};
  const int NR = T.NR, NZ = T.NZ;
  for (int j = 0; j < ne; ++j) {
    const int64_t i = i0 + j, e = chunk_begin + i;
    const Ev E{ev.pp, ev.pp1, ev.pp2, ev.n_size, e};
    const double w = (double)E.w();
    cplx* f = buf + (size_t)j * bsize;
    auto facc = [&](int o) { return mk(fac[(size_t)o * ld + i], fac[(size_t)(o + 1) * ld + i]); };
    for (int t = threadIdx.x; t < bsize; t += blockDim.x) {
      cplx v = mk(0, 0);
      if (t == 0) {
        v = mk(1, 0);
      } else if (t < G.yz(0, 0, 0)) {
        const int u = t - 1, k = u / (6 * NR), r = (u / 6) % NR, m = u % 6;
        v = facc(F.l() + 2 * r) * E.DL(T.L[r].sidx, k, m);
      } else if (t < G.dz(0, 0, 0)) {
        const int u = t - G.yz(0, 0, 0), k = u / (12 * NZ), q = (u / 12) % NZ, m = u % 12;
        v = facc(F.s1() + 2 * q) * E.DZ(T.Z[T.order[q]].sidx, k, m);
      } else if (t < G.pl(0, 0)) {
        const int u = t - G.dz(0, 0, 0), k = u / (12 * NZ), q = (u / 12) % NZ, m = u % 12;
        v = mk(E.DZ(T.Z[T.order[q]].sidx, k, m), 0);
      } else if (t < G.plz(0, 0)) {
        const int u = t - G.pl(0, 0), m = u / 6, n = u % 6;
        for (int ij = 0; ij < 4; ++ij) v += conj(E.A(ij >> 1, ij & 1, m)) * E.A(ij >> 1, ij & 1, n);
        v = v * w;
      } else if (t < G.pz(0, 0)) {
        const int u = t - G.plz(0, 0), m = u / 12, n = u % 12;
        for (int ij = 0; ij < 4; ++ij) v += conj(E.A(ij >> 1, ij & 1, m)) * E.AZ(ij >> 1, ij & 1, n);
        v = v * w;
      } else if (t < G.s2(0, 0)) {
        const int u = t - G.pz(0, 0), m = u / 12, n = u % 12;
        for (int ij = 0; ij < 4; ++ij) v += conj(E.AZ(ij >> 1, ij & 1, m)) * E.AZ(ij >> 1, ij & 1, n);
        v = v * w;
      } else if (t < G.rn2(0, 0)) {
        const int u = t - G.s2(0, 0), q = u / NZ, p = u % NZ;
        v = q <= p ? facc(F.s2() + 2 * tri(q, p, NZ)) : conj(facc(F.s2() + 2 * tri(p, q, NZ)));
      } else {
        const int u = t - G.rn2(0, 0), q = u / NZ, p = u % NZ;
        v = conj(facc(F.rn() + 2 * q)) * facc(F.rn() + 2 * p);
      }
      f[t] = v;
    }
  }
}

// Block (x = event share of the chunk, y = entry tile): accumulates its entries over its events and
// writes them to part[blockIdx.x][entry].
__global__ void __launch_bounds__(GRAM_THREADS) k_ens_gram(const PointTable* __restrict__ gtab, EventSet ev,
                                                         int64_t chunk_begin, int64_t count,
                                                         const double* __restrict__ fac, int64_t ld,
                                                         const GramEntry* __restrict__ entries, int n_entries,
                                                         cplx* part) {
  extern __shared__ __align__(16) unsigned char sm[];
  PointTable& T = *reinterpret_cast<PointTable*>(sm);
  load_table<GRAM_THREADS>(gtab, &T);
  const GramBuf G{T.NR, T.NZ};
  const int bsize = G.size();
  cplx* buf = reinterpret_cast<cplx*>(sm + ((sizeof(PointTable) + 15) & ~size_t(15)));
  GramEntry my[GRAM_EPT];
  cplx acc[GRAM_EPT];
  const int base = blockIdx.y * GRAM_THREADS * GRAM_EPT + threadIdx.x;
#pragma unroll
  for (int j = 0; j < GRAM_EPT; ++j) {
    const int en = base + j * GRAM_THREADS;
    my[j] = en < n_entries ? entries[en] : GramEntry{0, 0, 0, 0};
    acc[j] = mk(0, 0);
  }
  const int64_t per = (count + gridDim.x - 1) / gridDim.x;
  const int64_t i_begin = (int64_t)blockIdx.x * per, i_end = count < i_begin + per ? count : i_begin + per;
  for (int64_t i0 = i_begin; i0 < i_end; i0 += GRAM_EB) {
    const int ne = (int)(i_end - i0 < GRAM_EB ? i_end - i0 : GRAM_EB);
    __syncthreads();
    gram_stage(T, ev, chunk_begin, i0, ne, fac, ld, buf, bsize);
    __syncthreads();
    for (int j = 0; j < ne; ++j) {
      const cplx* f = buf + (size_t)j * bsize;
#pragma unroll
      for (int u = 0; u < GRAM_EPT; ++u) acc[u] += conj(f[my[u].o1]) * f[my[u].o2] * f[my[u].o3] * f[my[u].o4];
    }
  }
#pragma unroll
  for (int j = 0; j < GRAM_EPT; ++j) {
    const int en = base + j * GRAM_THREADS;
    if (en < n_entries) part[(size_t)blockIdx.x * n_entries + en] = acc[j];
  }
}

// Sums the rows of part [rows][n] into out[n] (added to), in row order.
__global__ void k_ens_sum_rows(const cplx* __restrict__ part, int rows, int n, cplx* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  cplx s = mk(0, 0);
  for (int r = 0; r < rows; ++r) s += part[(size_t)r * n + j];
  out[j] += s;
}

// ------------------------------------------------------------------ data terms of all toys
constexpr int ENS_MAX_SLOTS = 2 * (6 * MAX_LSTAR + 12 * MAX_PC);

// A work item: events [e0, e1) of toy t.
struct Tile {
  int64_t e0, e1;
  int t, pad;
};

// Per-warp scratch of the data kernel, laid out at run time for the model (offsets in doubles):
// the event's plane slots pp / pp1 / pp2 (303), its factor row, HZ_q[h], d v / d conj(HZ_q[h]),
// d v / d conj(H_L[h]), sum_ij conj(A_ijm) x[k, ij] (12 complex), sum_ij conj(AZ_ijm) z_q[k, ij].
struct EnsScratch {
  int pl, fac, hz, z, x, yl, yz, size;  // size: doubles per warp (a multiple of 2)
};
inline EnsScratch ens_scratch(int NR, int NZ) {
  EnsScratch s;
  const int nf = 2 * NR + 2 * NZ + NZ * (NZ + 1);
  s.pl = 0;
  s.fac = SLOT_PP3 + 1;  // 304: keeps the complex arrays 16-byte aligned
  s.hz = s.fac + ((nf + 1) & ~1);
  s.z = s.hz + 2 * 8 * NZ;
  s.x = s.z + 2 * 8 * NZ;
  s.yl = s.x + 16;
  s.yz = s.yl + 24;
  s.size = s.yz + 2 * 24 * NZ;
  return s;
}

constexpr int ENS_PV = (SLOT_PP3 + 31) / 32;  // plane values per lane (prefetch)
constexpr int ENS_FV = (2 * MAX_LSTAR + 2 * MAX_PC + MAX_PC * (MAX_PC + 1) + 31) / 32;  // factor values per lane

// Index descriptors the data kernel builds once per block: per slot, the plane slot of its angular
// factor (DL or DZ; bit 30 set for a Pc slot) and its factor-row / y indices; per y entry (12 Lambda*
// + 24 NZ Pc), the plane slot of A_00m or AZ_00m (bit 30 set for Pc) and the x / z base it contracts.
__host__ __device__ inline int ens_desc_count(int n_slot, int NZ) { return (n_slot + 12 + 24 * NZ + 1) & ~1; }

__host__ __device__ inline size_t ens_data_smem(int warps, int n_slot, int NZ, const EnsScratch& sc) {
  return ((sizeof(PointTable) + 15) & ~size_t(15)) + (size_t)n_slot * sizeof(cplx) +
         (size_t)ens_desc_count(n_slot, NZ) * sizeof(int2) + (size_t)warps * sc.size * sizeof(double);
}

// Persistent blocks take tiles from *next; per tile the block loads the toy's slot couplings and each
// warp evaluates one event at a time, the next event's plane slots and factors already on their way
// into registers.  Per toy: val[t] += sum sw ln v (-1e12 for v <= 0, as the reference), bad[t] counts
// events with v <= 0 or not finite, grad[t][s] += sum (sw / v) dv/dconj(c_s).  SPL: slots per lane
// (n_slot <= 32 SPL).
template <int WARPS, int SPL>
__global__ void __launch_bounds__(WARPS * 32) k_ens_data(const PointTable* __restrict__ gtab, EventSet ev,
                                                         const double* __restrict__ fac, int64_t ld,
                                                         const Tile* __restrict__ tiles, int n_tiles, int* next,
                                                         const cplx* __restrict__ coup, const int* __restrict__ on,
                                                         int n_slot, EnsScratch sc, double* val, cplx* grad,
                                                         unsigned long long* bad) {
  extern __shared__ __align__(16) unsigned char sm[];
  PointTable& T = *reinterpret_cast<PointTable*>(sm);
  load_table<WARPS * 32>(gtab, &T);
  cplx* c = reinterpret_cast<cplx*>(sm + ((sizeof(PointTable) + 15) & ~size_t(15)));
  int2* sdesc = reinterpret_cast<int2*>(c + n_slot);  // [n_slot] then the y entries
  int2* ydesc = sdesc + n_slot;
  double* wb = reinterpret_cast<double*>(sdesc + ens_desc_count(n_slot, T.NZ)) + (size_t)(threadIdx.x / 32) * sc.size;
  double* pl = wb + sc.pl;
  double* fr = wb + sc.fac;
  cplx* whz = reinterpret_cast<cplx*>(wb + sc.hz);  // [q][8]
  cplx* wz = reinterpret_cast<cplx*>(wb + sc.z);    // [q][8]
  cplx* wx = reinterpret_cast<cplx*>(wb + sc.x);    // [8]
  cplx* wyl = reinterpret_cast<cplx*>(wb + sc.yl);  // [12]
  cplx* wyz = reinterpret_cast<cplx*>(wb + sc.yz);  // [24 NZ]
  __shared__ int tile_id;
  const int lane = threadIdx.x & 31, warp = threadIdx.x / 32;
  const int h = lane & 7, part = lane >> 3;
  const int hi = h >> 2, hj = (h >> 1) & 1, hk = h & 1;
  const int NR = T.NR, NZ = T.NZ, NS = 6 * NR + 12 * NZ;
  const FactorLayout F{NR, NZ};
  const int nf = F.size(false);
  for (int s = threadIdx.x; s < n_slot; s += WARPS * 32) {
    const int k = s / NS, u = s % NS;
    if (u < 6 * NR) {
      const int r = u / 6, m = u % 6;
      sdesc[s] = make_int2(51 + T.L[r].sidx * 12 + k * 6 + m, (F.l() + 2 * r) | ((k * 6 + m) << 16));
    } else {
      const int q = (u - 6 * NR) / 12, m = (u - 6 * NR) % 12;
      sdesc[s] = make_int2((SLOT_PP2 + T.Z[T.order[q]].sidx * 24 + k * 12 + m) | (1 << 30), (k * NZ + q) * 12 + m);
    }
  }
  for (int t = threadIdx.x; t < 12 + 24 * NZ; t += WARPS * 32) {
    if (t < 12) {
      ydesc[t] = make_int2(3 + 2 * (t % 6), t / 6);
    } else {
      const int u = t - 12, k = u / (12 * NZ), q = (u / 12) % NZ, m = u % 12;
      ydesc[t] = make_int2((SLOT_PP1 + 2 * m) | (1 << 30), q * 8 + k);
    }
  }
  // (made visible by the __syncthreads at the top of the tile loop)
  float pv[ENS_PV];
  double fv[ENS_FV];
  float swv = 0;
  auto fetch = [&](int64_t e) {
#pragma unroll
    for (int i = 0; i < ENS_PV; ++i) {
      const int j = lane + 32 * i;
      const float* src = j < SLOT_PP1 ? ev.pp + (size_t)j * ev.n_size
                                      : (j < SLOT_PP2 ? ev.pp1 + (size_t)(j - SLOT_PP1) * ev.n_size
                                                      : ev.pp2 + (size_t)(j - SLOT_PP2) * ev.n_size);
      pv[i] = j < SLOT_PP3 ? __ldg(src + e) : 0.0f;
    }
#pragma unroll
    for (int i = 0; i < ENS_FV; ++i) {
      const int f = lane + 32 * i;
      fv[i] = f < nf ? __ldg(fac + (size_t)f * ld + e) : 0.0;
    }
    swv = __ldg(ev.sw + e);
  };
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) tile_id = atomicAdd(next, 1);
    __syncthreads();
    const int ti = tile_id;
    if (ti >= n_tiles) break;
    const Tile tl = tiles[ti];
    if (!on[tl.t]) continue;
    for (int s = threadIdx.x; s < n_slot; s += WARPS * 32) c[s] = coup[(size_t)tl.t * n_slot + s];
    __syncthreads();
    cplx acc[SPL];
#pragma unroll
    for (int j = 0; j < SPL; ++j) acc[j] = mk(0, 0);
    double value = 0;
    unsigned long long nbad = 0;
    if (tl.e0 + warp < tl.e1) fetch(tl.e0 + warp);
    for (int64_t e = tl.e0 + warp; e < tl.e1; e += WARPS) {
#pragma unroll
      for (int i = 0; i < ENS_PV; ++i)
        if (lane + 32 * i < SLOT_PP3) pl[lane + 32 * i] = (double)pv[i];
#pragma unroll
      for (int i = 0; i < ENS_FV; ++i)
        if (lane + 32 * i < nf) fr[lane + 32 * i] = fv[i];
      const double sw = (double)swv;
      __syncwarp();
      if (e + WARPS < tl.e1) fetch(e + WARPS);  // the next event's loads overlap this event's work
      const EvS E{pl};
      // H_L[h]: lane (h, part) sums the Lambda* r = part mod 4
      cplx hl = mk(0, 0);
      for (int r = part; r < NR; r += 4) {
        const int sidx = T.L[r].sidx;
        const cplx* cr = c + hk * NS + r * 6;
        cplx f = mk(0, 0);
#pragma unroll
        for (int m = 0; m < 6; ++m) cmac(f, cr[m], E.A(hi, hj, m) * E.DL(sidx, hk, m));
        cmac(hl, mk(fr[F.l() + 2 * r], fr[F.l() + 2 * r + 1]), f);
      }
      hl += shfl_xor(hl, 8);
      hl += shfl_xor(hl, 16);
      for (int q = part; q < NZ; q += 4) {
        const int sidx = T.Z[T.order[q]].sidx;
        const cplx* cq = c + hk * NS + 6 * NR + q * 12;
        cplx f = mk(0, 0);
#pragma unroll
        for (int m = 0; m < 12; ++m) cmac(f, cq[m], E.AZ(hi, hj, m) * E.DZ(sidx, hk, m));
        whz[q * 8 + h] = f;
      }
      __syncwarp();
      double vp = 0;
      if (part == 0) {
        cplx sx = mk(0, 0);
        for (int q = 0; q < NZ; ++q) cmac(sx, mk(fr[F.s1() + 2 * q], fr[F.s1() + 2 * q + 1]), whz[q * 8 + h]);
        vp = norm2(hl) + 2.0 * (hl.re * sx.re + hl.im * sx.im);
        wx[h] = hl + sx;
      }
      for (int q = part; q < NZ; q += 4) {
        cplx tq = mk(0, 0);
        for (int p = 0; p < NZ; ++p) {
          const int o = F.s2() + 2 * (q <= p ? tri(q, p, NZ) : tri(p, q, NZ));
          const cplx s2 = q <= p ? mk(fr[o], fr[o + 1]) : mk(fr[o], -fr[o + 1]);
          cmac(tq, s2, whz[p * 8 + h]);
        }
        const cplx hz = whz[q * 8 + h];
        vp += hz.re * tq.re + hz.im * tq.im;
        wz[q * 8 + h] = conj(mk(fr[F.s1() + 2 * q], fr[F.s1() + 2 * q + 1])) * hl + tq;
      }
      const double v = warp_sum(vp);
      __syncwarp();
      for (int t = lane; t < 12 + 24 * NZ; t += 32) {
        // y = sum_ij conj(A_ijm) x[(ij << 1) | k]  (AZ and z_q for a Pc entry); A_ijm at base + 12 ij
        // (AZ_ijm at base + 24 ij), x / z at xb + 2 ij
        const int2 d = ydesc[t];
        const bool pc = d.x >> 30;
        const int base = d.x & 0xffff, step = pc ? 24 : 12;
        const cplx* xz = pc ? wz : wx;
        cplx y = mk(0, 0);
#pragma unroll
        for (int ij = 0; ij < 4; ++ij) {
          const int o = base + step * ij;
          cmac(y, mk(pl[o], -pl[o + 1]), xz[d.y + 2 * ij]);
        }
        if (pc)
          wyz[t - 12] = y;
        else
          wyl[t] = y;
      }
      __syncwarp();
      const bool good = v > 0 && isfinite(v);
      const double scale = good ? sw / v : 0.0;
#pragma unroll
      for (int j = 0; j < SPL; ++j) {
        const int s = lane + 32 * j;
        if (s < n_slot) {
          const int2 d = sdesc[s];
          const double ang = pl[d.x & 0xffff];
          cplx g;
          if (d.x >> 30) {
            g = wyz[d.y] * ang;
          } else {
            const cplx L = mk(fr[d.y & 0xffff], fr[(d.y & 0xffff) + 1]);
            g = conj(L * ang) * wyl[d.y >> 16];
          }
          cmac(acc[j], mk(scale, 0), g);
        }
      }
      if (lane == 0) {
        value += v > 0 ? log(v) * sw : -1e12;
        nbad += good ? 0 : 1;
      }
      __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
      const int s = lane + 32 * j;
      if (s < n_slot) {
        atomicAdd(&grad[(size_t)tl.t * n_slot + s].re, acc[j].re);
        atomicAdd(&grad[(size_t)tl.t * n_slot + s].im, acc[j].im);
      }
    }
    if (lane == 0) {
      atomicAdd(val + tl.t, value);
      if (nbad) atomicAdd(bad + tl.t, nbad);
    }
  }
}

// Per toy (one block each): I = c^H M c, In = c^H Mn c, and the NLL with its gradient in the slots,
//   nll = shift + W_t ln(I / W_mc) - D_t (+1000 when |In / I - 1| > 0.3, as the reference's guard),
//   d nll / d conj(c) = W_t (M c) / I - sum (sw / v) dv / dconj(c).
// out[t]: nll, D_t, I, In; gout[t][s] (optional): the gradient.
__global__ void k_ens_finish(int n_slot, const cplx* __restrict__ M, const cplx* __restrict__ Mn,
                             const cplx* __restrict__ coup, const int* __restrict__ on, const double* __restrict__ val,
                             const cplx* __restrict__ grad, const double* __restrict__ wdata, double w_mc,
                             double shift, double* out, cplx* gout) {
  const int t = blockIdx.x;
  if (!on[t]) return;
  const cplx* c = coup + (size_t)t * n_slot;
  __shared__ double red[2][32];
  double I = 0, In = 0;
  for (int a = threadIdx.x; a < n_slot; a += blockDim.x) {
    cplx mc = mk(0, 0), mnc = mk(0, 0);
    for (int b = 0; b < n_slot; ++b) {
      cmac(mc, M[(size_t)a * n_slot + b], c[b]);
      cmac(mnc, Mn[(size_t)a * n_slot + b], c[b]);
    }
    I += c[a].re * mc.re + c[a].im * mc.im;
    In += c[a].re * mnc.re + c[a].im * mnc.im;
    if (gout) gout[(size_t)t * n_slot + a] = mc;  // M c for now
  }
  I = warp_sum(I);
  In = warp_sum(In);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x / 32] = I;
    red[1][threadIdx.x / 32] = In;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x / 32;
    I = threadIdx.x < nw ? red[0][threadIdx.x] : 0.0;
    In = threadIdx.x < nw ? red[1][threadIdx.x] : 0.0;
    I = warp_sum(I);
    In = warp_sum(In);
    if (threadIdx.x == 0) {
      red[0][0] = I;
      red[1][0] = In;
    }
  }
  __syncthreads();
  I = red[0][0];
  In = red[1][0];
  const double W = wdata[t];
  if (gout) {
    for (int a = threadIdx.x; a < n_slot; a += blockDim.x) {
      const size_t o = (size_t)t * n_slot + a;
      gout[o] = gout[o] * (W / I) - grad[o];
    }
  }
  if (threadIdx.x == 0) {
    double nll = shift + W * log(I / w_mc) - val[t];
    if (fabs(In / I - 1.0) > (double)0.3f) nll += 1000.0;
    out[4 * t] = nll;
    out[4 * t + 1] = val[t];
    out[4 * t + 2] = I;
    out[4 * t + 3] = In;
  }
}

}  // namespace ens
}  // namespace pwa

// ------------------------------------------------------------------ host side
using namespace pwa;
using namespace pwa::ens;

struct pwa_ens {
  CtxView cv;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  PointTable* h_T = nullptr;
  PointTable* d_T = nullptr;
  void* d_tab = nullptr;
  int NR = 0, NZ = 0, NS = 0, n_slot = 0;
  int n_toys = 0;
  std::vector<int64_t> first, count;
  std::vector<double> wdata;
  double w_mc = 0;
  uint8_t* d_kind = nullptr;
  double* d_fac = nullptr;  // factor rows of the data events, [F][nda]
  int64_t ld = 0;
  std::vector<cplx> M, Mn;  // Gram matrices (host copies)
  cplx *d_M = nullptr, *d_Mn = nullptr;
  // launch shape and work list
  int warps = 8, tile_events = 1024, blocks = 0;
  Tile* d_tiles = nullptr;
  int n_tiles = 0;
  // per-call buffers: device and pinned host mirrors
  cplx *d_coup = nullptr, *d_grad = nullptr, *d_gout = nullptr;
  int* d_on = nullptr;
  int* d_next = nullptr;
  double *d_val = nullptr, *d_wdata = nullptr, *d_out = nullptr;
  unsigned long long* d_bad = nullptr;
  cplx *h_coup = nullptr, *h_gout = nullptr;
  int* h_on = nullptr;
  double* h_out = nullptr;
  unsigned long long* h_bad = nullptr;
  double* d_shift = nullptr;
  double shift = 0;
  cudaGraphExec_t graph = nullptr;
  double last_ms = 0, factors_ms = 0, gram_ms = 0;
  std::vector<void*> owned;
};

namespace {

int ens_fail(pwa_ens* s, cudaError_t e);

template <class T>
cudaError_t ens_alloc(pwa_ens* s, T** p, size_t count) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e == cudaSuccess) s->owned.push_back(*p);
  return e;
}

void ens_free(pwa_ens* s) {
  if (!s) return;
  cudaSetDevice(s->cv.device);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  for (void* p : s->owned) cudaFree(p);
  cudaFree(s->d_tiles);
  cudaFreeHost(s->h_T);
  cudaFreeHost(s->h_coup);
  cudaFreeHost(s->h_gout);
  cudaFreeHost(s->h_on);
  cudaFreeHost(s->h_out);
  cudaFreeHost(s->h_bad);
  if (s->e0) cudaEventDestroy(s->e0);
  if (s->e1) cudaEventDestroy(s->e1);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

// m(J/psi p) windows of the 20-offset smearing, on the float mass as the reference tests them.
inline bool in_window(float mz) { return (mz > 4.4 && mz < 4.48) || (mz > 4.27 && mz < 4.34); }

// Event classes as the single-point evaluator's segments give them for toy windows and the MC.
std::vector<uint8_t> event_kinds(const pwa_ens* s, const std::vector<float>& mz, const std::vector<int64_t>& band1,
                                 const std::vector<int64_t>& band2) {
  const int64_t n = s->cv.n, nda = s->cv.nda;
  std::vector<uint8_t> k(n, EK_NONE);
  if (s->cv.gauss) {
    std::fill(k.begin(), k.end(), (uint8_t)EK_GRID);
    return k;
  }
  for (int t = 0; t < s->n_toys; ++t) {
    const int64_t f = s->first[t], wn = s->count[t], a = band1[t], b = band2[t];
    const int64_t b1e = f + std::max<int64_t>(0, std::min(wn, a));
    const int64_t b2e = std::max(b1e, f + std::min(wn, a + b));
    const int64_t r0 = f + std::min(wn, std::max<int64_t>(0, a + b));
    for (int64_t e = f; e < b1e; ++e) k[e] = EK_S30;
    for (int64_t e = b1e; e < b2e; ++e) k[e] = EK_S150;
    for (int64_t e = r0; e < f + wn; ++e) k[e] = in_window(mz[e]) ? EK_S20 : EK_NONE;
  }
  for (int64_t e = nda; e < n; ++e) k[e] = in_window(mz[e]) ? EK_S20 : EK_NONE;
  return k;
}

// Slot index of Lambda* (r, k, m) and of Pc entry at order position q (q, k, m).
inline int slot_l(const pwa_ens* s, int k, int r, int m) { return k * s->NS + r * 6 + m; }
inline int slot_z(const pwa_ens* s, int k, int q, int m) { return k * s->NS + 6 * s->NR + q * 12 + m; }

void table_slots(const pwa_ens* s, const PointTable& T, double* out) {
  for (int k = 0; k < 2; ++k) {
    for (int r = 0; r < s->NR; ++r)
      for (int m = 0; m < 6; ++m) {
        const cplx c = T.L[r].c[k * 6 + m];
        out[2 * slot_l(s, k, r, m)] = c.re;
        out[2 * slot_l(s, k, r, m) + 1] = c.im;
      }
    for (int q = 0; q < s->NZ; ++q)
      for (int m = 0; m < 12; ++m) {
        const cplx c = T.Z[T.order[q]].c[k * 12 + m];
        out[2 * slot_z(s, k, q, m)] = c.re;
        out[2 * slot_z(s, k, q, m) + 1] = c.im;
      }
  }
}

// The Gram entries of active slot pairs a <= b (same proton helicity): kind 0 for M, 1 for the Pc
// part of Mn.
struct EntryRef {
  int a, b, kind;
};
void gram_entries(const pwa_ens* s, const std::vector<uint8_t>& active, std::vector<GramEntry>* ent,
                  std::vector<EntryRef>* ref) {
  const GramBuf G{s->NR, s->NZ};
  const int NR = s->NR, NZ = s->NZ;
  auto add = [&](int a, int b, int kind, int o1, int o2, int o3, int o4) {
    if (!active[a] || !active[b]) return;
    ent->push_back(GramEntry{(int16_t)o1, (int16_t)o2, (int16_t)o3, (int16_t)o4});
    ref->push_back(EntryRef{a, b, kind});
  };
  for (int k = 0; k < 2; ++k) {
    for (int r = 0; r < NR; ++r)
      for (int m = 0; m < 6; ++m) {
        const int a = slot_l(s, k, r, m);
        for (int r2 = 0; r2 < NR; ++r2)
          for (int m2 = 0; m2 < 6; ++m2) {
            const int b = slot_l(s, k, r2, m2);
            if (b >= a) add(a, b, 0, G.ql(k, r, m), G.ql(k, r2, m2), G.pl(m, m2), G.one());
          }
        for (int q = 0; q < NZ; ++q)
          for (int m2 = 0; m2 < 12; ++m2)
            add(a, slot_z(s, k, q, m2), 0, G.ql(k, r, m), G.yz(k, q, m2), G.plz(m, m2), G.one());
      }
    for (int q = 0; q < NZ; ++q)
      for (int m = 0; m < 12; ++m) {
        const int a = slot_z(s, k, q, m);
        for (int q2 = 0; q2 < NZ; ++q2)
          for (int m2 = 0; m2 < 12; ++m2) {
            const int b = slot_z(s, k, q2, m2);
            if (b < a) continue;
            add(a, b, 0, G.dz(k, q, m), G.dz(k, q2, m2), G.pz(m, m2), G.s2(q, q2));
            add(a, b, 1, G.dz(k, q, m), G.dz(k, q2, m2), G.pz(m, m2), G.rn2(q, q2));
          }
      }
  }
}

size_t gram_smem(const pwa_ens* s) {
  return ((sizeof(PointTable) + 15) & ~size_t(15)) + (size_t)GRAM_EB * GramBuf{s->NR, s->NZ}.size() * sizeof(cplx);
}

// Factor rows of the data of every toy, then the Gram matrices over the MC in chunks.
int ens_setup(pwa_ens* s, const std::vector<uint8_t>& active) {
  const CtxView& cv = s->cv;
  cudaError_t e;
  EventSet ev{cv.pp, cv.pp1, cv.pp2, cv.sw, cv.n_size, cv.n, cv.nda};
  const size_t tsm = (sizeof(PointTable) + 15) & ~size_t(15);
  if ((e = cudaFuncSetAttribute(k_ens_factors, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm)))
    return ens_fail(s, e);
  const FactorLayout F{s->NR, s->NZ};
  s->ld = std::max<int64_t>(cv.nda, 1);
  if ((e = ens_alloc(s, &s->d_fac, (size_t)F.size(false) * s->ld))) return ens_fail(s, e);
  cudaEventRecord(s->e0, s->st);
  for (int t = 0; t < s->n_toys; ++t) {
    if (s->count[t] == 0) continue;
    k_ens_factors<<<(unsigned)((s->count[t] + 127) / 128), 128, tsm, s->st>>>(
        s->d_T, ev, s->d_kind, s->first[t], s->count[t], cv.grid, cv.grid_nb, s->d_fac + s->first[t], s->ld, 0);
  }
  cudaEventRecord(s->e1, s->st);
  if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(s->st))) return ens_fail(s, e);
  float ms = 0;
  cudaEventElapsedTime(&ms, s->e0, s->e1);
  s->factors_ms = ms;
  // Gram entries and the chunked accumulation over the MC
  std::vector<GramEntry> ent;
  std::vector<EntryRef> ref;
  gram_entries(s, active, &ent, &ref);
  const int n_ent = (int)ent.size();
  const int64_t n_mc = cv.n - cv.nda;
  s->M.assign((size_t)s->n_slot * s->n_slot, mk(0, 0));
  s->Mn.assign((size_t)s->n_slot * s->n_slot, mk(0, 0));
  if (n_ent > 0 && n_mc > 0) {
    const int64_t CH = std::min<int64_t>(n_mc, 1 << 16);
    const int tiles_y = (n_ent + GRAM_THREADS * GRAM_EPT - 1) / (GRAM_THREADS * GRAM_EPT);
    const int gx = std::max(1, (2 * cv.sm_count + tiles_y - 1) / tiles_y);
    GramEntry* d_ent = nullptr;
    double* d_cf = nullptr;
    cplx *d_part = nullptr, *d_acc = nullptr;
    const size_t smem = gram_smem(s);
    if ((e = cudaFuncSetAttribute(k_ens_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) ||
        (e = cudaMalloc(&d_ent, n_ent * sizeof(GramEntry))) ||
        (e = cudaMalloc(&d_cf, (size_t)F.size(true) * CH * sizeof(double))) ||
        (e = cudaMalloc(&d_part, (size_t)gx * n_ent * sizeof(cplx))) || (e = cudaMalloc(&d_acc, n_ent * sizeof(cplx)))) {
      cudaFree(d_ent);
      cudaFree(d_cf);
      cudaFree(d_part);
      return ens_fail(s, e);
    }
    e = cudaMemcpyAsync(d_ent, ent.data(), n_ent * sizeof(GramEntry), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_acc, 0, n_ent * sizeof(cplx), s->st);
    cudaEventRecord(s->e0, s->st);
    for (int64_t c0 = cv.nda; c0 < cv.n && e == cudaSuccess; c0 += CH) {
      const int64_t cnt = std::min<int64_t>(CH, cv.n - c0);
      k_ens_factors<<<(unsigned)((cnt + 127) / 128), 128, tsm, s->st>>>(s->d_T, ev, s->d_kind, c0, cnt, cv.grid,
                                                                         cv.grid_nb, d_cf, CH, 1);
      k_ens_gram<<<dim3(gx, tiles_y), GRAM_THREADS, smem, s->st>>>(s->d_T, ev, c0, cnt, d_cf, CH, d_ent, n_ent,
                                                                    d_part);
      k_ens_sum_rows<<<(n_ent + 255) / 256, 256, 0, s->st>>>(d_part, gx, n_ent, d_acc);
      e = cudaGetLastError();
    }
    cudaEventRecord(s->e1, s->st);
    std::vector<cplx> acc(n_ent);
    if (e == cudaSuccess) e = cudaMemcpyAsync(acc.data(), d_acc, n_ent * sizeof(cplx), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(d_ent);
    cudaFree(d_cf);
    cudaFree(d_part);
    cudaFree(d_acc);
    if (e) return ens_fail(s, e);
    cudaEventElapsedTime(&ms, s->e0, s->e1);
    s->gram_ms = ms;
    const int n = s->n_slot;
    for (int j = 0; j < n_ent; ++j) {
      const EntryRef& r = ref[j];
      std::vector<cplx>& dst = r.kind == 0 ? s->M : s->Mn;
      dst[(size_t)r.a * n + r.b] = acc[j];
      dst[(size_t)r.b * n + r.a] = conj(acc[j]);
      // the Lambda* block of Mn is that of M (no Lambda* - Pc term without interference)
      const bool both_l = (r.a % s->NS) < 6 * s->NR && (r.b % s->NS) < 6 * s->NR;
      if (r.kind == 0 && both_l) {
        s->Mn[(size_t)r.a * n + r.b] = acc[j];
        s->Mn[(size_t)r.b * n + r.a] = conj(acc[j]);
      }
    }
  }
  if ((e = cudaMemcpyAsync(s->d_M, s->M.data(), s->M.size() * sizeof(cplx), cudaMemcpyHostToDevice, s->st)) ||
      (e = cudaMemcpyAsync(s->d_Mn, s->Mn.data(), s->Mn.size() * sizeof(cplx), cudaMemcpyHostToDevice, s->st)) ||
      (e = cudaStreamSynchronize(s->st)))
    return ens_fail(s, e);
  return PWA_OK;
}

int ens_fail(pwa_ens*, cudaError_t e) { return cuda_fail(e); }

// The work list for the current tile size.
int ens_tiles(pwa_ens* s) {
  std::vector<Tile> tl;
  for (int t = 0; t < s->n_toys; ++t)
    for (int64_t e0 = s->first[t]; e0 < s->first[t] + s->count[t]; e0 += s->tile_events)
      tl.push_back(Tile{e0, std::min(e0 + s->tile_events, s->first[t] + s->count[t]), t, 0});
  cudaFree(s->d_tiles);
  s->d_tiles = nullptr;
  s->n_tiles = (int)tl.size();
  cudaError_t e = cudaMalloc(&s->d_tiles, std::max<size_t>(tl.size(), 1) * sizeof(Tile));
  if (e == cudaSuccess && !tl.empty())
    e = cudaMemcpy(s->d_tiles, tl.data(), tl.size() * sizeof(Tile), cudaMemcpyHostToDevice);
  if (e) return cuda_fail(e);
  return PWA_OK;
}

// Kernel instance for a launch shape and slot count (slots per lane 8, 12, 16 or 21).
template <int W, int SPL>
cudaError_t data_t(pwa_ens* s, bool launch, size_t smem, int* occ) {
  if (!launch) {
    cudaError_t e = cudaFuncSetAttribute(k_ens_data<W, SPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k_ens_data<W, SPL>, W * 32, smem);
    return e;
  }
  const EventSet ev{s->cv.pp, s->cv.pp1, s->cv.pp2, s->cv.sw, s->cv.n_size, s->cv.n, s->cv.nda};
  k_ens_data<W, SPL><<<s->blocks, W * 32, smem, s->st>>>(s->d_T, ev, s->d_fac, s->ld, s->d_tiles, s->n_tiles,
                                                         s->d_next, s->d_coup, s->d_on, s->n_slot,
                                                         ens_scratch(s->NR, s->NZ), s->d_val, s->d_grad, s->d_bad);
  return cudaGetLastError();
}

template <int W>
cudaError_t data_w(pwa_ens* s, bool launch, size_t smem, int* occ) {
  const int spl = (s->n_slot + 31) / 32;
  if (spl <= 8) return data_t<W, 8>(s, launch, smem, occ);
  if (spl <= 12) return data_t<W, 12>(s, launch, smem, occ);
  if (spl <= 16) return data_t<W, 16>(s, launch, smem, occ);
  return data_t<W, 21>(s, launch, smem, occ);
}

// Configures (launch = false: shared-memory size, occupancy into *occ) or launches the data kernel.
cudaError_t data_kernel(pwa_ens* s, bool launch, int* occ = nullptr) {
  const size_t smem = ens_data_smem(s->warps, s->n_slot, s->NZ, ens_scratch(s->NR, s->NZ));
  switch (s->warps) {
    case 4: return data_w<4>(s, launch, smem, occ);
    case 8: return data_w<8>(s, launch, smem, occ);
    case 12: return data_w<12>(s, launch, smem, occ);
    default: return data_w<16>(s, launch, smem, occ);
  }
}

// Captures one ensemble step (inputs in, both kernels, results out) into a CUDA graph.
int ens_capture(pwa_ens* s) {
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  const size_t nc = (size_t)s->n_toys * s->n_slot;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal);
  if (e) return cuda_fail(e);
  cudaMemcpyAsync(s->d_coup, s->h_coup, nc * sizeof(cplx), cudaMemcpyHostToDevice, s->st);
  cudaMemcpyAsync(s->d_on, s->h_on, s->n_toys * sizeof(int), cudaMemcpyHostToDevice, s->st);
  cudaMemsetAsync(s->d_val, 0, s->n_toys * sizeof(double), s->st);
  cudaMemsetAsync(s->d_bad, 0, s->n_toys * sizeof(unsigned long long), s->st);
  cudaMemsetAsync(s->d_grad, 0, nc * sizeof(cplx), s->st);
  cudaMemsetAsync(s->d_next, 0, sizeof(int), s->st);
  cudaError_t le = data_kernel(s, true);
  k_ens_finish<<<s->n_toys, 256, 0, s->st>>>(s->n_slot, s->d_M, s->d_Mn, s->d_coup, s->d_on, s->d_val, s->d_grad,
                                             s->d_wdata, s->w_mc, s->shift, s->d_out, s->d_gout);
  cudaMemcpyAsync(s->h_out, s->d_out, 4 * s->n_toys * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  cudaMemcpyAsync(s->h_gout, s->d_gout, nc * sizeof(cplx), cudaMemcpyDeviceToHost, s->st);
  cudaMemcpyAsync(s->h_bad, s->d_bad, s->n_toys * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->st);
  e = cudaStreamEndCapture(s->st, &g);
  if (le && !e) e = le;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s->graph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e) {
    s->graph = nullptr;
    return cuda_fail(e);
  }
  return PWA_OK;
}

}  // namespace

extern "C" {

int pwa_ens_set_launch(pwa_ens* s, int warps, int tile_events);

int pwa_ens_create(pwa_ctx* ctx, const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                   int NX, float FFR, float FFB, int n_toys, const int64_t* first, const int64_t* count,
                   const int64_t* nda_smr, const int64_t* nda_fine, const double* sum_w_data, double sum_w_mc,
                   const uint8_t* active, pwa_ens** out) {
  if (!ctx || !pl || !out || n_toys < 1 || !first || !count || !nda_smr || !nda_fine || !sum_w_data) return PWA_E_ARG;
  *out = nullptr;
  if (NX > 0) return PWA_E_UNSUPPORTED;
  pwa_ens* s = new pwa_ens();
  int rc = ctx_view(ctx, &s->cv);
  if (rc) {
    delete s;
    return rc;
  }
  const CtxView& cv = s->cv;
  for (int t = 0; t < n_toys; ++t)
    if (first[t] < 0 || count[t] < 0 || first[t] + count[t] > cv.nda) {
      delete s;
      return PWA_E_ARG;
    }
  s->n_toys = n_toys;
  s->first.assign(first, first + n_toys);
  s->count.assign(count, count + n_toys);
  s->wdata.assign(sum_w_data, sum_w_data + n_toys);
  s->w_mc = sum_w_mc;
  cudaError_t e = cudaSetDevice(cv.device);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cv.st);  // the context's work on its events is done
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_T, sizeof(PointTable));
  if (e) {
    ens_free(s);
    return cuda_fail(e);
  }
  if ((rc = build_point_table(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, s->h_T, cv.build_flags))) {
    ens_free(s);
    return rc;
  }
  s->NR = NR;
  s->NZ = NZ;
  s->NS = 6 * NR + 12 * NZ;
  s->n_slot = 2 * s->NS;
  if ((e = ens_alloc(s, &s->d_T, 1))) {
    ens_free(s);
    return cuda_fail(e);
  }
  if (cv.use_tables) {
    if ((e = ens_alloc(s, reinterpret_cast<uint8_t**>(&s->d_tab), TAB_BYTES))) {
      ens_free(s);
      return cuda_fail(e);
    }
    attach_tables(s->h_T, s->d_tab);
  }
  e = cudaMemcpyAsync(s->d_T, s->h_T, sizeof(PointTable), cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess && s->h_T->tab.enabled) e = launch_build_tables(s->d_T, TAB_NODES, cv.sm_count, s->st);
  // event classes (the float m(J/psi p) plane decides the window, as in the reference)
  std::vector<float> mz(cv.n);
  if (e == cudaSuccess && cv.n)
    e = cudaMemcpyAsync(mz.data(), cv.pp + cv.n_size, cv.n * sizeof(float), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e) {
    ens_free(s);
    return cuda_fail(e);
  }
  const std::vector<uint8_t> kinds =
      event_kinds(s, mz, std::vector<int64_t>(nda_smr, nda_smr + n_toys), std::vector<int64_t>(nda_fine, nda_fine + n_toys));
  const size_t nc = (size_t)n_toys * s->n_slot;
  if ((e = ens_alloc(s, &s->d_kind, cv.n)) ||
      (e = cudaMemcpy(s->d_kind, kinds.data(), cv.n, cudaMemcpyHostToDevice)) ||
      (e = ens_alloc(s, &s->d_M, (size_t)s->n_slot * s->n_slot)) ||
      (e = ens_alloc(s, &s->d_Mn, (size_t)s->n_slot * s->n_slot)) || (e = ens_alloc(s, &s->d_coup, nc)) ||
      (e = ens_alloc(s, &s->d_grad, nc)) || (e = ens_alloc(s, &s->d_gout, nc)) ||
      (e = ens_alloc(s, &s->d_on, n_toys)) || (e = ens_alloc(s, &s->d_next, 1)) ||
      (e = ens_alloc(s, &s->d_val, n_toys)) || (e = ens_alloc(s, &s->d_wdata, n_toys)) ||
      (e = ens_alloc(s, &s->d_out, 4 * (size_t)n_toys)) || (e = ens_alloc(s, &s->d_bad, n_toys)) ||
      (e = cudaMemcpy(s->d_wdata, sum_w_data, n_toys * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMallocHost(&s->h_coup, nc * sizeof(cplx))) || (e = cudaMallocHost(&s->h_gout, nc * sizeof(cplx))) ||
      (e = cudaMallocHost(&s->h_on, n_toys * sizeof(int))) ||
      (e = cudaMallocHost(&s->h_out, 4 * (size_t)n_toys * sizeof(double))) ||
      (e = cudaMallocHost(&s->h_bad, n_toys * sizeof(unsigned long long)))) {
    ens_free(s);
    return cuda_fail(e);
  }
  std::vector<uint8_t> act(s->n_slot, 1);
  if (active) act.assign(active, active + s->n_slot);
  if ((rc = ens_setup(s, act))) {
    ens_free(s);
    return rc;
  }
  if ((rc = pwa_ens_set_launch(s, s->warps, s->tile_events))) {
    ens_free(s);
    return rc;
  }
  *out = s;
  return PWA_OK;
}

int pwa_ens_destroy(pwa_ens* s) {
  ens_free(s);
  return PWA_OK;
}

int pwa_ens_slot_count(const pwa_ens* s) { return s ? s->n_slot : 0; }

int pwa_ens_slots(const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX, float FFR,
                  float FFB, double* h_slots) {
  if (!pl || !h_slots) return PWA_E_ARG;
  if (NX != 0) return PWA_E_UNSUPPORTED;
  PointTable* T = new PointTable();
  const int rc = build_point_table(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, T);
  if (!rc) {
    pwa_ens shape;
    shape.NR = NR;
    shape.NZ = NZ;
    shape.NS = 6 * NR + 12 * NZ;
    table_slots(&shape, *T, h_slots);
  }
  delete T;
  return rc;
}

int pwa_ens_gram(const pwa_ens* s, double* h_M, double* h_Mn) {
  if (!s) return PWA_E_ARG;
  if (h_M) std::memcpy(h_M, s->M.data(), s->M.size() * sizeof(cplx));
  if (h_Mn) std::memcpy(h_Mn, s->Mn.data(), s->Mn.size() * sizeof(cplx));
  return PWA_OK;
}

int pwa_ens_set_launch(pwa_ens* s, int warps, int tile_events) {
  if (!s || (warps != 4 && warps != 8 && warps != 12 && warps != 16) || tile_events < 32) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(s->cv.device);
  if (e) return cuda_fail(e);
  // a shape whose shared memory does not fit one block is refused and the current shape kept
  int max_smem = 0;
  if ((e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->cv.device)))
    return cuda_fail(e);
  if (ens_data_smem(warps, s->n_slot, s->NZ, ens_scratch(s->NR, s->NZ)) > (size_t)max_smem) return PWA_E_SIZE;
  const int old_warps = s->warps, old_tile = s->tile_events;
  s->warps = warps;
  s->tile_events = tile_events;
  int occ = 1;
  e = data_kernel(s, false, &occ);
  if (e) {
    s->warps = old_warps;
    s->tile_events = old_tile;
    cudaGetLastError();
    return cuda_fail(e);
  }
  s->blocks = s->cv.sm_count * std::max(occ, 1);
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  return ens_tiles(s);
}

int pwa_ens_eval(pwa_ens* s, const double* h_slots, const int* h_on, double nll_shift, double* h_out, double* h_grad,
                 int64_t* h_bad) {
  if (!s || !h_slots || !h_out) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(s->cv.device);
  if (e) return cuda_fail(e);
  if (!s->graph || nll_shift != s->shift) {
    s->shift = nll_shift;
    const int rc = ens_capture(s);
    if (rc) return rc;
  }
  const size_t nc = (size_t)s->n_toys * s->n_slot;
  std::memcpy(s->h_coup, h_slots, nc * sizeof(cplx));
  for (int t = 0; t < s->n_toys; ++t) s->h_on[t] = h_on ? (h_on[t] != 0) : 1;
  if ((e = cudaEventRecord(s->e0, s->st)) || (e = cudaGraphLaunch(s->graph, s->st)) ||
      (e = cudaEventRecord(s->e1, s->st)) || (e = cudaStreamSynchronize(s->st)))
    return cuda_fail(e);
  float ms = 0;
  cudaEventElapsedTime(&ms, s->e0, s->e1);
  s->last_ms = ms;
  for (int t = 0; t < s->n_toys; ++t) {
    if (!s->h_on[t]) continue;
    for (int j = 0; j < 4; ++j) h_out[4 * t + j] = s->h_out[4 * t + j];
    if (h_bad) h_bad[t] = (int64_t)s->h_bad[t];
    if (h_grad) std::memcpy(h_grad + 2 * (size_t)t * s->n_slot, s->h_gout + (size_t)t * s->n_slot, s->n_slot * sizeof(cplx));
  }
  return PWA_OK;
}

double pwa_ens_last_ms(const pwa_ens* s) { return s ? s->last_ms : 0.0; }

int pwa_ens_setup_ms(const pwa_ens* s, double* factors_ms, double* gram_ms) {
  if (!s) return PWA_E_ARG;
  if (factors_ms) *factors_ms = s->factors_ms;
  if (gram_ms) *gram_ms = s->gram_ms;
  return PWA_OK;
}

}  // extern "C"
