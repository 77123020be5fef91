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
  const int64_t i_begin = (int64_t)blockIdx.x * per, i_end = min(count, i_begin + per);
  for (int64_t i0 = i_begin; i0 < i_end; i0 += GRAM_EB) {
    const int ne = (int)min<int64_t>(GRAM_EB, i_end - i0);
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
