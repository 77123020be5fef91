// Batched NLL evaluation at many parameter points in one pass over the events.
//
// Minuit's numerical gradient evaluates the likelihood at a centre point and at 2N points that each
// move one parameter.  A moved parameter touches one part of the amplitude: the couplings or the
// lineshape of one Lambda* (or the Lambda* scale shared by all of them), the couplings of one set of
// Pc entries, or the lineshapes of one Pc group (a K-matrix J^P group or one Breit-Wigner Pc).  Per
// event the centre is evaluated once and every point is formed from it by exact FP64 algebra on the
// difference of its float parameter block and the centre's:
//   Lambda* point:  H_L[h] += q_r^p f_r^p[h] - q_r^0 f_r^0[h] for the changed resonances r
//                   (f_r[h] = sum_m c_rkm A_ijm DL_rkm, q_r the lineshape); the Pc sums stay.
//   Pc couplings:   S_b[h] += sum_{q in Q} R_q(m_b) dHZ_q[h], dHZ_q[h] = sum_m dc_qkm AZ_ijm DZ_qkm,
//                   at every resolution offset b (R_q the entry lineshape, from the centre).
//   Pc lineshapes:  S_b[h] += sum_{q in g} (R_q^p(m_b) - R_q^0(m_b)) HZ_q[h], R^p from the point's own
//                   lineshape table.
// |A|^2 then follows as in the single-point kernels: sum_h |H_L + S_0|^2 for unsmeared events, and
// sum_h |H_L|^2 + 2 w Re(conj(H_L) sum_b S_b) + w^2 u sum_b |S_b|^2 for smeared ones (the reference's
// BW1/BW2 form, kernel_calEva.cu:676-810).  Points that differ from the centre in anything else are
// evaluated by the single-point path.
//
// Work split: one warp per event.  The warp stages the event's 303 basis planes in shared memory,
// evaluates the centre (Lambda* terms, Pc angular amplitudes HZ_q[h], the entry lineshapes R at up to
// 32 masses per round and S_b[h] = sum_q R_q(m_b) HZ_q[h]), then each lane takes one parameter point.
// Per-point results go to per-block FP64 sums; a finalize kernel reduces them per point.
#include <cstring>
#include <vector>

#include "pwa_device.cuh"

namespace pwa {

constexpr int BATCH_WARPS = 4;
constexpr int BATCH_THREADS = BATCH_WARPS * 32;
constexpr int BATCH_MAXQ = 8;  // Pc entries per coupling point
constexpr int N_PLANES = 303;  // pp 111 + pp1 96 + pp2 96

// Per-warp shared-memory layout of the batched kernel for a model with NR Lambda* and NZ Pc entries.
struct BatchLayout {
  int nzp, rs;  // Pc entries rounded up to 4; row stride of R (odd, conflict-free row writes)
  size_t bs, lk, q0, f0, hl0, a10, a20, hz, R, S0, vbuf, warp_bytes, acc, total;
};
__host__ __device__ inline size_t bal16(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline BatchLayout batch_layout(int NR, int NZ, int npts) {
  BatchLayout L;
  L.nzp = (NZ + 3) & ~3;
  L.rs = L.nzp + 1;
  size_t o = 0;
  L.bs = o;
  o = bal16(o + N_PLANES * sizeof(double));
  L.lk = o;
  o = bal16(o + sizeof(LstarKin));
  L.q0 = o;
  o = bal16(o + (size_t)(NR > 0 ? NR : 1) * sizeof(cplx));
  L.f0 = o;
  o = bal16(o + (size_t)(NR > 0 ? NR : 1) * 8 * sizeof(cplx));
  L.hl0 = o;
  o = bal16(o + 8 * sizeof(cplx));
  L.a10 = o;
  o = bal16(o + 8 * sizeof(cplx));
  L.a20 = o;
  o = bal16(o + 8 * sizeof(double));
  L.hz = o;
  o = bal16(o + (size_t)(L.nzp > 0 ? L.nzp : 1) * 8 * sizeof(cplx));
  L.R = o;
  o = bal16(o + (size_t)32 * L.rs * sizeof(cplx));
  L.S0 = o;
  o = bal16(o + (size_t)32 * 9 * sizeof(cplx));
  L.vbuf = o;
  o = bal16(o + (size_t)npts * 2 * sizeof(double));
  L.warp_bytes = o;
  L.acc = BATCH_WARPS * L.warp_bytes;
  L.total = L.acc + (size_t)npts * 4 * sizeof(double);
  return L;
}

// Event accessors on the staged planes.
struct StagedEv {
  const double* s;
  __device__ __forceinline__ double mkp() const { return s[0]; }
  __device__ __forceinline__ double mz() const { return s[1]; }
  __device__ __forceinline__ float w() const { return s[2]; }
  __device__ __forceinline__ cplx A(int i, int j, int m) const {
    const int a = 3 + (i * 12 + j * 6 + m) * 2;
    return mk(s[a], s[a + 1]);
  }
  __device__ __forceinline__ double DL(int sx, int k, int m) const { return s[51 + sx * 12 + k * 6 + m]; }
  __device__ __forceinline__ cplx AZ(int i, int j, int m) const {
    const int a = 111 + (i * 24 + j * 12 + m) * 2;
    return mk(s[a], s[a + 1]);
  }
  __device__ __forceinline__ double DZ(int sx, int k, int m) const { return s[207 + sx * 24 + k * 12 + m]; }
};

// f_r[h] = sum_m c_rkm A_ijm DL_{s_r,k,m} for helicity h = (i, j, k).
__device__ __forceinline__ cplx lstar_angular(const LstarEntry& L, const StagedEv& E, int h) {
  const int i = h >> 2, j = (h >> 1) & 1, k = h & 1;
  cplx f = mk(0, 0);
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const cplx c = L.c[k * 6 + m];
    if (nonzero(c)) cmac(f, c, E.A(i, j, m) * E.DL(L.sidx, k, m));
  }
  return f;
}

// sum_m c_m AZ_ijm DZ_{sx,k,m} for helicity h and a 24-slot coupling array c[k * 12 + m].
__device__ __forceinline__ cplx pc_angular(const cplx* c, int sx, const StagedEv& E, int h) {
  const int i = h >> 2, j = (h >> 1) & 1, k = h & 1;
  cplx v = mk(0, 0);
#pragma unroll
  for (int m = 0; m < 12; ++m) {
    const cplx cc = c[k * 12 + m];
    if (nonzero(cc)) cmac(v, cc, E.AZ(i, j, m) * E.DZ(sx, k, m));
  }
  return v;
}

// Lineshape of every entry of group g at mass m from the point's table (false when it cannot serve
// m), or exactly.
template <bool FIX>
__device__ __forceinline__ bool group_lineshapes(const PointTable& T, int g, double m, cplx (&out)[MAX_GROUP_ENTRIES]) {
  const PcGroup& gr = T.grp[g];
  const int first = gr.first, cnt = gr.count;
  TabAt ta;
  if (tab_at(T.tab, m, ta)) {
#pragma unroll
    for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) {
      if (q >= cnt) break;
      out[q] = tab_get(ta, T.tab.stride, first + q);
    }
    return true;
  }
  if (!FIX) return false;
  cplx ex[MAX_GROUP_ENTRIES];
  pc_group_exact(T, g, pc_kin(T, m), ex);
#pragma unroll
  for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) {
    if (q >= cnt) break;
    out[q] = ex[q];
  }
  return true;
}

// sum_m c[k * 6 + m] A_ijm DL_{sx,k,m} for helicity h (c: a Lambda* coupling array).
__device__ __forceinline__ cplx lstar_angular_c(const cplx* c, int sx, const StagedEv& E, int h) {
  const int i = h >> 2, j = (h >> 1) & 1, k = h & 1;
  cplx f = mk(0, 0);
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const cplx cc = c[k * 6 + m];
    if (nonzero(cc)) cmac(f, cc, E.A(i, j, m) * E.DL(sx, k, m));
  }
  return f;
}

template <int NB>
__device__ __forceinline__ const float* batch_offsets() {
  if constexpr (NB == 0) {
    return nullptr;
  } else {
    return smear_table<NB>();
  }
}

// NB > 0: NB resolution offsets (the reference's quantile schemes); band 0 (tail window events) adds
// row 0 at the event mass for the non-interfering MC term, band 1 (data bands) does not.  NB = 0: the
// weighted grid scheme of the Gaussian resolution model (grid[2b] absolute offset, grid[2b+1] weight,
// grid_nb offsets, band 0).  FIX = false: table lookups only, events with a mass no table can serve (centre or a
// lineshape point's) are appended to defer[]; FIX = true evaluates those masses exactly and runs over
// the deferred list (events [0, *n_list)) or, without tables, over the whole segment.
template <int NB, bool FIX>
__global__ void __launch_bounds__(BATCH_THREADS)
    k_batch(EventSet ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
            const PointTable* __restrict__ T0p, const BatchPoint* __restrict__ pts, int npts, Partial* parts,
            int band, int32_t* defer, int* defer_count, const double* __restrict__ grid, int grid_nb) {
  extern __shared__ __align__(16) unsigned char sm[];
  const PointTable& T0 = *T0p;
  const int NR = T0.NR, NZ = T0.NZ;
  const BatchLayout Ly = batch_layout(NR, NZ, npts);
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  unsigned char* wb = sm + warp * Ly.warp_bytes;
  double* bs = reinterpret_cast<double*>(wb + Ly.bs);
  LstarKin* lks = reinterpret_cast<LstarKin*>(wb + Ly.lk);  // the event's Lambda* kinematics
  cplx* q0 = reinterpret_cast<cplx*>(wb + Ly.q0);
  cplx* f0 = reinterpret_cast<cplx*>(wb + Ly.f0);  // [r][h]
  cplx* hl0 = reinterpret_cast<cplx*>(wb + Ly.hl0);
  cplx* a10 = reinterpret_cast<cplx*>(wb + Ly.a10);
  double* a20 = reinterpret_cast<double*>(wb + Ly.a20);
  cplx* hz = reinterpret_cast<cplx*>(wb + Ly.hz);  // [q][h]
  cplx* R = reinterpret_cast<cplx*>(wb + Ly.R);    // [row][q], stride Ly.rs
  cplx* S0 = reinterpret_cast<cplx*>(wb + Ly.S0);  // [row][h], stride 9
  double* vbuf = reinterpret_cast<double*>(wb + Ly.vbuf);
  double* acc = reinterpret_cast<double*>(sm + Ly.acc);  // [p][4]
  for (int i = threadIdx.x; i < npts * 4; i += BATCH_THREADS) acc[i] = 0.0;
  __syncthreads();

  const StagedEv E{bs};
  const int h8 = lane & 7, part = lane >> 3;
  const float* qoff = batch_offsets<NB>();
  constexpr bool GRID = NB == 0;
  const float wf = (float)(1.0 / (NB > 0 ? NB : 1));
  const double wgt = GRID ? 1.0 : (double)wf;
  const double c2 = GRID ? 1.0 : wgt * wgt * (double)(1.0f / wf);
  const int shift = band == 0 ? 1 : 0;  // row 0 at the event mass
  const int nlook = (GRID ? grid_nb : NB) + shift;
  // mass and weight of lookup row l (row l < shift: the event mass)
  auto row_mass = [&](int l, double mz, double mres) {
    const int b = l - shift;
    return b < 0 ? mz : GRID ? mz + __ldg(grid + 2 * b) : mz + (double)qoff[b] * mres;
  };
  auto row_weight = [&](int l) { return GRID ? __ldg(grid + 2 * (l - shift) + 1) : 1.0; };
  const int nrounds = (nlook + 31) / 32;
  const int nzp = Ly.nzp, rs = Ly.rs;

  if (n_list) end = begin + *n_list;
  const int64_t count = end - begin;
  int64_t c0, c1, w0, wstep;
  if (n_list) {
    c0 = 0;
    c1 = count;
    w0 = (int64_t)blockIdx.x * BATCH_WARPS + warp;
    wstep = (int64_t)gridDim.x * BATCH_WARPS;
  } else {
    int64_t chunk = (count + gridDim.x - 1) / gridDim.x;
    c0 = (int64_t)blockIdx.x * chunk;
    c1 = min(count, c0 + chunk);
    w0 = warp;
    wstep = BATCH_WARPS;
  }

  for (int64_t p = c0 + w0; p < c1; p += wstep) {
    const int64_t e = event_index(list, begin, p);
    for (int i = lane; i < N_PLANES; i += 32) {
      const float* src = i < 111 ? ev.pp + (int64_t)i * ev.n_size
                                 : (i < 207 ? ev.pp1 + (int64_t)(i - 111) * ev.n_size
                                            : ev.pp2 + (int64_t)(i - 207) * ev.n_size);
      bs[i] = (double)__ldg(src + e);
    }
    __syncwarp();
    const double mkp = E.mkp(), mz = E.mz();
    const double mres = MRES0 + mz * (MRES1 + mz * MRES2);
    // centre: Lambda* lineshapes, f_r[h], H_L[h]; Pc angular amplitudes HZ_q[h]
    if (lane < NR || lane == 0) {
      const LstarKin lk = lstar_kin(T0, mkp);
      if (lane < NR) q0[lane] = lstar_lineshape(T0.L[lane], lk);
      if (lane == 0) *lks = lk;
    }
    __syncwarp();
    {
      cplx hl = mk(0, 0);
      for (int r = part; r < NR; r += 4) {
        const cplx f = lstar_angular(T0.L[r], E, h8);
        f0[r * 8 + h8] = f;
        cmac(hl, q0[r], f);
      }
      hl += shfl_xor(hl, 8);
      hl += shfl_xor(hl, 16);
      if (part == 0) hl0[h8] = hl;
      for (int q = part; q < nzp; q += 4)
        hz[q * 8 + h8] = q < NZ ? pc_angular(T0.Z[T0.order[q]].c, T0.Z[T0.order[q]].sidx, E, h8) : mk(0, 0);
    }
    __syncwarp();
    bool fail = false;
    // one round of centre rows: R[b][q] at lookup l0 + b, S0[b][h]; the centre's smeared sums
    auto centre_round = [&](int l0, bool sums) {
      const int l = l0 + lane;
      cplx* row = R + lane * rs;
      if (l < nlook) {
        const double m = row_mass(l, mz, mres);
        if (FIX)
          lookup_entries(T0, m, row);
        else
          fail |= !lookup_table(T0, m, row);
      } else {
        for (int q = 0; q < NZ; ++q) row[q] = mk(0, 0);
      }
      for (int q = NZ; q < nzp; ++q) row[q] = mk(0, 0);
      __syncwarp();
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        cplx s = mk(0, 0);
        for (int q = 0; q < NZ; ++q) cmac(s, row[q], hz[q * 8 + h]);
        S0[lane * 9 + h] = s;
      }
      __syncwarp();
      if (sums) {
        // lane (h, part) sums the offset rows b = part, part + 4, ... of this round
        cplx a1 = mk(0, 0);
        double a2 = 0;
        for (int b = part; b < 32; b += 4) {
          const int ll = l0 + b;
          if (ll < shift || ll >= nlook) continue;
          const cplx s = S0[b * 9 + h8];
          const double wb = row_weight(ll);
          a1 += wb * s;
          a2 += wb * norm2(s);
        }
        a1 += shfl_xor(a1, 8);
        a1 += shfl_xor(a1, 16);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 8);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 16);
        if (part == 0) {
          a10[h8] = (l0 == 0 ? mk(0, 0) : a10[h8]) + a1;
          a20[h8] = (l0 == 0 ? 0.0 : a20[h8]) + a2;
        }
        __syncwarp();
      }
    };
    // the centre's sums over all offset rows first; with several rounds the rows are recomputed
    // below only in passes whose points read them
    for (int rd = 0; rd < nrounds; ++rd) centre_round(rd * 32, true);
    const bool centre_fail = !FIX && __any_sync(0xffffffffu, fail);
    if (!centre_fail) {
      for (int pass = 0; pass < npts; pass += 32) {
        const int pidx = pass + lane;
        const bool act = pidx < npts;
        const BatchPoint& bp = pts[act ? pidx : 0];
        const int kind = act ? bp.kind : BP_SAME;
        const bool own = kind == BP_PCC || kind == BP_PCG;  // sums over the rows are the point's own
        cplx a1[8];
        double a2[8];
        double vns = 0;  // sum_h |S_0[h]|^2 at the event mass (non-interfering term, smeared band 0)
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          a1[h] = mk(0, 0);
          a2[h] = 0;
        }
        const bool need_rows = nrounds == 1 || __any_sync(0xffffffffu, kind == BP_PCC || kind == BP_PCG);
        for (int rd = 0; need_rows && rd < nrounds; ++rd) {
          const int l0 = rd * 32;
          if (nrounds > 1) centre_round(l0, false);
          const int rows = min(32, nlook - l0);
          if (kind == BP_PCC) {
            const int nq = bp.nq;
#pragma unroll
            for (int h = 0; h < 8; ++h) {
              cplx d[BATCH_MAXQ];
              int pos[BATCH_MAXQ];
#pragma unroll
              for (int u = 0; u < BATCH_MAXQ; ++u) {
                if (u >= nq) break;
                pos[u] = bp.qpos[u];
                d[u] = pc_angular(bp.dc + u * 24, bp.qsidx[u], E, h);
              }
              for (int b = 0; b < rows; ++b) {
                cplx sv = S0[b * 9 + h];
#pragma unroll
                for (int u = 0; u < BATCH_MAXQ; ++u) {
                  if (u >= nq) break;
                  cmac(sv, R[b * rs + pos[u]], d[u]);
                }
                if (l0 + b < shift) {
                  vns += norm2(sv);
                } else {
                  const double wb = row_weight(l0 + b);
                  a1[h] += wb * sv;
                  a2[h] += wb * norm2(sv);
                }
              }
            }
          } else if (kind == BP_PCG) {
            const PointTable& Tp = *bp.T;
            const int g = bp.group;
            const int first = Tp.grp[g].first, cnt = Tp.grp[g].count;
            for (int b = 0; b < rows; ++b) {
              const int l = l0 + b;
              const double m = row_mass(l, mz, mres);
              cplx dr[MAX_GROUP_ENTRIES];
              if (!group_lineshapes<FIX>(Tp, g, m, dr)) {
                fail = true;
#pragma unroll
                for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) dr[q] = mk(0, 0);
              }
#pragma unroll
              for (int q = 0; q < MAX_GROUP_ENTRIES; ++q)
                if (q < cnt) dr[q] -= R[b * rs + first + q];
                else break;
#pragma unroll
              for (int h = 0; h < 8; ++h) {
                cplx sv = S0[b * 9 + h];
#pragma unroll
                for (int q = 0; q < MAX_GROUP_ENTRIES; ++q)
                  if (q < cnt) cmac(sv, dr[q], hz[(first + q) * 8 + h]);
                  else break;
                if (l < shift) {
                  vns += norm2(sv);
                } else {
                  const double wb = row_weight(l);
                  a1[h] += wb * sv;
                  a2[h] += wb * norm2(sv);
                }
              }
            }
          }
        }
        // the point's Lambda* amplitudes, then |A|^2 with and without interference
        if (act) {
          cplx hlp[8];
#pragma unroll
          for (int h = 0; h < 8; ++h) hlp[h] = hl0[h];
          if (kind == BP_LSTAR) {
            // the kinematic inputs of the lineshapes (barrier orders, radii) equal the centre's
            const PointTable& Tp = *bp.T;
            const LstarKin& lk = *lks;
            const unsigned lm = bp.lmask, lsm = bp.lsmask, lcm = bp.lcmask;
            int u = 0;
            for (int r = 0; r < NR; ++r) {
              if (!(lm >> r & 1)) continue;
              const bool ls = lsm >> r & 1, cc = lcm >> r & 1;
              if (!ls && cc && bp.ldc) {  // couplings only: q_r * f(dc)
                const cplx* dc = bp.dc + 24 * u++;
#pragma unroll
                for (int h = 0; h < 8; ++h) cmac(hlp[h], q0[r], lstar_angular_c(dc, T0.L[r].sidx, E, h));
              } else {
                if (cc) ++u;
                const cplx qp = lstar_lineshape(Tp.L[r], lk);
                if (!cc) {  // lineshape only: (q^p - q^0) f_r
                  const cplx dq = qp - q0[r];
#pragma unroll
                  for (int h = 0; h < 8; ++h) cmac(hlp[h], dq, f0[r * 8 + h]);
                } else {
#pragma unroll
                  for (int h = 0; h < 8; ++h) {
                    cmac(hlp[h], qp, lstar_angular(Tp.L[r], E, h));
                    cmac(hlp[h], mk(-q0[r].re, -q0[r].im), f0[r * 8 + h]);
                  }
                }
              }
            }
          }
          if (!own && shift) {
#pragma unroll
            for (int h = 0; h < 8; ++h) vns += norm2(S0[h]);
          }
          double v = 0, vn = vns;
#pragma unroll
          for (int h = 0; h < 8; ++h) {
            const cplx s1 = own ? a1[h] : a10[h];
            const double s2 = own ? a2[h] : a20[h];
            v += norm2(hlp[h]) + 2.0 * wgt * (hlp[h].re * s1.re + hlp[h].im * s1.im) + c2 * s2;
            vn += norm2(hlp[h]);
          }
          vbuf[pidx * 2] = v;
          vbuf[pidx * 2 + 1] = vn;
        }
      }
    }
    const bool deferred = !FIX && (centre_fail || __any_sync(0xffffffffu, fail));
    if (deferred) {
      if (lane == 0) defer[atomicAdd(defer_count, 1)] = (int32_t)e;
    } else {
      const float wfe = E.w();
      const bool data_w = wfe <= -1000.f;
      for (int pi = lane; pi < npts; pi += 32) {
        const double v = vbuf[pi * 2], vn = vbuf[pi * 2 + 1];
        double fxe = v, vnw = 0;
        if (!band && !data_w) {
          fxe = v * (double)wfe;
          vnw = vn * (double)wfe;
        }
        double* a = acc + pi * 4;
        if (!(fxe > 0) || !isfinite(fxe)) atomicAdd(a + 3, 1.0);
        if (e < ev.nda) {
          atomicAdd(a + 0, (fxe > 0) ? log(fxe) * (double)__ldg(ev.sw + e) : -1e12);
        } else {
          atomicAdd(a + 1, fxe);
          if (!band) atomicAdd(a + 2, vnw);
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();
  for (int pi = threadIdx.x; pi < npts; pi += BATCH_THREADS) {
    const double* a = acc + pi * 4;
    parts[(size_t)blockIdx.x * npts + pi] = Partial{a[0], a[1], a[2], a[3]};
  }
}

// ------------------------------------------------------------------------------- unsmeared events
// Unsmeared events: lane = event (32 consecutive events per warp), all lanes walk the points
// together, so the point data and couplings are warp-uniform reads and the lanes never diverge.
// Per lane the centre's H_L[h], H_Z[h] stay in registers; the entry lineshapes R_q and the Lambda*
// lineshapes q_r go to per-warp shared memory ([q][lane]), and the Pc angular amplitudes HZ_q[h] of
// the group a lineshape point moves are rebuilt when the group changes (points come sorted by kind
// and group).  Per point the warp sums the events' contributions with shuffles and one lane adds
// them to the block's per-point sums.
constexpr int BU_WARPS = 4;
constexpr int BU_THREADS = BU_WARPS * 32;

struct BatchUnLayout {
  size_t q0, r0, hzg, warp_bytes, acc, total;
};
__host__ __device__ inline BatchUnLayout batch_un_layout(int NR, int NZ, int gmax, int npts) {
  BatchUnLayout L;
  size_t o = 0;
  L.q0 = o;
  o = bal16(o + (size_t)(NR > 0 ? NR : 1) * 32 * sizeof(cplx));
  L.r0 = o;
  o = bal16(o + (size_t)(NZ > 0 ? NZ : 1) * 32 * sizeof(cplx));
  L.hzg = o;
  o = bal16(o + (size_t)(gmax > 0 ? gmax : 1) * 8 * 32 * sizeof(cplx));
  L.warp_bytes = o;
  L.acc = BU_WARPS * o;
  L.total = L.acc + (size_t)npts * 4 * sizeof(double);
  return L;
}

// Largest Pc group of a point table.
__host__ __device__ inline int max_group(const PointTable& T) {
  int g = 0;
  for (int i = 0; i < T.ngroups; ++i) g = T.grp[i].count > g ? T.grp[i].count : g;
  return g;
}

// out[h] += q * sum_m c[k * 6 + m] A_ijm DL_{sx,k,m} for all 8 helicities h = (i, j, k): per m the four
// A_ijm and the two DL values are loaded once.
__device__ __forceinline__ void lstar_acc(const cplx* c, int sx, const Ev& E, cplx q, cplx* out) {
#pragma unroll 1
  for (int m = 0; m < 6; ++m) {
    const cplx c0 = c[m], c1 = c[6 + m];
    const bool n0 = nonzero(c0), n1 = nonzero(c1);
    if (!n0 && !n1) continue;
    const cplx w0 = (q * c0) * E.DL(sx, 0, m), w1 = (q * c1) * E.DL(sx, 1, m);
#pragma unroll
    for (int ij = 0; ij < 4; ++ij) {
      const cplx a = E.A(ij >> 1, ij & 1, m);
      cmac(out[2 * ij], a, w0);
      cmac(out[2 * ij + 1], a, w1);
    }
  }
}

// out[h] += q * sum_m c[k * 12 + m] AZ_ijm DZ_{sx,k,m} for all 8 helicities.
__device__ __forceinline__ void pc_acc(const cplx* c, int sx, const Ev& E, cplx q, cplx* out) {
#pragma unroll 1
  for (int m = 0; m < 12; ++m) {
    const cplx c0 = c[m], c1 = c[12 + m];
    if (!nonzero(c0) && !nonzero(c1)) continue;
    const cplx w0 = (q * c0) * E.DZ(sx, 0, m), w1 = (q * c1) * E.DZ(sx, 1, m);
#pragma unroll
    for (int ij = 0; ij < 4; ++ij) {
      const cplx a = E.AZ(ij >> 1, ij & 1, m);
      cmac(out[2 * ij], a, w0);
      cmac(out[2 * ij + 1], a, w1);
    }
  }
}

template <bool FIX>
__global__ void __launch_bounds__(BU_THREADS)
    k_batch_un(EventSet ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
               const PointTable* __restrict__ T0p, const __grid_constant__ BatchGroupMap gm,
               const BatchPoint* __restrict__ pts, int npts, Partial* parts, int32_t* defer, int* defer_count) {
  extern __shared__ __align__(16) unsigned char sm[];
  const PointTable& T0 = *T0p;
  const int NR = T0.NR, NZ = T0.NZ;
  const BatchUnLayout Ly = batch_un_layout(NR, NZ, gm.max_slots, npts);
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  unsigned char* wb = sm + warp * Ly.warp_bytes;
  cplx* q0s = reinterpret_cast<cplx*>(wb + Ly.q0);   // [r][lane]
  cplx* r0s = reinterpret_cast<cplx*>(wb + Ly.r0);   // [q][lane]
  cplx* hzg = reinterpret_cast<cplx*>(wb + Ly.hzg);  // [entry of group][h][lane]
  double* acc = reinterpret_cast<double*>(sm + Ly.acc);
  for (int i = threadIdx.x; i < npts * 4; i += BU_THREADS) acc[i] = 0.0;
  __syncthreads();

  if (n_list) end = begin + *n_list;
  const int64_t count = end - begin;
  int64_t c0, c1, w0, wstep;
  if (n_list) {
    c0 = 0;
    c1 = count;
    w0 = ((int64_t)blockIdx.x * BU_WARPS + warp) * 32;
    wstep = (int64_t)gridDim.x * BU_WARPS * 32;
  } else {
    int64_t chunk = (count + gridDim.x - 1) / gridDim.x;
    chunk = (chunk + BU_THREADS - 1) / BU_THREADS * BU_THREADS;
    c0 = (int64_t)blockIdx.x * chunk;
    c1 = min(count, c0 + chunk);
    w0 = warp * 32;
    wstep = BU_THREADS;
  }
  for (int64_t base = c0 + w0; base < c1; base += wstep) {
    const int64_t pp = base + lane;
    const bool valid = pp < c1;
    const Ev E{ev.pp, ev.pp1, ev.pp2, ev.n_size, event_index(list, begin, valid ? pp : c0)};
    const double mkp = E.mkp(), mz = E.mz();
    // centre
    cplx HL0[8], HZ0[8];
#pragma unroll
    for (int h = 0; h < 8; ++h) HL0[h] = HZ0[h] = mk(0, 0);
    // the kinematic inputs of the Lambda* lineshapes are the same for every point of the batch
    const LstarKin lk0 = lstar_kin(T0, mkp);
    {
      for (int r = 0; r < NR; ++r) {
        const cplx q = lstar_lineshape(T0.L[r], lk0);
        q0s[r * 32 + lane] = q;
        lstar_acc(T0.L[r].c, T0.L[r].sidx, E, q, HL0);
      }
    }
    bool fail = false;
    if (NZ > 0) {
      cplx rr[MAX_PC];
      if (FIX)
        lookup_entries(T0, mz, rr);
      else
        fail = !lookup_table(T0, mz, rr);
      for (int q = 0; q < NZ; ++q) {
        r0s[q * 32 + lane] = rr[q];
        const PcEntry& Z = T0.Z[T0.order[q]];
        pc_acc(Z.c, Z.sidx, E, rr[q], HZ0);
      }
    }
    if (!FIX) {
      // a point's lineshape table must serve this mass too (checked before anything is summed); the
      // batch puts its lineshape points first
      for (int pi = 0; pi < npts; ++pi) {
        const BatchPoint& bp = pts[pi];
        if (bp.kind != BP_PCG) break;
        TabAt ta;
        fail |= !tab_at(bp.T->tab, mz, ta);
      }
    }
    const bool deferred = !FIX && valid && fail;
    if (deferred) defer[atomicAdd(defer_count, 1)] = (int32_t)E.e;
    const bool live = valid && !deferred;
    const float wf = E.w();
    const bool data_w = wf <= -1000.f;
    const bool is_data = E.e < ev.nda;
    const double swe = (live && is_data) ? (double)__ldg(ev.sw + E.e) : 0.0;
    int cur_group = -1;
    __syncwarp();
    for (int pi = 0; pi < npts; ++pi) {
      const BatchPoint& bp = pts[pi];
      const int kind = bp.kind;
      cplx d[8];  // change of H_L (Lambda* points) or of H_Z (Pc points)
#pragma unroll
      for (int h = 0; h < 8; ++h) d[h] = mk(0, 0);
      if (kind == BP_LSTAR) {
        const PointTable& Tp = *bp.T;
        const unsigned lm = bp.lmask, lsm = bp.lsmask, lcm = bp.lcmask;
        int u = 0;
        for (int r = 0; r < NR; ++r) {
          if (!(lm >> r & 1)) continue;
          const bool ls = lsm >> r & 1, cc = lcm >> r & 1;
          const cplx q0 = q0s[r * 32 + lane];
          const int sx = T0.L[r].sidx;
          if (!ls && cc && bp.ldc) {  // couplings only
            lstar_acc(bp.dc + 24 * u++, sx, E, q0, d);
          } else {
            if (cc) ++u;
            const cplx qp = lstar_lineshape(Tp.L[r], lk0);
            if (!cc) {
              lstar_acc(T0.L[r].c, sx, E, qp - q0, d);
            } else {
              lstar_acc(Tp.L[r].c, sx, E, qp, d);
              lstar_acc(T0.L[r].c, sx, E, mk(-q0.re, -q0.im), d);
            }
          }
        }
      } else if (kind == BP_PCC) {
        for (int u = 0; u < bp.nq; ++u) {
          pc_acc(bp.dc + u * 24, bp.qsidx[u], E, r0s[bp.qpos[u] * 32 + lane], d);
        }
      } else if (kind == BP_PCG) {
        const PointTable& Tp = *bp.T;
        const int g = bp.group;
        const int first = T0.grp[g].first, cnt = T0.grp[g].count;
        const int ns = gm.nslot[g];
        if (g != cur_group) {
          for (int sl = 0; sl < ns; ++sl) {
            const PcEntry& Z = T0.Z[T0.order[gm.rep[g * 8 + sl]]];
            cplx t[8];
#pragma unroll
            for (int h = 0; h < 8; ++h) t[h] = mk(0, 0);
            pc_acc(Z.c, Z.sidx, E, mk(1, 0), t);
#pragma unroll
            for (int h = 0; h < 8; ++h) hzg[(sl * 8 + h) * 32 + lane] = t[h];
          }
          cur_group = g;
        }
        cplx dr[MAX_GROUP_ENTRIES];
        if (!group_lineshapes<FIX>(Tp, g, mz, dr)) {
#pragma unroll
          for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) dr[q] = q < cnt ? r0s[(first + q) * 32 + lane] : mk(0, 0);
        }
        cplx dsl[MAX_GROUP_ENTRIES];  // lineshape change summed per coupling slot
#pragma unroll
        for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) dsl[q] = mk(0, 0);
#pragma unroll
        for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) {
          if (q >= cnt) break;
          const cplx dq = dr[q] - r0s[(first + q) * 32 + lane];
          const int sl = gm.slot[first + q];
#pragma unroll
          for (int t = 0; t < MAX_GROUP_ENTRIES; ++t)
            if (t == sl) dsl[t] += dq;
        }
#pragma unroll
        for (int sl = 0; sl < MAX_GROUP_ENTRIES; ++sl) {
          if (sl >= ns) break;
#pragma unroll
          for (int h = 0; h < 8; ++h) cmac(d[h], dsl[sl], hzg[(sl * 8 + h) * 32 + lane]);
        }
      }
      const bool to_hl = kind == BP_LSTAR;
      double v = 0, vn = 0;
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const cplx hl = to_hl ? HL0[h] + d[h] : HL0[h], hz = to_hl ? HZ0[h] : HZ0[h] + d[h];
        v += norm2(hl + hz);
        vn += norm2(hl) + norm2(hz);
      }
      const double fxe = data_w ? v : v * (double)wf;
      double a0 = 0, a1 = 0, a2 = 0;
      bool bad = false;
      if (live) {
        bad = !(fxe > 0) || !isfinite(fxe);
        if (is_data) {
          a0 = (fxe > 0) ? log(fxe) * swe : -1e12;
        } else {
          a1 = fxe;
          a2 = data_w ? 0.0 : vn * (double)wf;
        }
      }
      a0 = warp_sum(a0);
      a1 = warp_sum(a1);
      a2 = warp_sum(a2);
      const int nbad = __popc(__ballot_sync(0xffffffffu, bad));
      if (lane == 0) {
        double* a = acc + pi * 4;
        atomicAdd(a + 0, a0);
        atomicAdd(a + 1, a1);
        atomicAdd(a + 2, a2);
        if (nbad) atomicAdd(a + 3, (double)nbad);
      }
    }
    __syncwarp();
  }
  __syncthreads();
  for (int pi = threadIdx.x; pi < npts; pi += BU_THREADS) {
    const double* a = acc + pi * 4;
    parts[(size_t)blockIdx.x * npts + pi] = Partial{a[0], a[1], a[2], a[3]};
  }
}

// ------------------------------------------------------------------------------- host side
template <int NB, bool FIX>
static cudaError_t set_batch_smem(int optin) {
  return cudaFuncSetAttribute(k_batch<NB, FIX>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
}

cudaError_t configure_batch_kernels() {
  int dev = 0, optin = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev))) return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
  optin -= 1024;  // the kernels' static shared memory stays below 1 KB
  if ((e = set_batch_smem<20, false>(optin)) || (e = set_batch_smem<20, true>(optin)) ||
      (e = set_batch_smem<30, false>(optin)) || (e = set_batch_smem<30, true>(optin)) ||
      (e = set_batch_smem<150, false>(optin)) || (e = set_batch_smem<150, true>(optin)) ||
      (e = set_batch_smem<0, false>(optin)) || (e = set_batch_smem<0, true>(optin)))
    return e;
  if ((e = cudaFuncSetAttribute(k_batch_un<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin)) ||
      (e = cudaFuncSetAttribute(k_batch_un<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin)))
    return e;
  return cudaSuccess;
}

static bool same_bytes(const void* a, const void* b, size_t n) { return std::memcmp(a, b, n) == 0; }

BatchGroupMap batch_group_map(const PointTable& T0) {
  BatchGroupMap m;
  std::memset(&m, 0, sizeof(m));
  for (int g = 0; g < T0.ngroups; ++g) {
    const PcGroup& gr = T0.grp[g];
    int ns = 0;
    for (int q = 0; q < gr.count; ++q) {
      const int pos = gr.first + q;
      const cplx* c = T0.Z[T0.order[pos]].c;
      int sl = 0;
      while (sl < ns && !same_bytes(T0.Z[T0.order[m.rep[g * 8 + sl]]].c, c, 24 * sizeof(cplx))) ++sl;
      if (sl == ns) m.rep[g * 8 + ns++] = pos;
      m.slot[pos] = sl;
    }
    m.nslot[g] = ns;
    m.max_slots = ns > m.max_slots ? ns : m.max_slots;
  }
  return m;
}

bool classify_point(const PointTable& T0, const PointTable& Tp, BatchPoint* bp, cplx* dc_host) {
  *bp = BatchPoint{};
  // structure and global constants must agree
  if (T0.NR != Tp.NR || T0.NZ != Tp.NZ || T0.ngroups != Tp.ngroups || T0.ffr != Tp.ffr || T0.ffb != Tp.ffb ||
      T0.lmask_lstar_R != Tp.lmask_lstar_R || T0.lmask_lstar_B != Tp.lmask_lstar_B ||
      T0.lmask_pc_B != Tp.lmask_pc_B || T0.lmask_pc_R != Tp.lmask_pc_R || T0.needs_sigma_pi != Tp.needs_sigma_pi ||
      !same_bytes(T0.order, Tp.order, sizeof(T0.order)))
    return false;
  for (int g = 0; g < T0.ngroups; ++g) {
    const PcGroup &a = T0.grp[g], &b = Tp.grp[g];
    if (a.km != b.km || a.sidx != b.sidx || a.first != b.first || a.count != b.count) return false;
  }
  unsigned lmask = 0;
  for (int r = 0; r < T0.NR; ++r)
    if (!same_bytes(&T0.L[r], &Tp.L[r], sizeof(LstarEntry))) lmask |= 1u << r;
  // Pc entries by order position: couplings changed, anything else changed
  int ncoup = 0, nconst = 0, cgroup = -1;
  bool multi_group = false;
  int qpos[MAX_PC];
  for (int pos = 0; pos < T0.NZ; ++pos) {
    const int i = T0.order[pos];
    PcEntry a = T0.Z[i], b = Tp.Z[i];
    const bool coup = !same_bytes(a.c, b.c, sizeof(a.c));
    std::memset(a.c, 0, sizeof(a.c));
    std::memset(b.c, 0, sizeof(b.c));
    const bool cons = !same_bytes(&a, &b, sizeof(PcEntry));
    if (coup) qpos[ncoup++] = pos;
    if (cons) {
      ++nconst;
      int g = 0;
      while (g < T0.ngroups && !(pos >= T0.grp[g].first && pos < T0.grp[g].first + T0.grp[g].count)) ++g;
      if (cgroup >= 0 && cgroup != g) multi_group = true;
      cgroup = g;
    }
  }
  for (int ik = 0; ik < 4; ++ik) {
    if (same_bytes(&T0.G[ik], &Tp.G[ik], sizeof(KmGroup))) continue;
    int g = 0;
    while (g < T0.ngroups && T0.grp[g].km != ik) ++g;
    if (g == T0.ngroups) continue;  // group not in the model
    if (cgroup >= 0 && cgroup != g) multi_group = true;
    cgroup = g;
    ++nconst;
  }
  const int parts = (lmask ? 1 : 0) + (ncoup ? 1 : 0) + (nconst ? 1 : 0);
  if (parts == 0) {
    bp->kind = BP_SAME;
    return true;
  }
  if (parts > 1 || multi_group) return false;
  if (lmask) {
    bp->kind = BP_LSTAR;
    bp->lmask = lmask;
    int u = 0;
    for (int r = 0; r < T0.NR; ++r) {
      if (!(lmask >> r & 1)) continue;
      LstarEntry a = T0.L[r], b = Tp.L[r];
      const bool coup = !same_bytes(a.c, b.c, sizeof(a.c));
      std::memset(a.c, 0, sizeof(a.c));
      std::memset(b.c, 0, sizeof(b.c));
      if (!same_bytes(&a, &b, sizeof(LstarEntry))) bp->lsmask |= 1u << r;
      if (coup) {
        bp->lcmask |= 1u << r;
        if (u < BATCH_MAXQ)
          for (int sl = 0; sl < 12; ++sl) dc_host[u * 24 + sl] = Tp.L[r].c[sl] - T0.L[r].c[sl];
        ++u;
      }
    }
    bp->ldc = u <= BATCH_MAXQ ? 1 : 0;
    return true;
  }
  if (ncoup) {
    if (ncoup > BATCH_MAXQ) return false;
    bp->kind = BP_PCC;
    bp->nq = ncoup;
    for (int u = 0; u < ncoup; ++u) {
      const int i = T0.order[qpos[u]];
      bp->qpos[u] = qpos[u];
      bp->qsidx[u] = T0.Z[i].sidx;
      for (int s = 0; s < 24; ++s) dc_host[u * 24 + s] = Tp.Z[i].c[s] - T0.Z[i].c[s];
    }
    return true;
  }
  bp->kind = BP_PCG;
  bp->group = cgroup;
  return true;
}

// Offsets of a segment's smearing scheme for the batched kernels: 0 unsmeared (k_batch_un), -1 the
// weighted grid (k_batch<0>), else the quantile scheme's NB.
static int batch_nb(int kind) {
  return kind == SMEAR_20 ? 20 : kind == SMEAR_30 ? 30 : kind == SMEAR_150 ? 150 : kind == SMEAR_GRID ? -1 : 0;
}

static int batch_grid(const Segment& s, const PointTable& T0, const BatchGroupMap& gm, int npts, int sm_count) {
  const int64_t n = s.end - s.begin;
  int occ = 1;
  int64_t b;
  if (batch_nb(s.kind) == 0) {
    b = (n + BU_THREADS - 1) / BU_THREADS;
    const size_t smem = batch_un_layout(T0.NR, T0.NZ, gm.max_slots, npts).total;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_un<false>, BU_THREADS, smem);
  } else {
    b = (n + BATCH_WARPS - 1) / BATCH_WARPS;
    const size_t smem = batch_layout(T0.NR, T0.NZ, npts).total;
    switch (batch_nb(s.kind)) {
      case 20: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch<20, false>, BATCH_THREADS, smem); break;
      case 30: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch<30, false>, BATCH_THREADS, smem); break;
      case -1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch<0, false>, BATCH_THREADS, smem); break;
      default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch<150, false>, BATCH_THREADS, smem); break;
    }
  }
  if (occ < 1) occ = 1;
  const int64_t cap = (int64_t)sm_count * occ;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

int batch_segment_rows(const Segment& s, const PointTable& T0, const BatchGroupMap& gm, int npts, int sm_count,
                       bool deferred) {
  const int g = batch_grid(s, T0, gm, npts, sm_count);
  return deferred ? 2 * g : g;
}

template <int NB>
static void launch_batch_kind(const EventSet& ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
                              const PointTable* d_T0, const BatchPoint* d_pts, int npts, Partial* out, int band,
                              int32_t* defer, int* defer_count, bool fix, int grid, size_t smem, cudaStream_t st,
                              const double* sgrid, int sgrid_nb) {
  if (fix)
    k_batch<NB, true><<<grid, BATCH_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band,
                                                         defer, defer_count, sgrid, sgrid_nb);
  else
    k_batch<NB, false><<<grid, BATCH_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band,
                                                          defer, defer_count, sgrid, sgrid_nb);
}

static void launch_batch_nb(int nb, const EventSet& ev, int64_t begin, int64_t end, const int32_t* list,
                            const int* n_list, const PointTable* d_T0, const BatchGroupMap& gm,
                            const BatchPoint* d_pts, int npts, Partial* out, int band, int32_t* defer,
                            int* defer_count, bool fix, int grid, size_t smem, cudaStream_t st, const Segment& seg) {
  const double* sg = seg.grid;
  const int sn = seg.grid_nb;
  switch (nb) {
    case 0:
      if (fix)
        k_batch_un<true><<<grid, BU_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, gm, d_pts, npts, out,
                                                          defer, defer_count);
      else
        k_batch_un<false><<<grid, BU_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, gm, d_pts, npts, out,
                                                           defer, defer_count);
      break;
    case -1: launch_batch_kind<0>(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
    case 20: launch_batch_kind<20>(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
    case 30: launch_batch_kind<30>(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
    default: launch_batch_kind<150>(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
  }
}

cudaError_t launch_batch_segment(const EventSet& ev, const Segment& seg, const PointTable* d_T0, const PointTable& T0,
                                 const BatchGroupMap& gm, const BatchPoint* d_pts, int npts, Partial* out,
                                 int32_t* defer, int* defer_count, int sm_count, cudaStream_t st) {
  if (seg.end <= seg.begin) return cudaSuccess;
  if (npts < 1 || npts > BATCH_MAX_POINTS) return cudaErrorInvalidValue;
  const int nb = batch_nb(seg.kind);
  if (nb < 0 && (!seg.grid || seg.grid_nb < 1 || seg.grid_nb > GRID_MAX_NB)) return cudaErrorInvalidValue;
  const int band = (seg.kind == SMEAR_30 || seg.kind == SMEAR_150) ? 1 : 0;
  const size_t smem = nb == 0 ? batch_un_layout(T0.NR, T0.NZ, gm.max_slots, npts).total
                              : batch_layout(T0.NR, T0.NZ, npts).total;
  const int grid = batch_grid(seg, T0, gm, npts, sm_count);
  if (defer) {
    launch_batch_nb(nb, ev, seg.begin, seg.end, seg.list, nullptr, d_T0, gm, d_pts, npts, out, band, defer,
                    defer_count, false, grid, smem, st, seg);
    launch_batch_nb(nb, ev, 0, 0, defer, defer_count, d_T0, gm, d_pts, npts, out + (size_t)grid * npts, band,
                    nullptr, nullptr, true, grid, smem, st, seg);
  } else {
    launch_batch_nb(nb, ev, seg.begin, seg.end, seg.list, nullptr, d_T0, gm, d_pts, npts, out, band, nullptr,
                    nullptr, true, grid, smem, st, seg);
  }
  return cudaGetLastError();
}

}  // namespace pwa
