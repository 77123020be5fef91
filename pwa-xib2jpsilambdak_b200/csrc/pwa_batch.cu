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
// The smeared classes' kernel k_batch (pwa_batch_smeared.cuh, one translation unit per offset scheme)
// and the unsmeared class's k_batch_un (below).  Work split of k_batch: one warp per event.  The warp stages the event's 303 basis planes in shared memory,
// evaluates the centre (Lambda* terms, Pc angular amplitudes HZ_q[h], the entry lineshapes R at up to
// 32 masses per round and S_b[h] = sum_q R_q(m_b) HZ_q[h]), then each lane takes one parameter point.
// Per-point results go to per-block FP64 sums; a finalize kernel reduces them per point.
#include <algorithm>
#include <cstring>
#include <vector>

#include "pwa_batch_smeared.cuh"

namespace pwa {

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
  size_t q0, r0, hzg, hxs, warp_bytes, acc, total;
};
__host__ __device__ inline BatchUnLayout batch_un_layout(int NR, int NZ, int NX, int gmax, int npts) {
  BatchUnLayout L;
  size_t o = 0;
  L.q0 = o;
  o = bal16(o + (size_t)(NR > 0 ? NR : 1) * 32 * sizeof(cplx));
  L.r0 = o;
  o = bal16(o + (size_t)(NZ > 0 ? NZ : 1) * 32 * sizeof(cplx));
  L.hzg = o;
  o = bal16(o + (size_t)(gmax > 0 ? gmax : 1) * 8 * 32 * sizeof(cplx));
  L.hxs = o;  // the centre's Zcs amplitudes [h][lane] (models with Zcs entries)
  o = bal16(o + (size_t)(NX > 0 ? 8 * 32 : 0) * sizeof(cplx));
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
// A_ijm and the two DL values are loaded once.  The event planes come from L2 at every point and the
// kernel runs 8 warps per SM, so the m loop is unrolled (3 here, 6 in pc_acc) to let the loads of
// several m be in flight together: 10 % less time for the unsmeared class than one m at a time.
__device__ __forceinline__ void lstar_acc(const cplx* c, int sx, const Ev& E, cplx q, cplx* out) {
#pragma unroll 3
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
#pragma unroll 6
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

// Two points that move the same Lambda* couplings (differences ca, cb) from one pass over the planes:
// outa / outb as lstar_acc with ca / cb.
__device__ __forceinline__ void lstar_acc2(const cplx* ca, const cplx* cb, int sx, const Ev& E, cplx q, cplx* outa,
                                           cplx* outb) {
#pragma unroll 3
  for (int m = 0; m < 6; ++m) {
    const cplx a0 = ca[m], a1 = ca[6 + m], b0 = cb[m], b1 = cb[6 + m];
    if (!nonzero(a0) && !nonzero(a1) && !nonzero(b0) && !nonzero(b1)) continue;
    const double dl0 = E.DL(sx, 0, m), dl1 = E.DL(sx, 1, m);
    const cplx wa0 = (q * a0) * dl0, wa1 = (q * a1) * dl1, wb0 = (q * b0) * dl0, wb1 = (q * b1) * dl1;
#pragma unroll
    for (int ij = 0; ij < 4; ++ij) {
      const cplx a = E.A(ij >> 1, ij & 1, m);
      cmac(outa[2 * ij], a, wa0);
      cmac(outa[2 * ij + 1], a, wa1);
      cmac(outb[2 * ij], a, wb0);
      cmac(outb[2 * ij + 1], a, wb1);
    }
  }
}

// Two points that move the same Pc entry's couplings: outa / outb as pc_acc with ca / cb.
__device__ __forceinline__ void pc_acc2(const cplx* ca, const cplx* cb, int sx, const Ev& E, cplx q, cplx* outa,
                                        cplx* outb) {
#pragma unroll 4
  for (int m = 0; m < 12; ++m) {
    const cplx a0 = ca[m], a1 = ca[12 + m], b0 = cb[m], b1 = cb[12 + m];
    if (!nonzero(a0) && !nonzero(a1) && !nonzero(b0) && !nonzero(b1)) continue;
    const double dz0 = E.DZ(sx, 0, m), dz1 = E.DZ(sx, 1, m);
    const cplx wa0 = (q * a0) * dz0, wa1 = (q * a1) * dz1, wb0 = (q * b0) * dz0, wb1 = (q * b1) * dz1;
#pragma unroll
    for (int ij = 0; ij < 4; ++ij) {
      const cplx a = E.AZ(ij >> 1, ij & 1, m);
      cmac(outa[2 * ij], a, wa0);
      cmac(outa[2 * ij + 1], a, wa1);
      cmac(outb[2 * ij], a, wb0);
      cmac(outb[2 * ij + 1], a, wb1);
    }
  }
}

// ZCS: the model has Zcs entries (instantiated apart so that the common kernel stays as it was)
template <bool FIX, bool ZCS>
__global__ void __launch_bounds__(BU_THREADS)
    k_batch_un(EventSet ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
               const PointTable* __restrict__ T0p, const __grid_constant__ BatchGroupMap gm,
               const BatchPoint* __restrict__ pts, int npts, Partial* parts, int32_t* defer, int* defer_count) {
  extern __shared__ __align__(16) unsigned char sm[];
  const PointTable& T0 = *T0p;
  const int NR = T0.NR, NZ = T0.NZ;
  constexpr bool has_x = ZCS;  // Zcs entries (their amplitudes join the centre's H_L)
  const BatchUnLayout Ly = batch_un_layout(NR, NZ, T0.NX, gm.max_slots, npts);
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  unsigned char* wb = sm + warp * Ly.warp_bytes;
  cplx* q0s = reinterpret_cast<cplx*>(wb + Ly.q0);   // [r][lane]
  cplx* r0s = reinterpret_cast<cplx*>(wb + Ly.r0);   // [q][lane]
  cplx* hzg = reinterpret_cast<cplx*>(wb + Ly.hzg);  // [entry of group][h][lane]
  cplx* hxs = reinterpret_cast<cplx*>(wb + Ly.hxs);  // [h][lane]
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
        const cplx q = lstar_lineshape(T0, r, lk0);
        q0s[r * 32 + lane] = q;
        lstar_acc(T0.L[r].c, T0.L[r].sidx, E, q, HL0);
      }
    }
    // Zcs joins the centre's H_L; kept apart for the non-interfering term
    if (has_x) {
      for (int k = 0; k < 2; ++k) {
        cplx t[4];
#pragma unroll
        for (int ij = 0; ij < 4; ++ij) t[ij] = mk(0, 0);
        zcs_amplitudes<4>(T0, EvX{ev.pp3, ev.pp4, ev.n_size, E.e}, k, 0, t);
#pragma unroll
        for (int ij = 0; ij < 4; ++ij) {
          HL0[2 * ij + k] += t[ij];
          hxs[(2 * ij + k) * 32 + lane] = t[ij];
        }
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
    // |A|^2 of point pi from its amplitude change d (to H_L for Lambda* points, to H_Z otherwise), and
    // the warp's sums of it into the block's per-point sums
    auto finish = [&](int pi, int kind, const cplx(&d)[8]) {
      const bool to_hl = kind == BP_LSTAR;
      double v = 0, vn = 0;
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const cplx hl = to_hl ? HL0[h] + d[h] : HL0[h], hz = to_hl ? HZ0[h] : HZ0[h] + d[h];
        v += norm2(hl + hz);
        if (has_x) {
          const cplx hx = hxs[h * 32 + lane];
          vn += norm2(hl - hx) + norm2(hx) + norm2(hz);
        } else {
          vn += norm2(hl) + norm2(hz);
        }
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
    };
    for (int pi = 0; pi < npts; ++pi) {
      const BatchPoint& bp = pts[pi];
      const int kind = bp.kind;
      cplx d[8];  // change of H_L (Lambda* points) or of H_Z (Pc points)
#pragma unroll
      for (int h = 0; h < 8; ++h) d[h] = mk(0, 0);
      if (bp.pair) {
        // this point and the next move the same couplings: one pass over the planes for both
        const BatchPoint& bq = pts[pi + 1];
        cplx d2[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) d2[h] = mk(0, 0);
        if (kind == BP_LSTAR) {
          int u = 0;
          for (int r = 0; r < NR; ++r) {
            if (!(bp.lmask >> r & 1)) continue;
            lstar_acc2(bp.dc + 24 * u, bq.dc + 24 * u, T0.L[r].sidx, E, q0s[r * 32 + lane], d, d2);
            ++u;
          }
        } else {
          for (int u = 0; u < bp.nq; ++u)
            pc_acc2(bp.dc + u * 24, bq.dc + u * 24, bp.qsidx[u], E, r0s[bp.qpos[u] * 32 + lane], d, d2);
        }
        finish(pi, kind, d);
        finish(pi + 1, kind, d2);
        ++pi;
        continue;
      }
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
            const cplx qp = lstar_lineshape(Tp, r, lk0);
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
      finish(pi, kind, d);
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
cudaError_t configure_batch_kernels() {
  int dev = 0, optin = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev))) return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
  optin -= 1024;  // the kernels' static shared memory stays below 1 KB
  if ((e = batch_set_smem_20(optin)) || (e = batch_set_smem_30(optin)) || (e = batch_set_smem_150(optin)) ||
      (e = batch_set_smem_grid(optin)))
    return e;
  if ((e = cudaFuncSetAttribute(k_batch_un<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin)) ||
      (e = cudaFuncSetAttribute(k_batch_un<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin)) ||
      (e = cudaFuncSetAttribute(k_batch_un<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin)) ||
      (e = cudaFuncSetAttribute(k_batch_un<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin)))
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

// Inputs of a lineshape that live outside its own entry: the spline block it reads, or every entry of
// its revised K-matrix set (chain c: 0 Lambda*, 1 Pc).
static bool shape_inputs_differ(const PointTable& A, const PointTable& B, int c, int type, int aux) {
  if (type == LT_SPLINE)
    return !same_bytes(A.spl + aux, B.spl + aux, 9 * (c ? SPL_KNOTS_Z : SPL_KNOTS_L) * sizeof(float));
  if (type == LT_RKM) {
    const int set = A.rkm[c][aux].set;
    for (int j = 0; j < A.nrkm[c]; ++j)
      if (A.rkm[c][j].set == set && !same_bytes(&A.rkm[c][j], &B.rkm[c][j], sizeof(RkmEntry))) return true;
  }
  return false;
}

bool classify_point(const PointTable& T0, const PointTable& Tp, BatchPoint* bp, cplx* dc_host) {
  *bp = BatchPoint{};
  // structure and global constants must agree
  if (T0.NR != Tp.NR || T0.NZ != Tp.NZ || T0.ngroups != Tp.ngroups || T0.ffr != Tp.ffr || T0.ffb != Tp.ffb ||
      T0.lmask_lstar_R != Tp.lmask_lstar_R || T0.lmask_lstar_B != Tp.lmask_lstar_B ||
      T0.lmask_pc_B != Tp.lmask_pc_B || T0.lmask_pc_R != Tp.lmask_pc_R || T0.needs_sigma_pi != Tp.needs_sigma_pi ||
      !same_bytes(T0.order, Tp.order, sizeof(T0.order)) || !same_bytes(T0.nrkm, Tp.nrkm, sizeof(T0.nrkm)))
    return false;
  // Zcs entries are part of the centre's H_L: a point that moves one goes through the single-point path
  if (T0.NX != Tp.NX || T0.lmask_x_R != Tp.lmask_x_R || T0.lmask_x_B != Tp.lmask_x_B ||
      !same_bytes(T0.x_mmask, Tp.x_mmask, sizeof(T0.x_mmask)) || !same_bytes(T0.X, Tp.X, sizeof(T0.X)))
    return false;
  for (int g = 0; g < T0.ngroups; ++g) {
    const PcGroup &a = T0.grp[g], &b = Tp.grp[g];
    if (a.km != b.km || a.sidx != b.sidx || a.first != b.first || a.count != b.count) return false;
  }
  unsigned lmask = 0;
  for (int r = 0; r < T0.NR; ++r)
    if (!same_bytes(&T0.L[r], &Tp.L[r], sizeof(LstarEntry)) ||
        shape_inputs_differ(T0, Tp, 0, T0.L[r].type, T0.L[r].aux))
      lmask |= 1u << r;
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
    const bool cons = !same_bytes(&a, &b, sizeof(PcEntry)) || shape_inputs_differ(T0, Tp, 1, a.type, a.aux);
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
      if (!same_bytes(&a, &b, sizeof(LstarEntry)) || shape_inputs_differ(T0, Tp, 0, a.type, a.aux))
        bp->lsmask |= 1u << r;
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
    if (ncoup > BATCH_MAXQ_PC) return false;
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

// Blocks of a batched pass: one per BATCH_WARPS events (BU_THREADS for the unsmeared kernel), at most
// `waves` x the resident blocks (sm_count x occupancy); waves > 1 trades block start-up cost for a
// finer balance of uneven per-event work (the batch autotuner picks it per event class).
static int batch_grid(const Segment& s, const PointTable& T0, const BatchGroupMap& gm, int npts, int sm_count,
                      int waves) {
  const int64_t n = s.end - s.begin;
  int occ = 1;
  int64_t b;
  if (batch_nb(s.kind) == 0) {
    b = (n + BU_THREADS - 1) / BU_THREADS;
    const size_t smem = batch_un_layout(T0.NR, T0.NZ, T0.NX, gm.max_slots, npts).total;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_un<false, false>, BU_THREADS, smem);
  } else {
    b = (n + BATCH_WARPS - 1) / BATCH_WARPS;
    const int nb = batch_nb(s.kind);
    const size_t smem = batch_layout(T0.NR, T0.NZ, npts, batch_moments(nb), batch_row_cap(nb)).total;
    switch (batch_nb(s.kind)) {
      case 20: occ = batch_occupancy_20(smem); break;
      case 30: occ = batch_occupancy_30(smem); break;
      case -1: occ = batch_occupancy_grid(smem); break;
      default: occ = batch_occupancy_150(smem); break;
    }
  }
  if (occ < 1) occ = 1;
  const int64_t cap = (int64_t)sm_count * occ * std::max(1, waves);
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

int batch_segment_rows(const Segment& s, const PointTable& T0, const BatchGroupMap& gm, int npts, int sm_count,
                       bool deferred, int waves) {
  const int g = batch_grid(s, T0, gm, npts, sm_count, waves);
  return deferred ? 2 * g : g;
}

static void launch_batch_nb(int nb, const EventSet& ev, int64_t begin, int64_t end, const int32_t* list,
                            const int* n_list, const PointTable* d_T0, const BatchGroupMap& gm,
                            const BatchPoint* d_pts, int npts, Partial* out, int band, int32_t* defer,
                            int* defer_count, bool fix, int grid, size_t smem, cudaStream_t st, const Segment& seg) {
  const double* sg = seg.grid;
  const int sn = seg.grid_nb;
  switch (nb) {
    case 0:
      if (ev.pp3 && fix)
        k_batch_un<true, true><<<grid, BU_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, gm, d_pts, npts,
                                                                out, defer, defer_count);
      else if (ev.pp3)
        k_batch_un<false, true><<<grid, BU_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, gm, d_pts, npts,
                                                                 out, defer, defer_count);
      else if (fix)
        k_batch_un<true, false><<<grid, BU_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, gm, d_pts, npts,
                                                                 out, defer, defer_count);
      else
        k_batch_un<false, false><<<grid, BU_THREADS, smem, st>>>(ev, begin, end, list, n_list, d_T0, gm, d_pts,
                                                                  npts, out, defer, defer_count);
      break;
    case -1: batch_launch_grid(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
    case 20: batch_launch_20(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
    case 30: batch_launch_30(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
    default: batch_launch_150(ev, begin, end, list, n_list, d_T0, d_pts, npts, out, band, defer, defer_count, fix, grid, smem, st, sg, sn); break;
  }
}

cudaError_t launch_batch_segment(const EventSet& ev, const Segment& seg, const PointTable* d_T0, const PointTable& T0,
                                 const BatchGroupMap& gm, const BatchPoint* d_pts, int npts, Partial* out,
                                 int32_t* defer, int* defer_count, int sm_count, cudaStream_t st, int waves) {
  if (seg.end <= seg.begin) return cudaSuccess;
  if (npts < 1 || npts > BATCH_MAX_POINTS) return cudaErrorInvalidValue;
  const int nb = batch_nb(seg.kind);
  if (nb < 0 && (!seg.grid || seg.grid_nb < 1 || seg.grid_nb > GRID_MAX_NB)) return cudaErrorInvalidValue;
  const int band = (seg.kind == SMEAR_30 || seg.kind == SMEAR_150) ? 1 : 0;
  const size_t smem = nb == 0 ? batch_un_layout(T0.NR, T0.NZ, T0.NX, gm.max_slots, npts).total
                              : batch_layout(T0.NR, T0.NZ, npts, batch_moments(nb), batch_row_cap(nb)).total;
  const int grid = batch_grid(seg, T0, gm, npts, sm_count, waves);
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
