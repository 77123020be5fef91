// Likelihood kernels for sm_100a, FP64 arithmetic on the reference's float SoA basis.
//
// Work split (reference: src/kernel_calEva.cu:819-976):
//   * per parameter point, every Pc entry's lineshape is tabulated on a 10 keV grid of m(J/psi p)
//     (k_build_tables) and each grid interval is verified against exact evaluations
//     (k_check_tables); the event kernels interpolate, and evaluate exactly where the table cannot
//     serve a mass (thresholds, flagged intervals).
//   * unsmeared events (k_unsmeared): two lanes per event, one per proton helicity.
//   * smeared events (k_smeared<NB>, 20 / 30 / 150 resolution offsets): eight lanes per event, one per
//     helicity, holding the Pc angular amplitudes of every entry in registers; the lineshapes at
//     the offsets are computed eight at a time into per-warp shared memory and contracted by all
//     eight lanes.  Warp-synchronous, no block barriers in the event loop.
//   * every block writes FP64 partial sums (data sw ln fx, MC w fx, MC w fx without
//     interference); one finalize block reduces them with compensated summation.
#include <cstdio>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

#include "pwa_device.cuh"

namespace pwa {

// Unsmeared events.  Lane l of a warp takes event l % 16 of the warp's 16 and proton helicity
// k = l / 16, i.e. the four amplitudes H[dmu][lb][k] (GetAmpLz kernel_calEva.cu:85-190 and the Pc
// part of GetAmp2s :347-503): per group the coupling sums E_m = sum_entries lineshape * c_{k,m} are
// formed once and contracted with DZ * AZ; the Lambda* lineshapes are split between the two lanes of
// an event and exchanged.  mode 1: unweighted coherent |A|^2 to fx_out, no sums
// (host_store_amp2s).
//
// FIX = false: lineshapes come from the per-point table only; an event whose mass the table cannot
// serve is not evaluated but appended to defer[] (count in *defer_count).  FIX = true evaluates such
// masses exactly (out of line); it runs over the deferred list (events [0, *n_list) of list) or,
// without tables, over the whole segment.  Keeping the exact path out of the main kernel keeps its
// register allocation free of the call's save/restore.
template <bool FIX, bool ZCS, bool GEN>
__global__ void __launch_bounds__(EV_THREADS, 2)
    k_unsmeared(EventSet ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
                const PointTable* __restrict__ gtab, Partial* parts, double* fx_out, int mode, int32_t* defer,
                int* defer_count) {
  extern __shared__ __align__(16) unsigned char sm[];
  PointTable& T = *reinterpret_cast<PointTable*>(sm);
  load_table<EV_THREADS>(gtab, &T);
  const int lane = threadIdx.x & 31, k = lane >> 4, el = lane & 15;
  if (n_list) end = begin + *n_list;
  const Chunk ch = block_chunk(end - begin, EV_WARPS * UNSMEARED_PER_WARP, n_list != nullptr);
  Acc acc;
  for (int64_t base = ch.c0 + ch.warp0 * UNSMEARED_PER_WARP; base < ch.c1; base += ch.wstep * UNSMEARED_PER_WARP) {
    const int64_t p = base + el;
    const bool valid = p < ch.c1;
    const Ev E{ev.pp, ev.pp1, ev.pp2, ev.n_size, event_index(list, begin, valid ? p : 0)};
    const double mkp = E.mkp(), mz = E.mz();
    // Lambda*: F_m = sum_r lineshape_r c_{r,k,m} DL_{r,k,m}
    cplx F[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) F[m] = mk(0, 0);
    {
      const LstarKin lk = lstar_kin(T, mkp);
      for (int r0 = 0; r0 < T.NR; r0 += 2) {
        const int rm = r0 + k;
        const cplx mine = (rm < T.NR) ? lstar_lineshape<GEN>(T, rm, lk) : mk(0, 0);
        const cplx other = shfl_xor(mine, 16);
#pragma unroll
        for (int d = 0; d < 2; ++d) {
          const int r = r0 + d;
          if (r >= T.NR) break;
          const LstarEntry& L = T.L[r];
          const cplx q = (d == k) ? mine : other;
#pragma unroll
          for (int m = 0; m < 6; ++m) {
            const cplx c = L.c[k * 6 + m];
            if (!nonzero(c)) continue;
            cmac(F[m], q * c, mk(E.DL(L.sidx, k, m), 0.0));
          }
        }
      }
    }
    cplx H[4], HZ[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) H[q] = HZ[q] = mk(0, 0);
    const int lmask = T.lstar_mmask[k];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      if (!(lmask >> m & 1)) continue;
#pragma unroll
      for (int ij = 0; ij < 4; ++ij) cmac(H[ij], E.A(ij >> 1, ij & 1, m), F[m]);
    }
    // Zcs (GetAmpZcs): joins the Lambda* amplitudes; separate in the non-interference sum
    double vn = 0;
    if (ZCS) {
      cplx HX[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) HX[q] = mk(0, 0);
      zcs_amplitudes<4>(T, EvX{ev.pp3, ev.pp4, ev.n_size, E.e}, k, 0, HX);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        vn += norm2(H[q]) + norm2(HX[q]);
        H[q] += HX[q];
      }
    }
    // Pc
    bool deferred = false;
    if (T.NZ > 0) {
      TabAt ta;
      const bool tab_ok = tab_at(T.tab, mz, ta);
      cplx rawx[FIX ? MAX_PC : 1];
      if (FIX && !tab_ok) pc_entries_exact(T, mz, rawx);
      deferred = !FIX && !tab_ok;
      for (int g = 0; g < T.ngroups; ++g) {
        const PcGroup& gr = T.grp[g];
        cplx Eg[12];
#pragma unroll
        for (int m = 0; m < 12; ++m) Eg[m] = mk(0, 0);
        for (int q = 0; q < gr.count; ++q) {
          const int pos = gr.first + q;
          const cplx raw = tab_ok ? tab_get(ta, T.tab.stride, pos) : (FIX ? rawx[pos] : mk(0, 0));
          const PcEntry& Z = T.Z[T.order[pos]];
#pragma unroll
          for (int m = 0; m < 12; ++m) {
            const cplx c = Z.c[k * 12 + m];
            if (nonzero(c)) cmac(Eg[m], raw, c);
          }
        }
        const int gmask = gr.mmask[k];
#pragma unroll
        for (int m = 0; m < 12; ++m) {
          if (!(gmask >> m & 1)) continue;
          const cplx D = Eg[m] * E.DZ(gr.sidx, k, m);
#pragma unroll
          for (int ij = 0; ij < 4; ++ij) cmac(HZ[ij], E.AZ(ij >> 1, ij & 1, m), D);
        }
      }
    }
    double v = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      v += norm2(H[q] + HZ[q]);
      vn += ZCS ? norm2(HZ[q]) : norm2(H[q]) + norm2(HZ[q]);
    }
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    vn += __shfl_xor_sync(0xffffffffu, vn, 16);
    if (k == 0 && valid) {
      if (deferred) {
        defer[atomicAdd(defer_count, 1)] = (int32_t)E.e;
      } else if (mode == 1) {
        fx_out[E.e] = v;
      } else {
        const float wf = E.w();
        const bool data_w = wf <= -1000.f;
        const double fxe = data_w ? v : v * (double)wf;
        if (fx_out) fx_out[E.e] = fxe;
        acc.add(E.e, ev.nda, ev.sw, fxe, data_w ? 0.0 : vn * (double)wf, false);
      }
    }
  }
  if (mode != 1) block_reduce_store<EV_THREADS>(acc.data, acc.mc, acc.mcn, acc.bad, parts);
}

// Per-warp scratch of the smeared kernels: the event's plane slots (as doubles) and, in the
// exact-capable pass, the Pc entry lineshapes of the 8 offset rows of a round that the table cannot
// serve.
constexpr int RAW_ROW = MAX_PC + 1;
struct SmearWarp {
  double pl[SLOT_ALL];
  cplx raw[8 * RAW_ROW];
};

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
constexpr size_t UNSMEARED_SMEM = align16(sizeof(PointTable));
constexpr size_t SMEARED_SMEM = align16(sizeof(PointTable)) + EV_WARPS * sizeof(SmearWarp);

// D += A B for one 8x8x4 FP64 tile (warp-wide; A row-major, B column-major): lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) + i], i = 0, 1.
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Events smeared over NB resolution offsets (kernel_store_fx_SMR / _finebinning, kernel_calEva.cu:
// 819-900; TemplateGetAmp2s :583-784).  One warp per event: the warp first copies the plane slots
// the point reads into shared memory (one batch of independent loads), then for the 8 helicities h = (dmu, lb, k)
// the kernel forms the Lambda* amplitude H_L[h] and, per Pc entry q, the angular amplitude
// HZ_q[h] (couplings included, lineshape excluded); the offsets go in rounds of 8 rows b with
// lineshapes R_q(m_b), and the contraction S_b[h] = sum_q R_q(m_b) HZ_q[h] runs on the FP64 tensor
// path as two real products, [Re S | Im S] = [Re R | Im R] x [[Re HZ, Im HZ], [-Im HZ, Re HZ]].
// Lane (row g = l/4, column t = l%4) evaluates exactly its own operand elements: the lineshapes of
// entries q = t, t+4, t+8, t+12 at the offset of row g (A[g][k]) and HZ_q of helicity g (B[k][g]); it
// receives S_b[h] for row g and helicities 2t, 2t+1.  Finally
//   |A|^2 = sum_h |H_L|^2 + 2 w Re(conj(H_L) sum_b S_b) + w^2 u sum_b |S_b|^2,
// the reference's BW1/BW2 form (kernel_calEva.cu:676-810) with its float weight w = float(1/NB) and
// rescale u = float(1/w).  band = 1 for the two data bands (fx unweighted, no non-interference
// term), 0 for the tail-region window events (row 0 of the first round is then the event's own
// mass, for |A|^2 without interference).
//
// NB = 0: the weighted grid scheme (grid[2b] absolute offset in GeV, grid[2b+1] weight w_b, grid_nb
// offsets, sum of weights 1): |A|^2 = sum_b w_b |A(m + offset_b)|^2
//   = sum_h |H_L|^2 + 2 Re(conj(H_L) sum_b w_b S_b) + sum_b w_b |S_b|^2.
//
// FIX as for k_unsmeared: the main launch defers every event with a resolution offset the table
// cannot serve; the exact-capable launch evaluates such rows exactly (one lane per row).
template <int NB, bool FIX, bool ZCS>
__global__ void __launch_bounds__(EV_THREADS, 3)
    k_smeared(EventSet ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
              const PointTable* __restrict__ gtab, Partial* parts, double* fx_out, int band, int32_t* defer,
              int* defer_count, const double* __restrict__ grid, int grid_nb) {
  extern __shared__ __align__(16) unsigned char sm[];
  PointTable& T = *reinterpret_cast<PointTable*>(sm);
  load_table<EV_THREADS>(gtab, &T);
  SmearWarp& W = reinterpret_cast<SmearWarp*>(sm + align16(sizeof(PointTable)))[threadIdx.x / 32];
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;   // fragment row (offset row, B-operand helicity) and column
  const int h = lane & 7, part = lane >> 3;  // helicity and resonance share of the Lambda* sums
  const int hi = h >> 2, hj = (h >> 1) & 1, hk = h & 1;
  const int bi = g >> 2, bj = (g >> 1) & 1, bk = g & 1;
  const float* qoff = smear_table<NB>();
  const float wf = (float)(1.0 / (NB ? NB : 1));
  const double wgt = NB ? (double)wf : 1.0;
  const double c2 = NB ? wgt * wgt * (double)(1.0f / wf) : 1.0;
  if (n_list) end = begin + *n_list;
  const Chunk ch = block_chunk(end - begin, EV_WARPS, n_list != nullptr);
  const int shift = band ? 0 : 1;
  const int nlook = (NB ? NB : grid_nb) + shift;
  const int NZ = T.NZ;
  const int nq = (NZ + 3) >> 2;  // k-steps per real product (entries q = t + 4j, j < nq)
  const int pmask = T.pc_mmask[bk];
  const int lmask = T.lstar_mmask[hk];
  Acc acc;
  for (int64_t p = ch.c0 + ch.warp0; p < ch.c1; p += ch.wstep) {
    const int64_t e = event_index(list, begin, p);
    stage_event(T, ev, e, W.pl, lane);
    __syncwarp();
    const EvS E{W.pl};
    const double mkp = E.mkp(), mz = E.mz();
    // Lambda*: lane r evaluates lineshape r; lane (h, part) sums the resonances r = part mod 4
    cplx qmine = mk(0, 0);
    if (lane < T.NR) qmine = lstar_lineshape(T, lane, lstar_kin(T, mkp));
    cplx hl = mk(0, 0);
    for (int r0 = 0; r0 < T.NR; r0 += 4) {
      const int r = r0 + part;
      const cplx q = shfl(qmine, r & 31);
      if (r < T.NR) {
        const LstarEntry& L = T.L[r];
        const cplx* cl = L.c + hk * 6;
        const double* dl = E.p + 51 + L.sidx * 12 + hk * 6;
        cplx f = mk(0, 0);
#pragma unroll
        for (int m = 0; m < 6; ++m) {
          if (!(lmask >> m & 1)) continue;
          const cplx c = cl[m];
          if (nonzero(c)) cmac(f, c, E.A(hi, hj, m) * dl[m]);
        }
        cmac(hl, q, f);
      }
    }
    hl += shfl_xor(hl, 8);
    hl += shfl_xor(hl, 16);
    // Zcs joins H_L (H_L_Zcs of TemplateGetAmp2s); |A|^2 without interference keeps it separate
    double vlx = norm2(hl);
    if (ZCS) {
      cplx hx = mk(0, 0);
      zcs_amplitudes<1>(T, E, hk, 2 * hi + hj, &hx);
      vlx += norm2(hx);
      hl += hx;
    }
    const double hl2 = part == 0 ? norm2(hl) : 0.0;  // sum over lanes: sum_h |H_L[h]|^2
    vlx = part == 0 ? vlx : 0.0;
    const cplx hA = shfl(hl, 2 * t), hB = shfl(hl, 2 * t + 1);  // H_L of this lane's output columns
    // B operand: HZ_q[g] for q = t + 4j
    cplx hz[MAX_PC / 4];
#pragma unroll
    for (int j = 0; j < MAX_PC / 4; ++j) hz[j] = mk(0, 0);
#pragma unroll
    for (int m = 0; m < 12; ++m) {
      if (!(pmask >> m & 1)) continue;
      const cplx az = E.AZ(bi, bj, m);
#pragma unroll
      for (int j = 0; j < MAX_PC / 4; ++j) {
        const int q = t + 4 * j;
        if (q >= NZ) break;
        const PcEntry& Z = T.Z[T.order[q]];
        const cplx c = Z.c[bk * 12 + m];
        if (nonzero(c)) cmac(hz[j], c, az * E.DZ(Z.sidx, bk, m));
      }
    }
    const double mres = MRES0 + mz * (MRES1 + mz * MRES2);
    double a1 = 0, a2 = 0, vn = 0;
    bool fail = false;
    for (int l0 = 0; NZ > 0 && l0 < nlook; l0 += 8) {
      const int l = l0 + g;
      const bool row = l < nlook;
      double m = mz, wb = 1.0;
      if (row && l >= shift) {
        const int b = l - shift;
        m = NB ? mz + (double)qoff[b] * mres : mz + __ldg(grid + 2 * b);
        if (!NB) wb = __ldg(grid + 2 * b + 1);
      }
      TabAt ta;
      const bool ok = row && tab_at(T.tab, m, ta);
      if (FIX) {
        if (row && !ok && t == 0) pc_entries_exact(T, m, W.raw + g * RAW_ROW);
        __syncwarp();
      } else {
        fail |= row && !ok;
      }
      double are[MAX_PC / 4], aim[MAX_PC / 4];
#pragma unroll
      for (int j = 0; j < MAX_PC / 4; ++j) {
        const int q = t + 4 * j;
        cplx r = mk(0, 0);
        if (row && q < NZ) r = ok ? tab_get(ta, T.tab.stride, q) : (FIX ? W.raw[g * RAW_ROW + q] : mk(0, 0));
        are[j] = r.re;
        aim[j] = r.im;
      }
      if (FIX) __syncwarp();
      double sr0 = 0, sr1 = 0, si0 = 0, si1 = 0;
#pragma unroll
      for (int j = 0; j < MAX_PC / 4; ++j) {
        if (j >= nq) break;
        dmma(sr0, sr1, are[j], hz[j].re);
        dmma(si0, si1, are[j], hz[j].im);
        dmma(sr0, sr1, aim[j], -hz[j].im);
        dmma(si0, si1, aim[j], hz[j].re);
      }
      if (row) {
        const double n2 = sr0 * sr0 + si0 * si0 + sr1 * sr1 + si1 * si1;
        if (l < shift) {
          vn += n2;
        } else {
          a1 += wb * (hA.re * sr0 + hA.im * si0 + hB.re * sr1 + hB.im * si1);
          a2 += wb * n2;
        }
      }
    }
    const double v = warp_sum(hl2) + 2.0 * wgt * warp_sum(a1) + c2 * warp_sum(a2);
    const double vnt = warp_sum(vlx) + warp_sum(vn);
    const bool deferred = !FIX && __any_sync(0xffffffffu, fail);
    if (lane == 0) {
      if (deferred) {
        defer[atomicAdd(defer_count, 1)] = (int32_t)e;
      } else {
        double fxe = v, vnw = 0;
        if (!band) {
          const float wfe = (float)E.p[2];
          if (!(wfe <= -1000.f)) {
            fxe = v * (double)wfe;
            vnw = vnt * (double)wfe;
          }
        }
        if (fx_out) fx_out[e] = fxe;
        acc.add(e, ev.nda, ev.sw, fxe, vnw, band != 0);
      }
    }
    __syncwarp();
  }
  block_reduce_store<EV_THREADS>(acc.data, acc.mc, acc.mcn, acc.bad, parts);
}

// ------------------------------------------------------------------------------- tables
// Exact lineshapes of every Pc entry at every level-1 grid node.
__global__ void k_build_tables(const PointTable* __restrict__ T, int n_nodes) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *T->tab.nblocks = 0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_nodes; j += gridDim.x * blockDim.x) {
    cplx* dst = const_cast<cplx*>(T->tab.data) + (size_t)j * T->tab.stride;
    const PcKin kin = pc_kin(*T, T->tab.m_lo + j * T->tab.h);
    for (int g = T->tab.g_lo; g < T->tab.g_hi; ++g) pc_group_exact(*T, g, kin, dst + T->grp[g].first - T->tab.pos0);
  }
}

// Interpolation check of one interval: stencil nodes base[0 .. 5] (node stride `stride`) against an
// exact evaluation at the midpoint of the interval [m0, m0 + step], where the error factor
// prod_n (t - t_n) of the centred 6-point stencil peaks; per Pc group, the largest entry error must
// stay within TAB_CHECK_TOL of the group's largest entry.
__device__ bool interval_ok(const PointTable& T, const cplx* base, int stride, double m0, double step) {
  const double ts[1] = {0.5};
  for (int pt = 0; pt < 1; ++pt) {
    double w[6];
    lagrange6(ts[pt], w);
    const PcKin kin = pc_kin(T, m0 + ts[pt] * step);
    for (int g = T.tab.g_lo; g < T.tab.g_hi; ++g) {
      const PcGroup& gr = T.grp[g];
      cplx ex[MAX_PC];
      pc_group_exact(T, g, kin, ex);
      double emax = 0, vmax = 0;
      for (int q = 0; q < gr.count; ++q) {
        cplx acc = mk(0, 0);
        for (int n = 0; n < 6; ++n) acc += base[n * stride + gr.first - T.tab.pos0 + q] * w[n];
        // written so that a non-finite node or exact value propagates (fmax would drop a NaN)
        const double e = sqrt(norm2(acc - ex[q])), v = sqrt(norm2(ex[q]));
        if (!(e <= emax)) emax = e;
        if (!(v <= vmax)) vmax = v;
      }
      if (!(isfinite(emax) && emax <= TAB_CHECK_TOL * vmax)) return false;
    }
  }
  return true;
}

// True when [lo, hi] touches a guard interval; level 2 (sub = true) only keeps the stencil off the
// guard centres (the non-smooth points themselves) and leaves the rest to the interpolation check.
__device__ bool touches_guard(const LineTables& tab, double lo, double hi, bool sub) {
  for (int q = 0; q < tab.nguard; ++q) {
    double glo = tab.guard_lo[q], ghi = tab.guard_hi[q];
    if (sub) glo = ghi = 0.5 * (glo + ghi);
    if (hi >= glo && lo <= ghi) return true;
  }
  return false;
}

// Level-1 check of every interval; a failing interval gets a refinement block while blocks last.
__global__ void k_check_tables(const PointTable* __restrict__ T, int n_nodes) {
  const LineTables& tab = T->tab;
  int* cell = const_cast<int*>(tab.cell);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_nodes; j += gridDim.x * blockDim.x) {
    if (j < 2 || j + 3 >= n_nodes) {
      cell[j] = -1;
      continue;
    }
    const double m0 = tab.m_lo + j * tab.h;
    bool ok = !touches_guard(tab, m0 - 2 * tab.h, m0 + 3 * tab.h, false);
    if (ok) ok = interval_ok(*T, tab.data + (size_t)(j - 2) * tab.stride, tab.stride, m0, tab.h);
    int c = 0;
    if (!ok) {
      const int b = atomicAdd(tab.nblocks, 1);
      c = -1;
      if (b < TAB_MAX_BLOCKS) {
        tab.block_interval[b] = j;
        c = b + 1;
      }
    }
    cell[j] = c;
  }
}

// Exact lineshapes at the nodes of every refinement block: node s of block b sits at
// m_j + (s - 2) h / TAB_SUB.
__global__ void k_build_sub(const PointTable* __restrict__ T) {
  const LineTables& tab = T->tab;
  const int nb = min(*tab.nblocks, TAB_MAX_BLOCKS);
  const double hs = tab.h / TAB_SUB;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * TAB_SUB_NODES; t += gridDim.x * blockDim.x) {
    const int b = t / TAB_SUB_NODES, s = t % TAB_SUB_NODES;
    const double m = tab.m_lo + tab.block_interval[b] * tab.h + (s - 2) * hs;
    cplx* dst = const_cast<cplx*>(tab.sub) + ((size_t)b * TAB_SUB_NODES + s) * tab.stride;
    const PcKin kin = pc_kin(*T, m);
    for (int g = tab.g_lo; g < tab.g_hi; ++g) pc_group_exact(*T, g, kin, dst + T->grp[g].first - tab.pos0);
  }
}

// Check of every sub-interval of every refinement block.
__global__ void k_check_sub(const PointTable* __restrict__ T) {
  const LineTables& tab = T->tab;
  const int nb = min(*tab.nblocks, TAB_MAX_BLOCKS);
  const double hs = tab.h / TAB_SUB;
  unsigned char* bad = const_cast<unsigned char*>(tab.sub_bad);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * TAB_SUB; t += gridDim.x * blockDim.x) {
    const int b = t / TAB_SUB, i = t % TAB_SUB;
    const double m0 = tab.m_lo + tab.block_interval[b] * tab.h + i * hs;
    bool ok = !touches_guard(tab, m0 - 2 * hs, m0 + 3 * hs, true);
    if (ok) ok = interval_ok(*T, tab.sub + ((size_t)b * TAB_SUB_NODES + i) * tab.stride, tab.stride, m0, hs);
    bad[t] = ok ? 0 : 1;
  }
}

cudaError_t launch_build_tables(const PointTable* d_table, int n_nodes, int sm_count, cudaStream_t st) {
  k_build_tables<<<sm_count * 8, 128, 0, st>>>(d_table, n_nodes);
  k_check_tables<<<sm_count * 8, 128, 0, st>>>(d_table, n_nodes);
  k_build_sub<<<sm_count * 4, 128, 0, st>>>(d_table);
  k_check_sub<<<sm_count * 4, 128, 0, st>>>(d_table);
  return cudaGetLastError();
}

void attach_tables(PointTable* T, void* d_mem) {
  LineTables& tb = T->tab;
  unsigned char* p = static_cast<unsigned char*>(d_mem);
  tb.data = reinterpret_cast<const cplx*>(p);
  p += TAB_BYTES_DATA;
  tb.cell = reinterpret_cast<const int*>(p);
  p += TAB_BYTES_CELL;
  tb.sub = reinterpret_cast<const cplx*>(p);
  p += TAB_BYTES_SUB;
  tb.sub_bad = p;
  p += TAB_BYTES_SUB_BAD;
  tb.nblocks = reinterpret_cast<int*>(p);
  tb.block_interval = tb.nblocks + 1;
  tb.stride = T->NZ > 0 ? T->NZ : 1;
  tb.enabled = (T->NZ > 0 && d_mem) ? 1 : 0;
}

void attach_group_table(PointTable* T, int g, void* d_mem) {
  LineTables& tb = T->tab;
  unsigned char* p = static_cast<unsigned char*>(d_mem);
  tb.data = reinterpret_cast<const cplx*>(p);
  p += TAB_BYTES_GROUP_DATA;
  tb.cell = reinterpret_cast<const int*>(p);
  p += TAB_BYTES_CELL;
  tb.sub = reinterpret_cast<const cplx*>(p);
  p += TAB_BYTES_GROUP_SUB;
  tb.sub_bad = p;
  p += TAB_BYTES_SUB_BAD;
  tb.nblocks = reinterpret_cast<int*>(p);
  tb.block_interval = tb.nblocks + 1;
  tb.g_lo = g;
  tb.g_hi = g + 1;
  tb.pos0 = T->grp[g].first;
  tb.stride = T->grp[g].count;
  tb.enabled = (g >= 0 && g < T->ngroups && d_mem) ? 1 : 0;
}

// ------------------------------------------------------------------------------- finalize
// One warp per parameter point (block b reduces partials parts[i * stride + b], i < n, into res[b]).
__global__ void k_finalize(const Partial* parts, int n, int stride, double sum_w_mc, double sum_w_data,
                           double nll_shift, EvalResult* res) {
  // Neumaier compensated sums over the block partials
  __shared__ double s[4][32], c[4][32];
  const int l = threadIdx.x;
  double sum[4] = {0, 0, 0, 0}, comp[4] = {0, 0, 0, 0};
  for (int i = l; i < n; i += 32) {
    const Partial& pi = parts[(size_t)i * stride + blockIdx.x];
    const double x[4] = {pi.data, pi.mc, pi.mc_noint, pi.n_nonpos};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double t = sum[q] + x[q];
      comp[q] += (fabs(sum[q]) >= fabs(x[q])) ? (sum[q] - t) + x[q] : (x[q] - t) + sum[q];
      sum[q] = t;
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    s[q][l] = sum[q];
    c[q][l] = comp[q];
  }
  __syncwarp();
  if (l == 0) {
    double tot[4];
    for (int q = 0; q < 4; ++q) {
      double a = 0, cc = 0;
      for (int i = 0; i < 32; ++i) {
        const double x = s[q][i];
        const double t = a + x;
        cc += (fabs(a) >= fabs(x)) ? (a - t) + x : (x - t) + a;
        a = t;
        cc += c[q][i];
      }
      tot[q] = a + cc;
    }
    EvalResult r;
    r.data_term = tot[0];
    r.sumint = tot[1];
    r.sum_noint = tot[2];
    r.n_nonpos = tot[3];
    double nll = nll_shift + sum_w_data * log(tot[1] / sum_w_mc) - tot[0];
    if (fabs(tot[2] / tot[1] - 1.0) > (double)0.3f) nll += 1000.0;
    r.nll = nll;
    r.status = 0;
    res[blockIdx.x] = r;
  }
}

// ------------------------------------------------------------------------------- host side
// Resident blocks per SM of the event kernels by segment kind (from the occupancy calculator, set by
// configure_kernels); a segment launches at most sm_count times that many blocks.
static int g_occ[SMEAR_KINDS] = {1, 1, 1, 1, 1};

static int events_per_block(int kind) { return kind == SMEAR_NONE ? EV_WARPS * UNSMEARED_PER_WARP : EV_WARPS; }

int segment_blocks(const Segment& s, int sm_count) {
  const int per = events_per_block(s.kind);
  int64_t b = (s.end - s.begin + per - 1) / per;
  const int64_t cap = (int64_t)sm_count * g_occ[s.kind];
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// Blocks of the pass over a segment's deferred events (their number is known only on the device).
static int fix_blocks(const Segment& s, int sm_count) { return sm_count * g_occ[s.kind]; }

int segment_parts(const Segment& s, int sm_count, bool deferred) {
  return segment_blocks(s, sm_count) + (deferred ? fix_blocks(s, sm_count) : 0);
}

template <bool FIX, bool ZCS>
static void launch_kind_t(const EventSet& ev, int kind, int64_t begin, int64_t end, const int32_t* list,
                          const int* n_list, const PointTable* d_table, Partial* out, double* fx_out, int mode,
                          int32_t* defer, int* defer_count, int nb, const double* grid, int grid_nb,
                          cudaStream_t st) {
  switch (kind) {
    case SMEAR_NONE:
      if (ev.lgen)
        k_unsmeared<FIX, ZCS, true><<<nb, EV_THREADS, UNSMEARED_SMEM, st>>>(ev, begin, end, list, n_list, d_table,
                                                                           out, fx_out, mode, defer, defer_count);
      else
        k_unsmeared<FIX, ZCS, false><<<nb, EV_THREADS, UNSMEARED_SMEM, st>>>(ev, begin, end, list, n_list, d_table,
                                                                            out, fx_out, mode, defer, defer_count);
      break;
    case SMEAR_20:
      k_smeared<20, FIX, ZCS><<<nb, EV_THREADS, SMEARED_SMEM, st>>>(ev, begin, end, list, n_list, d_table, out,
                                                                     fx_out, 0, defer, defer_count, nullptr, 0);
      break;
    case SMEAR_30:
      k_smeared<30, FIX, ZCS><<<nb, EV_THREADS, SMEARED_SMEM, st>>>(ev, begin, end, list, n_list, d_table, out,
                                                                     fx_out, 1, defer, defer_count, nullptr, 0);
      break;
    case SMEAR_150:
      k_smeared<150, FIX, ZCS><<<nb, EV_THREADS, SMEARED_SMEM, st>>>(ev, begin, end, list, n_list, d_table, out,
                                                                      fx_out, 1, defer, defer_count, nullptr, 0);
      break;
    case SMEAR_GRID:
      k_smeared<0, FIX, ZCS><<<nb, EV_THREADS, SMEARED_SMEM, st>>>(ev, begin, end, list, n_list, d_table, out,
                                                                    fx_out, 0, defer, defer_count, grid, grid_nb);
      break;
  }
}

// The Zcs variants run when the event set carries the Zcs planes (the caller passes them only for a
// model with Zcs entries).
template <bool FIX>
static void launch_kind(const EventSet& ev, const Segment& seg, int64_t begin, int64_t end, const int32_t* list,
                        const int* n_list, const PointTable* d_table, Partial* out, double* fx_out, int mode,
                        int32_t* defer, int* defer_count, int nb, cudaStream_t st) {
  if (ev.pp3)
    launch_kind_t<FIX, true>(ev, seg.kind, begin, end, list, n_list, d_table, out, fx_out, mode, defer, defer_count,
                             nb, seg.grid, seg.grid_nb, st);
  else
    launch_kind_t<FIX, false>(ev, seg.kind, begin, end, list, n_list, d_table, out, fx_out, mode, defer, defer_count,
                              nb, seg.grid, seg.grid_nb, st);
}

// One segment: with a deferral buffer (tables on), the table-only pass over the segment and then the
// exact-capable pass over the events it deferred; without, the exact-capable pass over the segment.
static cudaError_t launch_passes(const EventSet& ev, const Segment& seg, const PointTable* d_table, Partial* out,
                                 double* fx_out, int mode, int32_t* defer, int* defer_count, int sm_count,
                                 cudaStream_t st) {
  if (seg.end <= seg.begin) return cudaSuccess;
  if (seg.kind < SMEAR_NONE || seg.kind >= SMEAR_KINDS) return cudaErrorInvalidValue;
  if (seg.kind == SMEAR_GRID && (!seg.grid || seg.grid_nb < 1 || seg.grid_nb > GRID_MAX_NB))
    return cudaErrorInvalidValue;
  const int nb = segment_blocks(seg, sm_count);
  if (defer) {
    launch_kind<false>(ev, seg, seg.begin, seg.end, seg.list, nullptr, d_table, out, fx_out, mode, defer,
                       defer_count, nb, st);
    launch_kind<true>(ev, seg, 0, 0, defer, defer_count, d_table, out ? out + nb : nullptr, fx_out, mode, nullptr,
                      nullptr, fix_blocks(seg, sm_count), st);
  } else {
    launch_kind<true>(ev, seg, seg.begin, seg.end, seg.list, nullptr, d_table, out, fx_out, mode, nullptr, nullptr,
                      nb, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_segment(const EventSet& ev, const Segment& seg, const PointTable* d_table, Partial* out,
                           double* fx_out, int32_t* defer, int* defer_count, int sm_count, cudaStream_t st) {
  return launch_passes(ev, seg, d_table, out, fx_out, 0, defer, defer_count, sm_count, st);
}

template <class K>
static cudaError_t configure_one(K kernel, size_t smem, int* occ) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e) return e;
  int n = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, EV_THREADS, smem))) return e;
  *occ = n > 0 ? n : 1;
  return cudaSuccess;
}

template <bool ZCS>
static cudaError_t configure_variant(int* occ) {
  cudaError_t e;
  int unused = 0;
  if ((e = configure_one(k_unsmeared<false, ZCS, false>, UNSMEARED_SMEM, ZCS ? &unused : &occ[SMEAR_NONE]))) return e;
  if ((e = configure_one(k_unsmeared<true, ZCS, false>, UNSMEARED_SMEM, &unused))) return e;
  if ((e = configure_one(k_unsmeared<false, ZCS, true>, UNSMEARED_SMEM, &unused))) return e;
  if ((e = configure_one(k_unsmeared<true, ZCS, true>, UNSMEARED_SMEM, &unused))) return e;
  if ((e = configure_one(k_smeared<20, false, ZCS>, SMEARED_SMEM, ZCS ? &unused : &occ[SMEAR_20]))) return e;
  if ((e = configure_one(k_smeared<30, false, ZCS>, SMEARED_SMEM, ZCS ? &unused : &occ[SMEAR_30]))) return e;
  if ((e = configure_one(k_smeared<150, false, ZCS>, SMEARED_SMEM, ZCS ? &unused : &occ[SMEAR_150]))) return e;
  if ((e = configure_one(k_smeared<0, false, ZCS>, SMEARED_SMEM, ZCS ? &unused : &occ[SMEAR_GRID]))) return e;
  if ((e = configure_one(k_smeared<0, true, ZCS>, SMEARED_SMEM, &unused))) return e;
  if ((e = configure_one(k_smeared<20, true, ZCS>, SMEARED_SMEM, &unused))) return e;
  if ((e = configure_one(k_smeared<30, true, ZCS>, SMEARED_SMEM, &unused))) return e;
  if ((e = configure_one(k_smeared<150, true, ZCS>, SMEARED_SMEM, &unused))) return e;
  return cudaSuccess;
}

cudaError_t configure_kernels() {
  cudaError_t e;
  if ((e = configure_variant<false>(g_occ))) return e;
  if ((e = configure_variant<true>(g_occ))) return e;
  return configure_batch_kernels();
}

cudaError_t launch_finalize_points(const Partial* parts, int rows, int npts, double sum_w_mc, double sum_w_data,
                                   double nll_shift, EvalResult* res, cudaStream_t st) {
  k_finalize<<<npts, 32, 0, st>>>(parts, rows, npts, sum_w_mc, sum_w_data, nll_shift, res);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const Partial* parts, int nparts, double sum_w_mc, double sum_w_data, double nll_shift,
                            EvalResult* res, cudaStream_t st) {
  k_finalize<<<1, 32, 0, st>>>(parts, nparts, 1, sum_w_mc, sum_w_data, nll_shift, res);
  return cudaGetLastError();
}

// Sum over MC events (index >= nda) of w * fx[e], w the event's weight plane; one partial per block.
__global__ void k_mc_integral(EventSet ev, const double* __restrict__ fx, Partial* parts) {
  double acc = 0;
  for (int64_t e = ev.nda + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ev.n;
       e += (int64_t)gridDim.x * blockDim.x)
    acc += fx[e] * (double)__ldg(ev.pp + 2 * ev.n_size + e);
  block_reduce_store<256>(0.0, acc, 0.0, 0.0, parts);
}

cudaError_t launch_mc_integral(const EventSet& ev, const double* fx, Partial* parts, int nblocks, EvalResult* res,
                               cudaStream_t st) {
  k_mc_integral<<<nblocks, 256, 0, st>>>(ev, fx, parts);
  k_finalize<<<1, 32, 0, st>>>(parts, nblocks, 1, 1.0, 0.0, 0.0, res);
  return cudaGetLastError();
}

cudaError_t launch_amp2(const EventSet& ev, const PointTable* d_table, double* out, int32_t* defer, int* defer_count,
                        int sm_count, cudaStream_t st) {
  const Segment seg{SMEAR_NONE, 0, ev.n, nullptr};
  return launch_passes(ev, seg, d_table, nullptr, out, 1, defer, defer_count, sm_count, st);
}

// A K-matrix group must have at most NPMAX poles.
static int G_valid_check(const KmGroup& G) { return (G.npole <= NPMAX) ? 0 : 1; }

// ------------------------------------------------------------------------------- point table
// Masses in the table range where the reference's complex square root (csqrt_branch) changes branch
// for one of the complex-mass channels (D* Sigma_c, D* Sigma_c*, D Sigma_c, D Sigma_c*): the lineshape
// jumps there, so interpolation must not straddle them.  Scan plus bisection, computed once.
// Masses where the reference's complex square root switches branch in the complex-mass channels of
// the K-matrix (the 4-channel default, or the 7-channel isospin split).
static const std::vector<double>& complex_branch_masses(bool isospin = false) {
  static std::vector<double> out[2];
  static std::once_flag once[2];
  std::call_once(once[isospin ? 1 : 0], [isospin] {
    std::vector<double>& res = out[isospin ? 1 : 0];
    std::vector<std::pair<cplx, cplx>> ch;
    if (!isospin) {
      ch = {{mk(KM_DST, 0), mk(KM_SC, KM_SC_HW)}, {mk(KM_DST, 0), mk(KM_SCST, KM_SCST_HW)},
            {mk(KM_D, 0), mk(KM_SC, KM_SC_HW)}, {mk(KM_D, 0), mk(KM_SCST, KM_SCST_HW)}};
    } else {
      const cplx dstm = mk(KMI_DSTM, 0), dst0 = mk(KMI_DST0, 0), dm = mk(KMI_DM, 0), d0 = mk(KMI_D0, 0);
      const cplx scpp = mk(KMI_SCPP, KMI_SCPP_HW), scp = mk(KMI_SCP, KMI_SCP_HW);
      const cplx scstpp = mk(KMI_SCSTPP, KMI_SCSTPP_HW), scstp = mk(KMI_SCSTP, KMI_SCSTP_HW);
      ch = {{dstm, scpp}, {dst0, scp}, {dstm, scstpp}, {dst0, scstp}, {dm, scpp}, {d0, scp}, {dm, scstpp},
            {d0, scstp}};
    }
    for (auto& cc : ch) {
      const cplx c[2] = {cc.first, cc.second};
      auto state = [&](double m) {
        const double s = m * m;
        const cplx a = c[0] + c[1], b = c[0] - c[1];
        const cplx p = (a * a - mk(s, 0)) * (b * b - mk(s, 0));
        if (fabs(p.re) < PWA_F(0.000001f) && fabs(p.im) < PWA_F(0.000001f)) return 2;
        return (signbit(p.im) && fabs(p.im / p.re) > PWA_F(0.001f)) ? 1 : 0;
      };
      const double lo = TAB_M_LO - 1e-3, hi = TAB_M_HI + 1e-3, dm = 1e-6;
      double prev_m = lo;
      int prev = state(lo);
      for (double m = lo + dm; m <= hi; m += dm) {
        const int st = state(m);
        if (st != prev) {
          double a = prev_m, b = m;
          for (int it = 0; it < 60; ++it) {
            const double c2 = 0.5 * (a + b);
            (state(c2) == prev ? a : b) = c2;
          }
          res.push_back(0.5 * (a + b));
          prev = st;
        }
        prev_m = m;
      }
    }
  });
  return out[isospin ? 1 : 0];
}

static bool nonzero_host(cplx c) { return c.re != 0.0 || c.im != 0.0; }

// Decodes the float parameter block (layout of cu_init_data, RooDalitzAmplitude.cxx:3141-3210;
// coupling offsets of cuda_configure_ampcount, kernel_calEva.cu:1014-1098; K-matrix output slots
// of cuda_configure_Pc_KMatrix, :978-1010) and hoists every parameter-only constant.
int build_point_table(const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                      float ffr, float ffb, PointTable* T, int flags) {
  const bool isospin = (flags & BUILD_KM_ISOSPIN) != 0;
  std::memset(T, 0, sizeof(PointTable));
  if (NR > MAX_LSTAR || NZ > MAX_PC || NX > MAX_ZCS || NR < 0 || NZ < 0 || NX < 0) return 4;  // PWA_E_SIZE
  if (para_size != NSET * (NR + NZ + NX)) return 3;                                           // PWA_E_LAYOUT
  T->NR = NR;
  T->NZ = NZ;
  T->NX = NX;
  T->ffr = ffr;
  T->ffb = ffb;
  const double mmin = M_K + M_P, mmax = M_LB - M_JPSI;
  const double thr_pk = (double)(float)(M_P + M_K);
  const double thr_pz = (double)(float)(M_P + M_JPSI);
  int cnt = para_size;
  // spline blocks follow the couplings, Lambda* waves first (cuda_configure_splcount,
  // kernel_calEva.cu:1100-1135)
  int splcount = para_size + vamp_size, spl_used = 0;
  const int spl_end = para_size + vamp_size + spline_size;
  auto take_spline = [&](int knots, int* aux) -> int {
    const int nf = 9 * knots;
    if (splcount + nf > spl_end) return 3;  // PWA_E_LAYOUT
    if (spl_used + nf > SPL_FLOATS) return 4;
    std::memcpy(T->spl + spl_used, pl + splcount, nf * sizeof(float));
    *aux = spl_used;
    spl_used += nf;
    splcount += nf;
    return 0;
  };
  // revised K-matrix entry of chain c: own-term constants in the chain's two-body system (threshold
  // thr, upper edge hi) and the p K constants of its KMatrixTerm
  auto take_rkm = [&](int c, const float* q, int* aux) -> int {
    if (T->nrkm[c] >= MAX_RKM) return 4;
    RkmEntry& R = T->rkm[c][T->nrkm[c]];
    *aux = T->nrkm[c]++;
    R.m = q[0];
    R.g = q[1];
    R.LR = (int)q[3];
    if (R.LR < 0 || R.LR > 5) return 5;
    R.set = (int)q[2] * 2 + ((int)q[5] > 0 ? 1 : 0);
    const double m1 = c ? M_JPSI : M_P, m2 = c ? M_P : M_K, m3 = c ? M_K : M_JPSI;
    const double thr = c ? (double)(float)(M_JPSI + M_P) : (double)(float)(M_P + M_K);
    const double lo = m1 + m2, hi = M_LB - m3;
    const double mc = (R.m > thr) ? R.m : (R.m >= 0) ? tanh_eff_mass(R.m, lo, hi) : (lo + hi) / 2.0;
    const double pc = two_body_p(mc, m1, m2);
    R.inv_pR0c = 1.0 / pc;
    R.polyR0c = bw_poly(R.LR, sq(T->ffr * pc));
    R.branch = (R.m <= 0) ? 3 : (R.m > thr) ? 0 : (R.m < thr) ? 1 : 2;
    if (R.branch == 1) R.inv_pR0sp = 1.0 / two_body_p(R.m, PWA_F(1.18937f), PWA_F(0.13957018f));
    R.factor = (R.m > 0) ? bw_norm(R.m, R.g) : 1.0;
    const double mk_ = (R.m > thr_pk) ? R.m : (R.m >= 0) ? tanh_eff_mass(R.m, mmin, mmax) : (mmin + mmax) / 2.0;
    const double pk = two_body_p(mk_, M_P, M_K);
    R.inv_pR0k = 1.0 / pk;
    R.polyR0k = bw_poly(R.LR, sq(T->ffr * pk));
    return 0;
  };
  auto coupling = [&](int idx) -> cplx {
    const float a = pl[idx], b = pl[idx + 1];
    // the reference skips couplings with float |c| < 1e-10 (kernel_calEva.cu:174,481)
    if (std::sqrt((double)a * a + (double)b * b) < 1e-10) return mk(0, 0);
    return mk(a, b);
  };
  for (int r = 0; r < NR; ++r) {
    const float* q = pl + r * NSET;
    LstarEntry& L = T->L[r];
    const int S2 = (int)q[2], type = (int)q[4];
    L.m_r = q[0];
    L.g_r = q[1];
    L.LR = (int)q[3];
    if (S2 < 1 || S2 > 9 || (S2 % 2) == 0) return 6;  // PWA_E_PARAM
    L.sidx = (S2 - 1) / 2;
    L.ncm = (S2 == 1) ? 4 : 6;
    if (type == REF_BREITWIGNER) {
      L.type = LT_BW;
    } else if (type == REF_NONRESONANT) {
      L.type = LT_NR;
    } else if (type == REF_MODELINDEPENDENT) {
      L.type = LT_SPLINE;
      if (int e = take_spline(SPL_KNOTS_L, &L.aux)) return e;
    } else if (type == REF_REVISEDKMATRIX) {
      L.type = LT_RKM;
      if (int e = take_rkm(0, q, &L.aux)) return e;
    } else {
      return 5;
    }
    const double m_r = L.m_r;
    if (m_r < 0) {
      L.branch = 2;
      L.pR0 = two_body_p((mmin + mmax) / 2.0, M_P, M_K);
    } else if (m_r > thr_pk) {
      L.branch = 0;
      L.pR0 = two_body_p(m_r, M_P, M_K);
    } else if (m_r > 0 && m_r < (double)1.43f) {
      L.branch = 1;
      L.pR0_sp = two_body_p(m_r, PWA_F(1.18937f), PWA_F(0.13957018f));
    } else if (m_r > 1e-10) {
      L.branch = 3;
      L.pR0 = two_body_p(tanh_eff_mass(m_r, mmin, mmax), M_P, M_K);
    } else {
      L.branch = 4;
    }
    L.polyR0 = bw_poly(L.LR, sq(T->ffr * L.pR0));
    L.norm = bw_norm(m_r, L.g_r);
    L.inv_pR0 = (L.pR0 != 0) ? 1.0 / L.pR0 : 0.0;
    L.sqrt_polyR0 = std::sqrt(L.polyR0);
    L.inv_pR0_sp = (L.pR0_sp != 0) ? 1.0 / L.pR0_sp : 0.0;
    if (L.type == LT_BW && (L.branch == 0 || L.branch == 3) && L.LR >= 1 && L.LR <= 5) T->lmask_lstar_R |= 1 << L.LR;
    if (L.type == LT_BW && L.branch == 1) T->needs_sigma_pi = 1;
    if (L.LR > 5) return 5;
    // Lambda_b barrier constants (BTerm; a spline wave passes mass -0.5, kernel_calEva.cu:143)
    const double J = 0.5 * S2;
    L.LB = (J <= 1) ? 0 : (int)(J - 1.5);
    const double mb = (L.type == LT_SPLINE) ? -0.5 : m_r;
    double pB0 = -1;
    if (mb < 0) pB0 = two_body_p(M_LB, M_JPSI, (mmin + mmax) / 2.0);
    if (mb > 1e-10 && mb + M_JPSI < M_LB) pB0 = two_body_p(M_LB, M_JPSI, mb);
    if (mb + M_JPSI > M_LB) pB0 = two_body_p(M_LB, M_JPSI, tanh_eff_mass(mb, mmin, mmax));
    if (pB0 < 0) return 6;  // resonance mass in [0, 1e-10]: barrier momentum undefined
    L.pB0 = pB0;
    L.polyB0 = bw_poly(L.LB, sq(T->ffb * pB0));
    L.lb_scale = ipow(M_LB / pB0, L.LB);
    L.sqrt_polyB0 = std::sqrt(L.polyB0);
    if (L.LB >= 1 && L.LB <= 5) T->lmask_lstar_B |= 1 << L.LB;
    if (L.LB > 5) return 5;
    for (int k = 0; k < 2; ++k)
      for (int m = 0; m < 6; ++m) {
        if (S2 == 1 && m >= 4) continue;
        L.c[k * 6 + m] = coupling(cnt);
        cnt += 2;
      }
  }
  int per_group[4] = {0, 0, 0, 0};
  for (int i = 0; i < NZ; ++i) {
    const int r = NR + i;
    const float* q = pl + r * NSET;
    PcEntry& Z = T->Z[i];
    const int S2 = (int)q[2], type = (int)q[4];
    Z.LR = (int)q[3];
    Z.m_r = q[0];
    Z.g_r = q[1];
    if (S2 < 1 || S2 > 7 || (S2 % 2) == 0) return 6;
    Z.sidx = (S2 - 1) / 2;
    if (type == REF_BREITWIGNER) {
      Z.type = LT_BW;
    } else if (type == REF_KMATRIX) {
      Z.type = LT_KM;
    } else if (type == REF_NONRESONANT) {
      Z.type = LT_NR;
    } else if (type == REF_MODELINDEPENDENT) {
      Z.type = LT_SPLINE;
      if (int e = take_spline(SPL_KNOTS_Z, &Z.aux)) return e;
    } else if (type == REF_REVISEDKMATRIX) {
      Z.type = LT_RKM;
      if (int e = take_rkm(1, q, &Z.aux)) return e;
    } else if (type == REF_TRIANGLE) {
      Z.type = LT_CUSP;
    } else {
      return 5;
    }
    if (Z.type == LT_KM) {
      Z.group = (Z.LR > 0) ? ((S2 == 3) ? 3 : 2) : ((S2 == 3) ? 1 : 0);
      if (S2 > 3) return 5;
      Z.slot = per_group[Z.group]++;
      if (Z.slot >= NPMAX + NKMC) return 4;
    }
    if (Z.type == LT_BW) {
      Z.bw_above = Z.m_r > thr_pz;
      Z.pR0 = Z.bw_above ? two_body_p(Z.m_r, M_P, M_JPSI) : 0.0;
      Z.polyR0 = bw_poly(Z.LR, sq(T->ffr * Z.pR0));
      Z.norm = bw_norm(Z.m_r, Z.g_r);
      Z.inv_pR0 = (Z.pR0 != 0) ? 1.0 / Z.pR0 : 0.0;
      Z.sqrt_polyR0 = std::sqrt(Z.polyR0);
      if (Z.bw_above && Z.LR >= 1 && Z.LR <= 5) T->lmask_pc_R |= 1 << Z.LR;
      if (Z.LR > 5) return 5;
    }
    const double J = 0.5 * S2;
    Z.LB = (int)(J - 0.5);
    const double mbz = (Z.type == LT_SPLINE) ? -0.5 : Z.m_r;  // BTermZ mass (kernel_calEva.cu:408)
    double pB0 = -1;
    if (mbz < 0) pB0 = two_body_p(M_LB, M_K, (M_JPSI + M_P + M_LB - M_K) / 2.0);
    if (mbz > 1e-10 && mbz + M_K < M_LB) pB0 = two_body_p(M_LB, M_K, mbz);
    Z.pB0_event = (pB0 < 0);
    Z.pB0 = pB0;
    Z.polyB0 = bw_poly(Z.LB, sq(T->ffb * pB0));
    Z.sqrt_polyB0 = std::sqrt(Z.polyB0);
    if (!Z.pB0_event && Z.LB >= 1 && Z.LB <= 5) T->lmask_pc_B |= 1 << Z.LB;
    if (Z.LB > 5) return 5;
    const double S = 0.5 * S2;
    for (int k = 0; k < 2; ++k) {
      int m = 0;
      for (int hpsi = -1; hpsi <= 1; ++hpsi)
        for (int ihz = 0; ihz < 2; ++ihz)
          for (int ihp = 0; ihp < 2; ++ihp) {
            const double hp = ihp ? 0.5 : -0.5;
            if (!(std::fabs(hpsi - hp) > S)) {
              Z.c[k * 12 + m] = coupling(cnt);
              cnt += 2;
            }
            ++m;
          }
    }
  }
  // Zcs entries (GetAmpZcs, kernel_calEva.cu:192-286; BTermX / BW_AMPX, cu_DPFPropogator.cu:205-246).
  // The kernel uses a Breit-Wigner whatever the type field says.
  const double thr_xk = (double)(float)(M_K + M_JPSI);
  for (int x = 0; x < NX; ++x) {
    const float* q = pl + (NR + NZ + x) * NSET;
    XEntry& X = T->X[x];
    const int S2 = (int)q[2];
    if (S2 < 0 || S2 > 6 || (S2 % 2) != 0) return 6;
    X.m_r = q[0];
    X.g_r = q[1];
    X.LR = (int)q[3];
    if (X.LR < 0 || X.LR > 5) return 5;
    X.sidx = S2 / 2;
    const double S = 0.5 * S2;
    X.bw_above = X.m_r > thr_xk;
    const double pR0 = X.bw_above ? two_body_p(X.m_r, M_K, M_JPSI) : 0.0;
    X.norm = bw_norm(X.m_r, X.g_r);
    X.inv_pR0 = (pR0 != 0) ? 1.0 / pR0 : 0.0;
    X.sqrt_polyR0 = std::sqrt(bw_poly(X.LR, sq(T->ffr * pR0)));
    if (X.bw_above && X.LR >= 1) T->lmask_x_R |= 1 << X.LR;
    X.LB = (int)(S - 0.5);  // C truncation toward zero
    if (X.LB > 5) return 5;
    if (X.m_r < 0) {
      X.lb_mode = 2;
    } else if (X.m_r > 1e-10 && X.m_r + M_P < M_LB) {
      X.lb_mode = 0;
      X.sqrt_polyB0 = std::sqrt(bw_poly(X.LB, sq(T->ffb * two_body_p(M_LB, M_P, X.m_r))));
      if (X.LB >= 1) T->lmask_x_B |= 1 << X.LB;
    } else {
      X.lb_mode = 1;
    }
    // the kernel reads N(J) consecutive couplings per proton helicity from the resonance's offset
    // (lambda_p in {0, 1}, lambda_Zcs = lambda_p -+ 1/2); the block holds ConfigureCouplings' count
    // (lambda_p = -+1/2)
    const int base = cnt;
    int rd = base;
    for (int k = 0; k < 2; ++k) {
      int m = 0;
      for (int hpsi = -1; hpsi <= 1; ++hpsi) {
        if (std::abs(hpsi) > S) continue;
        for (int hp = 0; hp <= 1; ++hp)
          for (int iz = 0; iz < 2; ++iz) {
            if (std::fabs(hp - 0.5 + iz) > S) continue;
            X.c[k * 12 + m] = coupling(rd);
            rd += 2;
            ++m;
          }
      }
    }
    for (int k = 0; k < 2; ++k)
      for (int hpsi = -1; hpsi <= 1; ++hpsi) {
        if (std::abs(hpsi) > S) continue;
        for (int ihp = 0; ihp < 2; ++ihp)
          for (int ihz = 0; ihz < 2; ++ihz) {
            const double hz = (ihp ? 0.5 : -0.5) + (ihz ? 0.5 : -0.5);
            if (!(std::fabs(hz) > S)) cnt += 2;
          }
      }
    if (rd > cnt) return 3;
    for (int k = 0; k < 2; ++k)
      for (int m = 0; m < 12; ++m)
        if (nonzero_host(X.c[k * 12 + m])) T->x_mmask[k] |= 1 << m;
  }
  if (cnt != para_size + vamp_size) return 3;
  if (splcount != spl_end) return 3;  // the spline blocks must fill spline_size exactly
  // K-matrix groups (Default_KMatrix pole scan and near-threshold mass shift, :674-746)
  const int kmcount = para_size + vamp_size + spline_size;
  for (int ik = 0; ik < 4; ++ik) {
    KmGroup& G = T->G[ik];
    G.J2 = (ik == 1 || ik == 3) ? 3 : 1;
    G.P = (ik >= 2) ? 1 : -1;
    G.Lna = (G.P == 1) ? 1 : 0;
    G.iso = isospin ? 1 : 0;
    const float* g_alpha = pl + kmcount + ik * (NPMAX + NKMC) * NKMC;
    const float* f_scat = g_alpha + NPMAX * NKMC;
    for (int i = 0; i < NKMC; ++i)
      for (int j = 0; j < NKMC; ++j) G.f[i][j] = f_scat[i * NKMC + j];
    int np = 0;
    for (int r = NR; r < NR + NZ; ++r) {
      const float* q = pl + r * NSET;
      if (!((int)q[4] == REF_KMATRIX && (int)q[2] == G.J2 && (int)q[5] == G.P && q[0] > 0)) continue;
      if (np >= NPMAX) return 4;
      const double mfit = q[0];
      const int ich = (int)q[1];
      double m0 = mfit;
      if (ich > 0 && isospin) {
        // Isospin_KMatrix (cu_DPFPropogator.cu:455-489): channels 1 and 3 only, the shift
        // Re(i g^2 / 3 (2 rho_charged + rho_neutral))
        const double mfit2 = mfit * mfit;
        cplx ra, rb;
        if (ich == 1) {
          ra = rho_complex(mfit2, mk(KMI_DSTM, 0), mk(KMI_SCPP, KMI_SCPP_HW));
          rb = rho_complex(mfit2, mk(KMI_DST0, 0), mk(KMI_SCP, KMI_SCP_HW));
        } else if (ich == 3) {
          ra = rho_complex(mfit2, mk(KMI_DM, 0), mk(KMI_SCPP, KMI_SCPP_HW));
          rb = rho_complex(mfit2, mk(KMI_D0, 0), mk(KMI_SCP, KMI_SCP_HW));
        } else {
          return 6;  // the reference prints "An unacceptable channel" and reads an unset mass
        }
        const double g = g_alpha[np * NKMC + ich];
        const cplx shift = mk(0, g * g / 3.0) * (ra * 2.0 + rb);
        m0 = std::sqrt(mfit2 + shift.re);
      } else if (ich > 0) {
        const double mfit2 = mfit * mfit;
        cplx rch;
        if (ich == 1)
          rch = rho_complex(mfit2, mk(KM_DST, 0), mk(KM_SC, KM_SC_HW));
        else if (ich == 2)
          rch = rho_complex(mfit2, mk(KM_D, 0), mk(KM_SCST, KM_SCST_HW));
        else if (ich == 3)
          rch = rho_complex(mfit2, mk(KM_D, 0), mk(KM_SC, KM_SC_HW));
        else
          return 6;
        const double g = g_alpha[np * NKMC + ich];
        const cplx shift = mk(0, g * g) * rch;
        m0 = std::sqrt(mfit2 + shift.re);
      } else if (ich < 0) {
        return 6;
      }
      G.m0sq[np] = m0 * m0;
      for (int j = 0; j < NKMC; ++j) G.g[np][j] = g_alpha[np * NKMC + j];
      ++np;
    }
    G.npole = np;
  }
  // groups: K-matrix J^P groups in order of first appearance, other entries singly
  int ng = 0, pos = 0;
  bool done[4] = {false, false, false, false};
  for (int i = 0; i < NZ; ++i) {
    const PcEntry& Z = T->Z[i];
    if (Z.type == LT_KM) {
      if (done[Z.group]) continue;
      done[Z.group] = true;
      PcGroup& g = T->grp[ng++];
      g.km = Z.group;
      g.sidx = Z.sidx;
      g.first = pos;
      g.count = 0;
      for (int j = 0; j < NZ; ++j)
        if (T->Z[j].type == LT_KM && T->Z[j].group == Z.group) {
          T->order[pos++] = j;
          if (++g.count > MAX_GROUP_ENTRIES) return 4;
        }
      if (G_valid_check(T->G[Z.group]) != 0) return 6;
    } else if (Z.type == LT_RKM) {  // a revised K-matrix set: its entries' lineshapes depend on each other
      const int set = T->rkm[1][Z.aux].set;
      bool seen = false;
      for (int j = 0; j < i; ++j) seen |= (T->Z[j].type == LT_RKM && T->rkm[1][T->Z[j].aux].set == set);
      if (seen) continue;
      PcGroup& g = T->grp[ng++];
      g.km = -1;
      g.sidx = Z.sidx;
      g.first = pos;
      g.count = 0;
      for (int j = i; j < NZ; ++j)
        if (T->Z[j].type == LT_RKM && T->rkm[1][T->Z[j].aux].set == set) {
          T->order[pos++] = j;
          ++g.count;
        }
    } else {
      PcGroup& g = T->grp[ng++];
      g.km = -1;
      g.sidx = Z.sidx;
      g.first = pos;
      g.count = 1;
      T->order[pos++] = i;
    }
  }
  T->ngroups = ng;
  // helicity slots m with a non-zero coupling, per proton helicity k: Lambda* entries, all Pc
  // entries, each Pc group
  for (int r = 0; r < NR; ++r)
    for (int k = 0; k < 2; ++k)
      for (int m = 0; m < 6; ++m) {
        const cplx c = T->L[r].c[k * 6 + m];
        if (c.re != 0.0 || c.im != 0.0) T->lstar_mmask[k] |= 1 << m;
      }
  for (int g = 0; g < ng; ++g) {
    PcGroup& gr = T->grp[g];
    for (int q = 0; q < gr.count; ++q)
      for (int k = 0; k < 2; ++k)
        for (int m = 0; m < 12; ++m) {
          const cplx c = T->Z[T->order[gr.first + q]].c[k * 12 + m];
          if (c.re != 0.0 || c.im != 0.0) gr.mmask[k] |= 1 << m;
        }
    T->pc_mmask[0] |= gr.mmask[0];
    T->pc_mmask[1] |= gr.mmask[1];
  }
  // plane slots the amplitude reads: masses and weight, the Lambda* angular factors and the
  // d-functions of the spins in use for the helicity slots in use, likewise for Pc and Zcs
  {
    bool use[SLOT_ALL] = {};
    use[0] = use[1] = use[2] = true;
    const int lm = T->lstar_mmask[0] | T->lstar_mmask[1];
    for (int r = 0; r < NR; ++r)
      for (int k = 0; k < 2; ++k)
        for (int m = 0; m < 6; ++m)
          if (lm >> m & 1) {
            for (int ij = 0; ij < 4; ++ij) use[3 + ((ij >> 1) * 12 + (ij & 1) * 6 + m) * 2] =
                use[4 + ((ij >> 1) * 12 + (ij & 1) * 6 + m) * 2] = true;
            use[51 + T->L[r].sidx * 12 + k * 6 + m] = true;
          }
    const int pm = T->pc_mmask[0] | T->pc_mmask[1];
    for (int i = 0; i < NZ; ++i)
      for (int k = 0; k < 2; ++k)
        for (int m = 0; m < 12; ++m)
          if (pm >> m & 1) {
            for (int ij = 0; ij < 4; ++ij) use[SLOT_PP1 + ((ij >> 1) * 24 + (ij & 1) * 12 + m) * 2] =
                use[SLOT_PP1 + 1 + ((ij >> 1) * 24 + (ij & 1) * 12 + m) * 2] = true;
            use[SLOT_PP2 + T->Z[i].sidx * 24 + k * 12 + m] = true;
          }
    if (NX > 0) use[SLOT_PP3] = true;
    const int xm = T->x_mmask[0] | T->x_mmask[1];
    for (int x = 0; x < NX; ++x)
      for (int k = 0; k < 2; ++k)
        for (int m = 0; m < 12; ++m)
          if (xm >> m & 1) {
            for (int ij = 0; ij < 4; ++ij) use[SLOT_PP3 + 1 + ((ij >> 1) * 24 + (ij & 1) * 12 + m) * 2] =
                use[SLOT_PP3 + 2 + ((ij >> 1) * 24 + (ij & 1) * 12 + m) * 2] = true;
            use[SLOT_PP4 + T->X[x].sidx * 24 + k * 12 + m] = true;
          }
    T->nstage = 0;
    for (int i = 0; i < SLOT_ALL; ++i)
      if (use[i]) T->stage[T->nstage++] = (short)i;
  }
  // table grid and guard intervals (tables stay disabled until the caller attaches table memory)
  LineTables& tb = T->tab;
  tb.enabled = 0;
  tb.n_nodes = TAB_NODES;
  tb.m_lo = TAB_M_LO;
  tb.h = TAB_H;
  tb.inv_h = 1.0 / TAB_H;
  tb.g_lo = 0;
  tb.g_hi = ng;
  tb.pos0 = 0;
  tb.nguard = 0;
  auto guard = [&](double m, double half) {
    if (tb.nguard < MAX_GUARDS && m > TAB_M_LO - 1e-3 && m < TAB_M_HI + 1e-3) {
      tb.guard_lo[tb.nguard] = m - half;
      tb.guard_hi[tb.nguard] = m + half;
      ++tb.nguard;
    }
  };
  const double cusp = 3e-4, step = 3.5 * TAB_H;
  guard(M_P + M_JPSI, cusp);  // J/psi p threshold
  guard(M_LB - M_K, cusp);    // upper kinematic edge (production barrier momentum)
  bool neg_parity = false, pos_parity = false;
  for (int ik = 0; ik < 4; ++ik) {
    bool used = false;
    for (int g = 0; g < ng; ++g) used |= (T->grp[g].km == ik);
    if (!used) continue;
    (T->G[ik].P == 1 ? pos_parity : neg_parity) = true;
    for (int p = 0; p < T->G[ik].npole; ++p) {  // pole clamp |m0^2 - s| < 1e-3
      const double a = T->G[ik].m0sq[p] - KM_DENORM_MIN, b = T->G[ik].m0sq[p] + KM_DENORM_MIN;
      if (a > 0) guard(std::sqrt(a), step);
      guard(std::sqrt(b), step);
    }
  }
  if (pos_parity && !isospin) {  // real-mass channel thresholds of the positive-parity groups
    guard(KM_DST + KM_SC, cusp);
    guard(KM_D + KM_SC, cusp);
    guard(KM_D + KM_SCST, cusp);
  }
  if (pos_parity && isospin) {
    guard(KMI_DSTM + KMI_SCPP, cusp);
    guard(KMI_DST0 + KMI_SCP, cusp);
    guard(KMI_DM + KMI_SCPP, cusp);
    guard(KMI_D0 + KMI_SCP, cusp);
    guard(KMI_DM + KMI_SCSTPP, cusp);
    guard(KMI_D0 + KMI_SCSTP, cusp);
  }
  if (neg_parity)
    for (double m : complex_branch_masses(isospin)) guard(m, step);
  // spline waves drop to zero outside their domain
  bool pc_spline = false;
  for (int i = 0; i < NZ; ++i) pc_spline |= (T->Z[i].type == LT_SPLINE);
  if (pc_spline) {
    guard(SPL_Z_LO, cusp);
    guard(SPL_Z_HI, cusp);
  }
  if (tb.nguard >= MAX_GUARDS) return 4;
  return 0;
}

// Host evaluation of the decoded lineshapes (diagnostics and CPU tests of the point table): Lambda*
// lineshape x production barrier at mkp, and every Pc entry's lineshape x barrier at mz, entries in
// parameter-block order.
void host_lineshapes(const PointTable& T, double mkp, double mz, cplx* lstar, cplx* pc) {
  const LstarKin lk = lstar_kin(T, mkp);
  const PcKin pk = pc_kin(T, mz);
  for (int r = 0; r < T.NR; ++r) lstar[r] = lstar_lineshape(T, r, lk);
  cplx raw[MAX_PC];
  for (int g = 0; g < T.ngroups; ++g) pc_group_exact(T, g, pk, raw + T.grp[g].first);
  for (int q = 0; q < T.NZ; ++q) pc[T.order[q]] = raw[q];
}

}  // namespace pwa
