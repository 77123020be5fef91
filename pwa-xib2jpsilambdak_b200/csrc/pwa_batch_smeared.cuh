// The batched kernel for smeared event classes (k_batch) and its helpers.  The kernel template is
// instantiated per offset scheme in its own translation unit (pwa_batch_nb.inc, included by
// pwa_batch_s20.cu, pwa_batch_s30.cu, pwa_batch_s150.cu, pwa_batch_grid.cu), which export the host
// wrappers declared at the end; the batched evaluation's host logic is in pwa_batch.cu.
#pragma once
#include "pwa_device.cuh"

namespace pwa {

constexpr int BATCH_WARPS = 4;
constexpr int BATCH_THREADS = BATCH_WARPS * 32;
constexpr int BATCH_MAXQ = 8;     // Lambda* entries with coupling differences per Lambda* point
constexpr int BATCH_MAXQ_PC = 4;  // Pc entries per coupling point (a shared coupling moves up to 4)
constexpr int N_PLANES = 303;  // pp 111 + pp1 96 + pp2 96
// Points whose values wait per warp until an event's table checks are known: the passes that hold
// lineshape points (at most 128 per batch, and they come first).
constexpr int BATCH_VBUF = 128;

// Per-warp shared-memory layout of the batched kernel for a model with NR Lambda* and NZ Pc entries.
struct BatchLayout {
  int nzp, rs;  // Pc entries rounded up to 4; row stride of R (odd, conflict-free row writes)
  size_t bs, lk, q0, f0, hl0, hx0, a10, a20, hz, R, S0, G, P, R1, Y, R0, s00, vbuf, warp_bytes, acc, total;
};
__host__ __device__ inline size_t bal16(size_t x) { return (x + 15) & ~size_t(15); }
// Coupling points from the centre's row moments when the offset rows fit one round (20 and 30
// offsets: fewer instructions per event); with several rounds (150 offsets, the weighted grid, NB = 0)
// the row loops measured faster, and without the moment buffers the blocks leave more of the unified
// L1 to the table lookups.
__host__ __device__ constexpr bool batch_moments(int nb) { return nb > 0 && nb + 1 <= 32; }
// Offset rows a round holds: the lookups of one event (with the row at the event mass) for 20 and 30
// offsets, a full round of 32 otherwise.
__host__ __device__ constexpr int batch_row_cap(int nb) { return nb > 0 && nb + 1 <= 32 ? nb + 1 : 32; }

__host__ __device__ inline BatchLayout batch_layout(int NR, int NZ, int npts, bool moments, int row_cap) {
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
  L.hx0 = o;
  o = bal16(o + 8 * sizeof(cplx));
  L.a10 = o;
  o = bal16(o + 8 * sizeof(cplx));
  L.a20 = o;
  o = bal16(o + 8 * sizeof(double));
  L.hz = o;
  o = bal16(o + (size_t)(L.nzp > 0 ? L.nzp : 1) * 8 * sizeof(cplx));
  L.R = o;
  o = bal16(o + (size_t)row_cap * L.rs * sizeof(cplx));
  L.S0 = o;
  o = bal16(o + (size_t)row_cap * 9 * sizeof(cplx));
  // moments of the centre's offset rows (coupling points): G triangle, P [q][h], R1, Y, row 0
  const size_t nq = moments ? (size_t)(L.nzp > 0 ? L.nzp : 1) : 0;
  L.G = o;
  o = bal16(o + nq * (nq + 1) / 2 * sizeof(cplx));
  L.P = o;
  o = bal16(o + nq * 8 * sizeof(cplx));
  L.R1 = o;
  o = bal16(o + nq * sizeof(cplx));
  L.Y = o;
  o = bal16(o + nq * sizeof(cplx));
  L.R0 = o;
  o = bal16(o + nq * sizeof(cplx));
  L.s00 = o;
  o = bal16(o + 8 * sizeof(cplx));
  L.vbuf = o;
  o = bal16(o + (size_t)(npts < BATCH_VBUF ? npts : BATCH_VBUF) * 2 * sizeof(double));
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

// Lineshape of every entry of group g at mass m from the point's table (a table of every group, or
// of group g alone; false when it cannot serve m), or exactly.
template <bool FIX>
__device__ __forceinline__ bool group_lineshapes(const PointTable& T, int g, double m, cplx (&out)[MAX_GROUP_ENTRIES]) {
  const PcGroup& gr = T.grp[g];
  const int first = gr.first, cnt = gr.count;
  TabAt ta;
  if (tab_at(T.tab, m, ta)) {
#pragma unroll
    for (int q = 0; q < MAX_GROUP_ENTRIES; ++q) {
      if (q >= cnt) break;
      out[q] = tab_get(ta, T.tab.stride, first - T.tab.pos0 + q);
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

// Index of the entry pair (a, b), a <= b < n, in a packed upper triangle.
__host__ __device__ __forceinline__ int gtri(int a, int b, int n) { return a * n - a * (a - 1) / 2 + (b - a); }

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
template <int NB, bool FIX, bool ZCS>
__global__ void __launch_bounds__(BATCH_THREADS)
    k_batch(EventSet ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list,
            const PointTable* __restrict__ T0p, const BatchPoint* __restrict__ pts, int npts, Partial* parts,
            int band, int32_t* defer, int* defer_count, const double* __restrict__ grid, int grid_nb) {
  extern __shared__ __align__(16) unsigned char sm[];
  const PointTable& T0 = *T0p;
  const int NR = T0.NR, NZ = T0.NZ;
  constexpr bool has_x = ZCS;  // Zcs entries (their amplitudes join the centre's H_L)
  constexpr int RC = batch_row_cap(NB);  // rows held per round
  const BatchLayout Ly = batch_layout(NR, NZ, npts, batch_moments(NB), RC);
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  unsigned char* wb = sm + warp * Ly.warp_bytes;
  double* bs = reinterpret_cast<double*>(wb + Ly.bs);
  LstarKin* lks = reinterpret_cast<LstarKin*>(wb + Ly.lk);  // the event's Lambda* kinematics
  cplx* q0 = reinterpret_cast<cplx*>(wb + Ly.q0);
  cplx* f0 = reinterpret_cast<cplx*>(wb + Ly.f0);  // [r][h]
  cplx* hl0 = reinterpret_cast<cplx*>(wb + Ly.hl0);  // Lambda* + Zcs amplitudes of the centre
  cplx* hx0 = reinterpret_cast<cplx*>(wb + Ly.hx0);  // the Zcs part alone (non-interfering term)
  cplx* a10 = reinterpret_cast<cplx*>(wb + Ly.a10);
  double* a20 = reinterpret_cast<double*>(wb + Ly.a20);
  cplx* hz = reinterpret_cast<cplx*>(wb + Ly.hz);  // [q][h]
  cplx* R = reinterpret_cast<cplx*>(wb + Ly.R);    // [row][q], stride Ly.rs
  cplx* S0 = reinterpret_cast<cplx*>(wb + Ly.S0);  // [row][h], stride 9
  cplx* G = reinterpret_cast<cplx*>(wb + Ly.G);    // sum_b w_b conj(R_bq) R_bq', q <= q' (gtri)
  cplx* P = reinterpret_cast<cplx*>(wb + Ly.P);    // [q][h]: sum_b w_b conj(S0_bh) R_bq
  cplx* R1 = reinterpret_cast<cplx*>(wb + Ly.R1);  // sum_b w_b R_bq
  cplx* Y = reinterpret_cast<cplx*>(wb + Ly.Y);    // sum_h conj(H_L[h]) HZ_q[h]
  cplx* R0 = reinterpret_cast<cplx*>(wb + Ly.R0);  // R_0q: the row at the event mass (band 0)
  cplx* s00 = reinterpret_cast<cplx*>(wb + Ly.s00);  // S0_0h
  double* vbuf = reinterpret_cast<double*>(wb + Ly.vbuf);
  double* acc = reinterpret_cast<double*>(sm + Ly.acc);  // [p][4]
  __shared__ int s_npcg;
  if (threadIdx.x == 0) s_npcg = 0;
  for (int i = threadIdx.x; i < npts * 4; i += BATCH_THREADS) acc[i] = 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < npts; i += BATCH_THREADS)
    if (pts[i].kind == BP_PCG) atomicMax(&s_npcg, i + 1);
  __syncthreads();
  // The lineshape points' table lookups decide whether an event is deferred (FIX = false): the values
  // of the passes up to the last lineshape point wait in vbuf until then, later passes go straight to
  // the sums, and a deferred event stops there.  A batch with lineshape points beyond the buffer's
  // reach (the host never builds one) defers every event to the exact pass.
  const int pcg_end = FIX ? 0 : (s_npcg + 31) & ~31;
  const bool vb_overflow = !FIX && min(pcg_end, npts) > BATCH_VBUF;

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
  constexpr bool MOMENTS = batch_moments(NB);
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
      if (lane < NR) q0[lane] = lstar_lineshape(T0, lane, lk);
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
      if (part == 0) {
        cplx hx = mk(0, 0);
        if (has_x) zcs_amplitudes<1>(T0, EvX{ev.pp3, ev.pp4, ev.n_size, e}, h8 & 1, h8 >> 1, &hx);
        hx0[h8] = hx;
        hl0[h8] = hl + hx;
      }
      for (int q = part; q < nzp; q += 4)
        hz[q * 8 + h8] = q < NZ ? pc_angular(T0.Z[T0.order[q]].c, T0.Z[T0.order[q]].sidx, E, h8) : mk(0, 0);
    }
    __syncwarp();
    bool fail = vb_overflow;
    // one round of centre rows: R[b][q] at lookup l0 + b, S0[b][h]; the centre's smeared sums
    auto centre_round = [&](int l0, bool sums) {
      const int l = l0 + lane;
      cplx* row = R + lane * rs;  // rows past RC are past nlook too and are never read
      if (lane < RC) {
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
      }
      __syncwarp();
      if (lane < RC) {
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          cplx s = mk(0, 0);
          for (int q = 0; q < NZ; ++q) cmac(s, row[q], hz[q * 8 + h]);
          S0[lane * 9 + h] = s;
        }
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
        // moments of the rows for the coupling points: G over the entry pairs (lane per pair), R1,
        // and the row at the event mass
        const int npair = MOMENTS ? NZ * (NZ + 1) / 2 : 0;
        for (int t = lane; t < npair; t += 32) {
          int qa = 0, rem = t;
          while (rem >= NZ - qa) {
            rem -= NZ - qa;
            ++qa;
          }
          const int qb = qa + rem;
          cplx g = mk(0, 0);
          for (int b = 0; b < 32; ++b) {
            const int ll = l0 + b;
            if (ll < shift || ll >= nlook) continue;
            cmac(g, row_weight(ll) * conj(R[b * rs + qa]), R[b * rs + qb]);
          }
          G[t] = (l0 == 0 ? mk(0, 0) : G[t]) + g;
        }
        for (int q = lane; MOMENTS && q < NZ; q += 32) {
          cplx r1 = mk(0, 0);
          for (int b = 0; b < 32; ++b) {
            const int ll = l0 + b;
            if (ll < shift || ll >= nlook) continue;
            r1 += row_weight(ll) * R[b * rs + q];
          }
          R1[q] = (l0 == 0 ? mk(0, 0) : R1[q]) + r1;
          if (l0 == 0 && shift) R0[q] = R[q];
        }
        if (l0 == 0 && shift && lane < 8) s00[lane] = S0[lane];
        __syncwarp();
      }
    };
    auto gram = [&](int qa, int qb) {
      const cplx g = G[gtri(min(qa, qb), max(qa, qb), NZ)];
      return mk(g.re, qa <= qb ? g.im : -g.im);
    };
    // the centre's sums over all offset rows first; with several rounds the rows are recomputed
    // below only in passes whose points read them
    for (int rd = 0; rd < nrounds; ++rd) centre_round(rd * 32, true);
    // P_qh = sum_q' conj(HZ_q'h) G(q', q); Y_q = sum_h conj(H_L[h]) HZ_qh
    for (int t = lane; MOMENTS && t < NZ * 8; t += 32) {
      const int q = t >> 3, h = t & 7;
      cplx pv = mk(0, 0);
      for (int q2 = 0; q2 < NZ; ++q2) cmac(pv, conj(hz[q2 * 8 + h]), gram(q2, q));
      P[t] = pv;
    }
    for (int q = lane; MOMENTS && q < NZ; q += 32) {
      cplx y = mk(0, 0);
#pragma unroll
      for (int h = 0; h < 8; ++h) cmac(y, conj(hl0[h]), hz[q * 8 + h]);
      Y[q] = y;
    }
    __syncwarp();
    double a20s = 0, n00 = 0;  // sum_h a20[h]; sum_h |S0_0h|^2
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      a20s += a20[h];
      if (shift) n00 += norm2(s00[h]);
    }
    const bool centre_fail = !FIX && __any_sync(0xffffffffu, fail);
    const float wfe = E.w();
    const bool data_w = wfe <= -1000.f;
    auto accumulate = [&](int pi, double v, double vn) {
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
    };
    bool dead = centre_fail, decided = FIX;  // warp-uniform
    auto decide = [&]() {
      dead = dead || __any_sync(0xffffffffu, fail);
      decided = true;
      if (!dead)
        for (int pi = lane; pi < min(pcg_end, npts); pi += 32) accumulate(pi, vbuf[pi * 2], vbuf[pi * 2 + 1]);
    };
    if (!centre_fail) {
      for (int pass = 0; pass < npts; pass += 32) {
        if (!decided && pass >= pcg_end) {
          decide();
          if (dead) break;
        }
        const int pidx = pass + lane;
        const bool act = pidx < npts;
        const BatchPoint& bp = pts[act ? pidx : 0];
        const int kind = act ? bp.kind : BP_SAME;
        const bool own = kind == BP_PCC || kind == BP_PCG;  // sums over the rows are the point's own
        if constexpr (MOMENTS) {
          // own points (coupling and lineshape points): dy = sum_h conj(H_L[h]) (a1[h] - a10[h]) and
          // s2 = sum_h a2[h], their smeared sums
          double dy = 0, s2 = a20s;
          double vns = 0;  // sum_h |S_0[h]|^2 at the event mass (non-interfering term, smeared band 0)
          if (kind == BP_PCC) {
            // from the centre's row moments: S_bh + sum_u R_b,q(u) d_uh summed over the rows gives
            // a1 = a10 + sum_u d_u R1_q(u) and a2 = a20 + 2 Re sum_u d_u P_q(u) + sum_uu' conj(d_u) d_u' G
            const int nq = bp.nq;
            int pos[BATCH_MAXQ_PC];
  #pragma unroll
            for (int u = 0; u < BATCH_MAXQ_PC; ++u) {
              if (u >= nq) break;
              pos[u] = bp.qpos[u];
            }
            double lin = 0, quad = 0;
            // one helicity at a time keeps this code small (the kernel is instruction-cache sensitive);
            // the angular sums take every coupling slot without a branch, so their loads issue together
  #pragma unroll 1
            for (int h = 0; h < 8; ++h) {
              const int i = h >> 2, j = (h >> 1) & 1, k = h & 1;
              cplx d[BATCH_MAXQ_PC];
              const cplx hc = conj(hl0[h]);
              cplx sv = s00[h];
  #pragma unroll
              for (int u = 0; u < BATCH_MAXQ_PC; ++u) {
                if (u >= nq) break;
                const cplx* cu = bp.dc + u * 24 + k * 12;
                const int sx = bp.qsidx[u];
                cplx du = mk(0, 0);
  #pragma unroll
                for (int m = 0; m < 12; ++m) cmac(du, cu[m], E.AZ(i, j, m) * E.DZ(sx, k, m));
                d[u] = du;
                const cplx hr = hc * R1[pos[u]];
                const cplx pr = P[pos[u] * 8 + h];
                dy += hr.re * du.re - hr.im * du.im;
                lin += 2.0 * (pr.re * du.re - pr.im * du.im);
                if (shift) cmac(sv, R0[pos[u]], du);
              }
  #pragma unroll
              for (int u = 0; u < BATCH_MAXQ_PC; ++u) {
                if (u >= nq) break;
                cplx gd = mk(0, 0);
  #pragma unroll
                for (int u2 = 0; u2 < BATCH_MAXQ_PC; ++u2) {
                  if (u2 >= nq) break;
                  cmac(gd, gram(pos[u], pos[u2]), d[u2]);
                }
                quad += d[u].re * gd.re + d[u].im * gd.im;  // Re(conj(d_u) (G d)_u)
              }
              if (shift) vns += norm2(sv);
            }
            s2 = a20s + lin + quad;
          }
          const bool need_rows = __any_sync(0xffffffffu, kind == BP_PCG);
          if (kind == BP_PCG) s2 = 0;
          for (int rd = 0; need_rows && rd < nrounds; ++rd) {
            const int l0 = rd * 32;
            if (nrounds > 1) centre_round(l0, false);
            const int rows = min(32, nlook - l0);
            if (kind == BP_PCG) {
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
                cplx y = mk(0, 0);
  #pragma unroll
                for (int q = 0; q < MAX_GROUP_ENTRIES; ++q)
                  if (q < cnt) {
                    dr[q] -= R[b * rs + first + q];
                    cmac(y, dr[q], Y[first + q]);
                  } else {
                    break;
                  }
                double t = 0;  // sum_h |S_bh + sum_q dR_bq HZ_qh|^2
  #pragma unroll
                for (int h = 0; h < 8; ++h) {
                  cplx sv = S0[b * 9 + h];
  #pragma unroll
                  for (int q = 0; q < MAX_GROUP_ENTRIES; ++q)
                    if (q < cnt) cmac(sv, dr[q], hz[(first + q) * 8 + h]);
                    else break;
                  t += norm2(sv);
                }
                if (l < shift) {
                  vns += t;
                } else {
                  const double wb = row_weight(l);
                  dy += wb * y.re;
                  s2 += wb * t;
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
                  const cplx qp = lstar_lineshape(Tp, r, lk);
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
            if (!own) vns = n00;
            double v = c2 * s2 + 2.0 * wgt * dy, vn = vns;
  #pragma unroll
            for (int h = 0; h < 8; ++h) {
              v += norm2(hlp[h]) + 2.0 * wgt * (hlp[h].re * a10[h].re + hlp[h].im * a10[h].im);
              vn += has_x ? norm2(hlp[h] - hx0[h]) + norm2(hx0[h]) : norm2(hlp[h]);
            }
            if (decided) {
              accumulate(pidx, v, vn);
            } else {
              vbuf[pidx * 2] = v;
              vbuf[pidx * 2 + 1] = vn;
            }
          }
        } else {
          // per-helicity sums over the offset rows for every own point
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
                cplx d[BATCH_MAXQ_PC];
                int pos[BATCH_MAXQ_PC];
  #pragma unroll
                for (int u = 0; u < BATCH_MAXQ_PC; ++u) {
                  if (u >= nq) break;
                  pos[u] = bp.qpos[u];
                  d[u] = pc_angular(bp.dc + u * 24, bp.qsidx[u], E, h);
                }
                for (int b = 0; b < rows; ++b) {
                  cplx sv = S0[b * 9 + h];
  #pragma unroll
                  for (int u = 0; u < BATCH_MAXQ_PC; ++u) {
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
                  const cplx qp = lstar_lineshape(Tp, r, lk);
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
            if (!own) vns = n00;
            double v = 0, vn = vns;
  #pragma unroll
            for (int h = 0; h < 8; ++h) {
              const cplx s1 = own ? a1[h] : a10[h];
              const double s2 = own ? a2[h] : a20[h];
              v += norm2(hlp[h]) + 2.0 * wgt * (hlp[h].re * s1.re + hlp[h].im * s1.im) + c2 * s2;
              vn += has_x ? norm2(hlp[h] - hx0[h]) + norm2(hx0[h]) : norm2(hlp[h]);
            }
            if (decided) {
              accumulate(pidx, v, vn);
            } else {
              vbuf[pidx * 2] = v;
              vbuf[pidx * 2 + 1] = vn;
            }
          }
        }
      }
    }
    if (!decided) decide();
    if (dead && lane == 0) defer[atomicAdd(defer_count, 1)] = (int32_t)e;
    __syncwarp();
  }
  __syncthreads();
  for (int pi = threadIdx.x; pi < npts; pi += BATCH_THREADS) {
    const double* a = acc + pi * 4;
    parts[(size_t)blockIdx.x * npts + pi] = Partial{a[0], a[1], a[2], a[3]};
  }
}


// Host wrappers of k_batch for one offset scheme (suffix: 20, 30, 150 quantile offsets; grid = the
// weighted grid), defined in that scheme's translation unit.
#define PWA_BATCH_WRAPPERS(sfx)                                                                             \
  cudaError_t batch_set_smem_##sfx(int optin);                                                              \
  int batch_occupancy_##sfx(size_t smem);                                                                   \
  void batch_launch_##sfx(const EventSet& ev, int64_t begin, int64_t end, const int32_t* list, const int* n_list, \
                          const PointTable* d_T0, const BatchPoint* d_pts, int npts, Partial* out, int band,      \
                          int32_t* defer, int* defer_count, bool fix, int grid, size_t smem, cudaStream_t st,     \
                          const double* sgrid, int sgrid_nb);
PWA_BATCH_WRAPPERS(20)
PWA_BATCH_WRAPPERS(30)
PWA_BATCH_WRAPPERS(150)
PWA_BATCH_WRAPPERS(grid)
#undef PWA_BATCH_WRAPPERS

}  // namespace pwa
