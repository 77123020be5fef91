// Likelihood kernels for sm_100a, FP64 arithmetic on the reference's float SoA basis.
//
// Work split (reference: src/kernel_calEva.cu:819-976):
//   * unsmeared events: one thread per event (persistent grid-stride loop); lineshapes at the
//     event's m(J/psi p), Lambda* and Pc helicity sums, |A|^2 with and without interference.
//   * smeared events (30 / 150 / 20 resolution offsets): a block takes a tile of 32 events.  Phase 1
//     builds the Lambda* amplitudes and the per-entry Pc angular amplitudes HZ_i[h] (couplings
//     included, lineshape excluded) in shared memory; phase 2 spreads the (event, offset) pairs over
//     8 lanes per event, each evaluating all Pc lineshapes (K-matrix solves) at its offsets and
//     accumulating S = sum_i BW_i HZ_i; phase 3 combines
//       |A|^2 = sum_h |H_L|^2 + 2 w Re(conj(H_L) sum_b S_b) + w^2 u sum_b |S_b|^2,
//     which is the reference's BW1/BW2 form (kernel_calEva.cu:676-810) with its float weight
//     w = float(1/NBINS) and rescale u = float(1/w).
//   * every block writes FP64 partial sums (data sw ln fx, MC w fx, MC w fx without
//     interference); one finalize block reduces them with compensated summation.
#include <cstdio>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "pwa_kernels.cuh"

namespace pwa {

// Resolution offsets in units of the mass resolution (reference data, Resonances.h:31-54).
#include "smear_tables.inc"

#ifndef PWA_SMEAR_MIN_BLOCKS
#define PWA_SMEAR_MIN_BLOCKS 2
#endif
#ifndef PWA_UNSMEARED_MIN_BLOCKS
#define PWA_UNSMEARED_MIN_BLOCKS 4
#endif

constexpr int TILE = 32;          // events per smeared tile
constexpr int SMEAR_THREADS = 256;
constexpr int LANES_PER_EVENT = SMEAR_THREADS / TILE;  // 8
constexpr int UNSMEARED_THREADS = 128;
constexpr int MAX_GROUP_ENTRIES = 8;

__device__ __forceinline__ double ldf(const float* p, int64_t i) { return (double)__ldg(p + i); }

// ------------------------------------------------------------------------------- lineshapes
// Quantities of one event mass that every lineshape at that mass shares: two-body momenta and
// 1/sqrt of the Blatt-Weisskopf polynomials for each barrier order L in use.  Each resonance then
// costs one division (its Breit-Wigner denominator) and no square root.
struct LstarKin {
  double mkp, inv_mkp, s, pR, pSP, pBm;
  double rsR[6], rsB[6];
};
struct PcKin {
  double mz, inv_mz, s, pR, pBm;
  double rsR[6], rsB[6];
};

__host__ __device__ inline void fill_rs(double* rs, int mask, double r, double p) {
  const double z = sq(r * p);
#pragma unroll
  for (int L = 1; L <= 5; ++L) rs[L] = (mask >> L & 1) ? 1.0 / sqrt(bw_poly(L, z)) : 1.0;
  rs[0] = 1.0;
}

__host__ __device__ inline LstarKin lstar_kin(const PointTable& T, double mkp) {
  LstarKin k;
  k.mkp = mkp;
  k.inv_mkp = 1.0 / mkp;
  k.s = mkp * mkp;
  k.pR = two_body_p(mkp, M_P, M_K);
  k.pSP = T.needs_sigma_pi ? two_body_p(mkp, PWA_F(1.18937f), PWA_F(0.13957018f)) : 0.0;
  const double pB = two_body_p(M_LB, M_JPSI, mkp);
  k.pBm = pB / M_LB;
  fill_rs(k.rsR, T.lmask_lstar_R, T.ffr, k.pR);
  fill_rs(k.rsB, T.lmask_lstar_B, T.ffb, pB);
  return k;
}

__host__ __device__ inline PcKin pc_kin(const PointTable& T, double mz) {
  PcKin k;
  k.mz = mz;
  k.inv_mz = 1.0 / mz;
  k.s = mz * mz;
  k.pR = two_body_p(mz, M_P, M_JPSI);
  const double pB = two_body_p(M_LB, M_K, mz);
  k.pBm = pB / M_LB;
  fill_rs(k.rsR, T.lmask_pc_R, T.ffr, k.pR);
  fill_rs(k.rsB, T.lmask_pc_B, T.ffb, pB);
  return k;
}

// Lambda* Breit-Wigner times the Lambda_b -> Lambda* J/psi barrier (BW_AMP, cu_DPFPropogator.cu:248-314;
// BTerm :155-181) with the parameter-only constants of the point table.
__host__ __device__ inline cplx lstar_lineshape(const LstarEntry& L, const LstarKin& k) {
  cplx bw = mk(1, 0);
  if (L.type == LT_BW) {
    if (L.branch == 2) {
      bw = mk(ipow(k.pR * L.inv_pR0, L.LR), 0);
    } else if (L.branch == 4) {
      bw = mk(0, 0);
    } else {
      double FR = 1.0, gamma = L.g_r, ratio;
      if (L.branch == 0) {
        FR = L.sqrt_polyR0 * k.rsR[L.LR];
        ratio = k.pR * L.inv_pR0;
        gamma = L.g_r * ipow(ratio, 2 * L.LR + 1) * (L.m_r * k.inv_mkp) * FR * FR;
      } else if (L.branch == 1) {
        ratio = k.pR * L.inv_pR0_sp;
        gamma = L.g_r * ipow(ratio, 2 * L.LR + 1) * (L.m_r * k.inv_mkp);
        gamma += PWA_F(0.0505f) * ipow(k.pSP * L.inv_pR0_sp, 2 * L.LR + 1) * (L.m_r * k.inv_mkp);
      } else {  // branch 3: m_r in [1.43, pK threshold]
        FR = L.sqrt_polyR0 * k.rsR[L.LR];
        ratio = k.pR * L.inv_pR0;
      }
      const double factor = FR * ipow(ratio, L.LR) * L.norm;
      const double de2 = L.m_r * L.m_r - k.s, gm = gamma * L.m_r;
      const double f = factor / (de2 * de2 + gm * gm);
      bw = mk(de2 * f, gm * f);
    }
  }
  const double bt = (L.LB ? L.sqrt_polyB0 * k.rsB[L.LB] : 1.0) * ipow(k.pBm, L.LB) * L.lb_scale;
  return bw * bt;
}

// Lambda_b -> Pc K barrier (BTermZ, cu_DPFPropogator.cu:183-203).
__host__ __device__ inline double pc_barrier(const PcEntry& Z, const PcKin& k) {
  const double F = (Z.pB0_event || Z.LB == 0) ? 1.0 : Z.sqrt_polyB0 * k.rsB[Z.LB];
  return F * ipow(k.pBm, Z.LB);
}

// Pc Breit-Wigner (BW_AMPZ, cu_DPFPropogator.cu:316-336).
__host__ __device__ inline cplx pc_bw(const PcEntry& Z, const PcKin& k) {
  double FR = 1.0, gamma = Z.g_r, ratio = 1.0;
  if (Z.bw_above) {
    FR = Z.sqrt_polyR0 * k.rsR[Z.LR];
    ratio = k.pR * Z.inv_pR0;
    gamma = Z.g_r * ipow(ratio, 2 * Z.LR + 1) * (Z.m_r * k.inv_mz) * FR * FR;
  }
  const double factor = FR * ipow(ratio, Z.LR) * Z.norm;
  const double de2 = Z.m_r * Z.m_r - k.s, gm = gamma * Z.m_r;
  const double f = factor / (de2 * de2 + gm * gm);
  return mk(de2 * f, gm * f);
}

// One J^P group of the coupled-channel K-matrix at mass mz (Default_KMatrix,
// cu_DPFPropogator.cu:588-813): P-vector outputs, npole poles first then 4 production terms.
__host__ __device__ inline void km_solve(const KmGroup& G, double mz, double ffb, cplx* out) {
  const double s = mz * mz;
  cplx rho[NKMC];
  rho[0] = rho_real(s, M_P, M_JPSI, G.Lna, ffb);
  if (G.P == -1) {
    const cplx dst = mk(KM_DST, 0), d = mk(KM_D, 0), sc = mk(KM_SC, KM_SC_HW), scst = mk(KM_SCST, KM_SCST_HW);
    rho[1] = rho_complex(s, dst, sc);
    if (G.J2 == 1) {
      rho[2] = rho_complex(s, dst, scst);
      rho[3] = rho_complex(s, d, sc);
    } else {
      rho[2] = rho_complex(s, dst, scst);
      rho[3] = rho_complex(s, d, scst);
    }
  } else {
    rho[1] = rho_real(s, KM_DST, KM_SC, G.Lna, ffb);
    rho[2] = rho_real(s, KM_D, KM_SC, G.Lna, ffb);
    rho[3] = rho_real(s, KM_D, KM_SCST, G.Lna, ffb);
  }
  double ms[NPMAX + 1] = {1, 1, 1, 1, 1};
  for (int p = 0; p < G.npole; ++p) {
    double den = G.m0sq[p] - s;
    if (fabs(den) < KM_DENORM_MIN) den = KM_DENORM_MIN;
    ms[0] *= den;
#pragma unroll
    for (int ip = 1; ip <= NPMAX; ++ip)
      if (ip != p + 1) ms[ip] *= den;
  }
  double mg[NPMAX][NKMC];
  for (int p = 0; p < G.npole; ++p)
#pragma unroll
    for (int j = 0; j < NKMC; ++j) mg[p][j] = G.g[p][j] * ms[p + 1];
  double kma[NKMC][NKMC];
#pragma unroll
  for (int i = 0; i < NKMC; ++i)
#pragma unroll
    for (int j = 0; j < NKMC; ++j) {
      if (j < i) continue;
      double v = G.f[i][j] * ms[0];
      for (int p = 0; p < G.npole; ++p) v += G.g[p][i] * mg[p][j];
      kma[i][j] = v;
      kma[j][i] = v;
    }
  cplx S[4][4];
#pragma unroll
  for (int i = 0; i < NKMC; ++i)
#pragma unroll
    for (int j = 0; j < NKMC; ++j) {
      // -i * (K * rho) + ms0 on the diagonal
      S[i][j] = mk(kma[i][j] * rho[j].im, -kma[i][j] * rho[j].re);
      if (i == j) S[i][j].re += ms[0];
    }
  cplx T[4];
  first_row_inverse4(S, T);
  const double na = (G.Lna >= 1) ? channel_barrier(s, M_P, M_JPSI, G.Lna, ffb) : 1.0;
  for (int p = 0; p < G.npole; ++p) {
    cplx acc = mk(0, 0);
#pragma unroll
    for (int i = 0; i < NKMC; ++i) acc += T[i] * mg[p][i];
    out[p] = acc * na;
  }
#pragma unroll
  for (int i = 0; i < NKMC; ++i) out[G.npole + i] = T[i] * (ms[0] * na);
}

// K-matrix outputs of group ik at mz from the per-point table (6-point Lagrange on the uniform grid);
// false when mz is in a guard interval or too close to the grid ends.
__device__ __forceinline__ bool table_lookup(const LineTables& tab, int ik, int nout, double mz, cplx* out) {
  if (!tab.enabled) return false;
  const double x = (mz - tab.m_lo) * tab.inv_h;
  const double fj = floor(x);
  if (!(fj >= 2.0 && fj + 3.0 < (double)tab.n_nodes)) return false;
  const int j = (int)fj;
  if (tab.bad[ik][j]) return false;
  const double t = x - fj;
  // Lagrange weights for nodes j-2 .. j+3 (denominators -120, 24, -12, 12, -24, 120)
  const double d0 = t + 2.0, d1 = t + 1.0, d2 = t, d3 = t - 1.0, d4 = t - 2.0, d5 = t - 3.0;
  const double p01 = d0 * d1, p012 = p01 * d2, p0123 = p012 * d3, p01234 = p0123 * d4;
  const double s5 = d5, s45 = d4 * s5, s345 = d3 * s45, s2345 = d2 * s345, s12345 = d1 * s2345;
  const double w[6] = {s12345 * (-1.0 / 120.0), d0 * s2345 * (1.0 / 24.0), p01 * s345 * (-1.0 / 12.0),
                       p012 * s45 * (1.0 / 12.0), p0123 * s5 * (-1.0 / 24.0), p01234 * (1.0 / 120.0)};
  const cplx* base = tab.data[ik] + (size_t)(j - 2) * TAB_SLOTS;
  for (int o = 0; o < nout; ++o) {
    cplx acc = mk(0, 0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const cplx v = base[k * TAB_SLOTS + o];
      acc.re = fma(w[k], v.re, acc.re);
      acc.im = fma(w[k], v.im, acc.im);
    }
    out[o] = acc;
  }
  return true;
}

// Exact solve for lookups the table cannot serve; kept out of line so that the rarely taken path
// does not set the register budget of the event kernels.
__device__ __noinline__ void km_solve_fallback(const KmGroup& G, double mz, double ffb, cplx* out) {
  km_solve(G, mz, ffb, out);
}

// Lineshape (with production barrier) of every entry of Pc group g at the mass of `k`.
__device__ __forceinline__ void pc_group_lineshapes(const PointTable& T, int g, const PcKin& k, cplx* raw) {
  const PcGroup& gr = T.grp[g];
  cplx kmo[NPMAX + NKMC];
  if (gr.km >= 0) {
    const KmGroup& G = T.G[gr.km];
    if (!table_lookup(T.tab, gr.km, G.npole + NKMC, k.mz, kmo)) km_solve_fallback(G, k.mz, T.ffb, kmo);
  }
  for (int q = 0; q < gr.count; ++q) {
    const PcEntry& Z = T.Z[T.order[gr.first + q]];
    cplx v;
    if (Z.type == LT_KM)
      v = kmo[Z.slot];
    else if (Z.type == LT_BW)
      v = pc_bw(Z, k);
    else
      v = mk(1, 0);
    raw[q] = v * pc_barrier(Z, k);
  }
}

// ------------------------------------------------------------------------------- SoA access
struct Ev {
  const float *pp, *pp1, *pp2;
  int64_t ns, e;
  __device__ __forceinline__ double mkp() const { return ldf(pp, e); }
  __device__ __forceinline__ double mz() const { return ldf(pp, e + ns); }
  __device__ __forceinline__ float w() const { return __ldg(pp + e + 2 * ns); }
  __device__ __forceinline__ cplx A(int i, int j, int m) const {
    const int a = 3 + (i * 12 + j * 6 + m) * 2;
    return mk(ldf(pp, e + a * ns), ldf(pp, e + (a + 1) * ns));
  }
  __device__ __forceinline__ double DL(int s, int k, int m) const { return ldf(pp, e + (51 + s * 12 + k * 6 + m) * ns); }
  __device__ __forceinline__ cplx AZ(int i, int j, int m) const {
    const int a = (i * 24 + j * 12 + m) * 2;
    return mk(ldf(pp1, e + a * ns), ldf(pp1, e + (a + 1) * ns));
  }
  __device__ __forceinline__ double DZ(int s, int k, int m) const { return ldf(pp2, e + (s * 24 + k * 12 + m) * ns); }
};

// Lambda* helicity amplitudes H[4*dmu + 2*lb + p] (GetAmpLz, kernel_calEva.cu:85-190).
__device__ __forceinline__ void lstar_amplitudes(const PointTable& T, const Ev& ev, double mkp, cplx (&H)[8]) {
  const LstarKin kin = lstar_kin(T, mkp);
  for (int r = 0; r < T.NR; ++r) {
    const LstarEntry& L = T.L[r];
    const cplx q = lstar_lineshape(L, kin);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      for (int m = 0; m < L.ncm; ++m) {
        const cplx c = L.c[k * 6 + m];
        if (c.re == 0.0 && c.im == 0.0) continue;
        const cplx D = (q * c) * ev.DL(L.sidx, k, m);
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) cmac(H[4 * i + 2 * j + k], ev.A(i, j, m), D);
      }
    }
  }
}

// Pc helicity amplitudes at the event's own mass (unsmeared; GetAmp2s :347-503).
__device__ __forceinline__ void pc_amplitudes(const PointTable& T, const Ev& ev, double mz, cplx (&H)[8]) {
  const PcKin kin = pc_kin(T, mz);
  for (int g = 0; g < T.ngroups; ++g) {
    const PcGroup& gr = T.grp[g];
    cplx raw[MAX_GROUP_ENTRIES];
    pc_group_lineshapes(T, g, kin, raw);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      cplx E[12];
#pragma unroll
      for (int m = 0; m < 12; ++m) E[m] = mk(0, 0);
      for (int q = 0; q < gr.count; ++q) {
        const PcEntry& Z = T.Z[T.order[gr.first + q]];
#pragma unroll
        for (int m = 0; m < 12; ++m) cmac(E[m], raw[q], Z.c[k * 12 + m]);
      }
#pragma unroll
      for (int m = 0; m < 12; ++m) {
        if (E[m].re == 0.0 && E[m].im == 0.0) continue;
        const cplx D = E[m] * ev.DZ(gr.sidx, k, m);
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) cmac(H[4 * i + 2 * j + k], ev.AZ(i, j, m), D);
      }
    }
  }
}

// ------------------------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int NT>
__device__ void block_reduce_store(double a, double b, double c, double d, Partial* out) {
  __shared__ double red[4][NT / 32];
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  d = warp_sum(d);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) {
    red[0][w] = a;
    red[1][w] = b;
    red[2][w] = c;
    red[3][w] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Partial p{0, 0, 0, 0};
    for (int i = 0; i < NT / 32; ++i) {
      p.data += red[0][i];
      p.mc += red[1][i];
      p.mc_noint += red[2][i];
      p.n_nonpos += red[3][i];
    }
    out[blockIdx.x] = p;
  }
}

template <int NT>
__device__ __forceinline__ void load_table(const PointTable* g, PointTable* s) {
  const int4* src = reinterpret_cast<const int4*>(g);
  int4* dst = reinterpret_cast<int4*>(s);
  constexpr int n = sizeof(PointTable) / sizeof(int4);
  for (int i = threadIdx.x; i < n; i += NT) dst[i] = src[i];
  __syncthreads();
}

// Per-event likelihood contributions (kernel_calEva.cu:894-917, :964-976, :1296-1321).
struct Acc {
  double data = 0, mc = 0, mcn = 0, bad = 0;
  __device__ __forceinline__ void add(int64_t e, int64_t nda, const float* sw, double fxe, double vn_w, bool band) {
    if (!(fxe > 0) || !isfinite(fxe)) bad += 1;
    if (e < nda) {
      data += (fxe > 0) ? log(fxe) * (double)__ldg(sw + e) : -1e12;
    } else {
      mc += fxe;
      if (!band) mcn += vn_w;
    }
  }
};

// ------------------------------------------------------------------------------- unsmeared
__global__ void __launch_bounds__(UNSMEARED_THREADS, PWA_UNSMEARED_MIN_BLOCKS)
    k_unsmeared(EventSet ev, int64_t nda, int64_t begin, int64_t end, const int32_t* list,
                const PointTable* __restrict__ gtab, Partial* parts, double* fx_out, int amp2_only) {
  __shared__ __align__(16) PointTable T;
  load_table<UNSMEARED_THREADS>(gtab, &T);
  Acc acc;
  const int64_t count = end - begin;
  for (int64_t p = (int64_t)blockIdx.x * UNSMEARED_THREADS + threadIdx.x; p < count;
       p += (int64_t)gridDim.x * UNSMEARED_THREADS) {
    const int64_t e = list ? (int64_t)list[begin + p] : begin + p;
    Ev E{ev.pp, ev.pp1, ev.pp2, ev.n_size, e};
    cplx HL[8], HZ[8];
#pragma unroll
    for (int h = 0; h < 8; ++h) HL[h] = HZ[h] = mk(0, 0);
    const double mkp = E.mkp(), mz = E.mz();
    lstar_amplitudes(T, E, mkp, HL);
    pc_amplitudes(T, E, mz, HZ);
    double v = 0, vn = 0;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      v += norm2(HL[h] + HZ[h]);
      vn += norm2(HL[h]) + norm2(HZ[h]);
    }
    if (amp2_only) {
      fx_out[e] = v;
      continue;
    }
    const float wf = E.w();
    const bool is_data_w = wf <= -1000.f;
    const double w = wf;
    const double fxe = is_data_w ? v : v * w;
    if (fx_out) fx_out[e] = fxe;
    acc.add(e, nda, ev.sw, fxe, is_data_w ? 0.0 : vn * w, false);
  }
  if (!amp2_only) block_reduce_store<UNSMEARED_THREADS>(acc.data, acc.mc, acc.mcn, acc.bad, parts);
}

// ------------------------------------------------------------------------------- smeared
struct SmearShared {
  PointTable T;
  cplx Q[MAX_LSTAR][TILE];    // Lambda* lineshapes per event
  double HZre[MAX_PC][8][TILE], HZim[MAX_PC][8][TILE];
  double HLre[8][TILE], HLim[8][TILE];
  double A1re[8][TILE], A1im[8][TILE], A2[8][TILE], VN[TILE];
  int64_t ev[TILE];
};

template <int NB>
__device__ __forceinline__ const float* smear_table();
template <>
__device__ __forceinline__ const float* smear_table<20>() { return kSmear20; }
template <>
__device__ __forceinline__ const float* smear_table<30>() { return kSmear30; }
template <>
__device__ __forceinline__ const float* smear_table<150>() { return kSmear150; }

template <int NB>
__global__ void __launch_bounds__(SMEAR_THREADS, PWA_SMEAR_MIN_BLOCKS)
    k_smeared(EventSet ev, int64_t nda, int64_t begin, int64_t end, const int32_t* list,
              const PointTable* __restrict__ gtab, Partial* parts, double* fx_out, int band) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmearShared& S = *reinterpret_cast<SmearShared*>(smem_raw);
  load_table<SMEAR_THREADS>(gtab, &S.T);
  const PointTable& T = S.T;
  const float* qoff = smear_table<NB>();
  // float weight 1/NBINS and its float reciprocal, as the reference (kernel_calEva.cu:676,771)
  const float wf = (float)(1.0 / NB);
  const double wgt = wf;
  const double c2 = wgt * wgt * (double)(1.0f / wf);
  const int tid = threadIdx.x;
  const int64_t count = end - begin;
  const int64_t ntiles = (count + TILE - 1) / TILE;
  Acc acc;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // event indices of this tile
    if (tid < TILE) {
      const int64_t p = tile * TILE + tid;
      S.ev[tid] = (p < count) ? (list ? (int64_t)list[begin + p] : begin + p) : -1;
    }
    __syncthreads();
    // phase 1a: Lambda* lineshapes per (resonance, event)
    for (int t = tid; t < T.NR * TILE; t += SMEAR_THREADS) {
      const int r = t / TILE, el = t % TILE;
      const int64_t e = S.ev[el];
      S.Q[r][el] = (e >= 0) ? lstar_lineshape(T.L[r], lstar_kin(T, ldf(ev.pp, e))) : mk(0, 0);
    }
    __syncthreads();
    // phase 1b/1c: helicity amplitudes; thread -> (event el, helicity h)
    {
      const int el = tid % TILE, h = tid / TILE;
      const int i = h >> 2, j = (h >> 1) & 1, k = h & 1;
      const int64_t e = S.ev[el];
      cplx hl = mk(0, 0);
      if (e >= 0) {
        Ev E{ev.pp, ev.pp1, ev.pp2, ev.n_size, e};
        for (int r = 0; r < T.NR; ++r) {
          const LstarEntry& L = T.L[r];
          const cplx q = S.Q[r][el];
          for (int m = 0; m < L.ncm; ++m) {
            const cplx c = L.c[k * 6 + m];
            if (c.re == 0.0 && c.im == 0.0) continue;
            cmac(hl, E.A(i, j, m), (q * c) * E.DL(L.sidx, k, m));
          }
        }
        cplx az[12];
#pragma unroll
        for (int m = 0; m < 12; ++m) az[m] = E.AZ(i, j, m);
        for (int q = 0; q < T.NZ; ++q) {
          const int zi = T.order[q];
          const PcEntry& Z = T.Z[zi];
          cplx hz = mk(0, 0);
#pragma unroll
          for (int m = 0; m < 12; ++m) {
            const cplx c = Z.c[k * 12 + m];
            if (c.re == 0.0 && c.im == 0.0) continue;
            cmac(hz, az[m], c * E.DZ(Z.sidx, k, m));
          }
          S.HZre[q][h][el] = hz.re;
          S.HZim[q][h][el] = hz.im;
        }
      } else {
        for (int q = 0; q < T.NZ; ++q) S.HZre[q][h][el] = S.HZim[q][h][el] = 0.0;
      }
      S.HLre[h][el] = hl.re;
      S.HLim[h][el] = hl.im;
    }
    __syncthreads();
    // phase 2: offsets; thread -> (event el, lane b0), bins b0, b0+8, ...
    {
      const int el = tid / LANES_PER_EVENT, b0 = tid % LANES_PER_EVENT;
      const int64_t e = S.ev[el];
      cplx a1[8];
      double a2[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        a1[h] = mk(0, 0);
        a2[h] = 0;
      }
      double vn = 0;
      if (e >= 0) {
        const double mz = ldf(ev.pp, e + ev.n_size);
        const double mres = MRES0 + mz * (MRES1 + mz * MRES2);
        const bool need_noint = (band == 0) && (e >= nda) && !(__ldg(ev.pp + e + 2 * ev.n_size) <= -1000.f);
        // b == -1 is the unsmeared evaluation for the MC non-interference sum
        for (int b = (need_noint && b0 == 0) ? -1 : b0; b < NB; b += (b < 0) ? (1 + b0) : LANES_PER_EVENT) {
          const double m = (b < 0) ? mz : mz + (double)qoff[b] * mres;
          const PcKin kin = pc_kin(T, m);
          cplx s8[8];
#pragma unroll
          for (int h = 0; h < 8; ++h) s8[h] = mk(0, 0);
          for (int g = 0; g < T.ngroups; ++g) {
            cplx raw[MAX_GROUP_ENTRIES];
            pc_group_lineshapes(T, g, kin, raw);
            const PcGroup& gr = T.grp[g];
            for (int q = 0; q < gr.count; ++q) {
              const int qq = gr.first + q;
#pragma unroll
              for (int h = 0; h < 8; ++h) cmac(s8[h], raw[q], mk(S.HZre[qq][h][el], S.HZim[qq][h][el]));
            }
          }
          if (b < 0) {
#pragma unroll
            for (int h = 0; h < 8; ++h) vn += norm2(mk(S.HLre[h][el], S.HLim[h][el])) + norm2(s8[h]);
          } else {
#pragma unroll
            for (int h = 0; h < 8; ++h) {
              a1[h] += s8[h];
              a2[h] += norm2(s8[h]);
            }
          }
        }
      }
      // reduce over the 8 lanes of this event (they are adjacent lanes of one warp)
#pragma unroll
      for (int o = 1; o < LANES_PER_EVENT; o <<= 1) {
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          a1[h].re += __shfl_xor_sync(0xffffffffu, a1[h].re, o);
          a1[h].im += __shfl_xor_sync(0xffffffffu, a1[h].im, o);
          a2[h] += __shfl_xor_sync(0xffffffffu, a2[h], o);
        }
        vn += __shfl_xor_sync(0xffffffffu, vn, o);
      }
      if (b0 == 0) {
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          S.A1re[h][el] = a1[h].re;
          S.A1im[h][el] = a1[h].im;
          S.A2[h][el] = a2[h];
        }
        S.VN[el] = vn;
      }
    }
    __syncthreads();
    // phase 3: combine per event
    if (tid < TILE) {
      const int el = tid;
      const int64_t e = S.ev[el];
      if (e >= 0) {
        double v = 0;
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const cplx hl = mk(S.HLre[h][el], S.HLim[h][el]);
          const cplx a1 = mk(S.A1re[h][el], S.A1im[h][el]);
          v += norm2(hl) + 2.0 * wgt * (hl.re * a1.re + hl.im * a1.im) + c2 * S.A2[h][el];
        }
        double fxe = v, vnw = 0;
        if (!band) {
          const float wfe = __ldg(ev.pp + e + 2 * ev.n_size);
          if (!(wfe <= -1000.f)) {
            fxe = v * (double)wfe;
            vnw = S.VN[el] * (double)wfe;
          }
        }
        if (fx_out) fx_out[e] = fxe;
        acc.add(e, nda, ev.sw, fxe, vnw, band != 0);
      }
    }
    __syncthreads();
  }
  block_reduce_store<SMEAR_THREADS>(acc.data, acc.mc, acc.mcn, acc.bad, parts);
}

// ------------------------------------------------------------------------------- tables
// Exact K-matrix outputs at every grid node of every active J^P group.
__global__ void k_build_tables(const PointTable* __restrict__ T, int n_nodes) {
  const int64_t total = 4 * (int64_t)n_nodes;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int ik = (int)(t / n_nodes), j = (int)(t % n_nodes);
    cplx* dst = const_cast<cplx*>(T->tab.data[ik]);
    if (!dst) continue;
    const double m = T->tab.m_lo + j * T->tab.h;
    cplx out[TAB_SLOTS];
#pragma unroll
    for (int o = 0; o < TAB_SLOTS; ++o) out[o] = mk(0, 0);
    km_solve(T->G[ik], m, T->ffb, out);
#pragma unroll
    for (int o = 0; o < TAB_SLOTS; ++o) dst[(size_t)j * TAB_SLOTS + o] = out[o];
  }
}

// Verifies every interval [j, j+1] of every table: the 6-point interpolant at three interior points
// against exact solves; flags the interval when the largest output error exceeds TAB_CHECK_TOL times
// the largest output magnitude.
__global__ void k_check_tables(const PointTable* __restrict__ T, int n_nodes) {
  const int64_t total = 4 * (int64_t)n_nodes;
  const LineTables& tab = T->tab;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int ik = (int)(t / n_nodes), j = (int)(t % n_nodes);
    if (!tab.data[ik]) continue;
    unsigned char* bad = const_cast<unsigned char*>(tab.bad[ik]);
    if (j < 2 || j + 3 >= n_nodes) {
      bad[j] = 1;
      continue;
    }
    const int nout = T->G[ik].npole + NKMC;
    const cplx* base = tab.data[ik] + (size_t)(j - 2) * TAB_SLOTS;
    bool ok = true;
    // the stencil [m_{j-2}, m_{j+3}] must not reach into a guard interval
    const double s_lo = tab.m_lo + (j - 2) * tab.h, s_hi = tab.m_lo + (j + 3) * tab.h;
    for (int q = 0; q < tab.nguard; ++q)
      if (s_hi >= tab.guard_lo[q] && s_lo <= tab.guard_hi[q]) ok = false;
    const double ts[3] = {0.2, 0.5, 0.8};
    for (int q = 0; q < 3 && ok; ++q) {
      const double tt = ts[q];
      const double d0 = tt + 2.0, d1 = tt + 1.0, d2 = tt, d3 = tt - 1.0, d4 = tt - 2.0, d5 = tt - 3.0;
      const double w[6] = {d1 * d2 * d3 * d4 * d5 * (-1.0 / 120.0), d0 * d2 * d3 * d4 * d5 * (1.0 / 24.0),
                           d0 * d1 * d3 * d4 * d5 * (-1.0 / 12.0), d0 * d1 * d2 * d4 * d5 * (1.0 / 12.0),
                           d0 * d1 * d2 * d3 * d5 * (-1.0 / 24.0), d0 * d1 * d2 * d3 * d4 * (1.0 / 120.0)};
      cplx ex[TAB_SLOTS];
      km_solve(T->G[ik], tab.m_lo + (j + tt) * tab.h, T->ffb, ex);
      double emax = 0, vmax = 0;
      for (int o = 0; o < nout; ++o) {
        cplx acc = mk(0, 0);
        for (int k = 0; k < 6; ++k) acc += base[k * TAB_SLOTS + o] * w[k];
        emax = fmax(emax, sqrt(norm2(acc - ex[o])));
        vmax = fmax(vmax, sqrt(norm2(ex[o])));
      }
      ok = isfinite(emax) && emax <= TAB_CHECK_TOL * vmax;
    }
    bad[j] = ok ? 0 : 1;
  }
}

cudaError_t launch_build_tables(const PointTable* d_table, int n_nodes, int sm_count, cudaStream_t st) {
  k_build_tables<<<sm_count * 8, 128, 0, st>>>(d_table, n_nodes);
  k_check_tables<<<sm_count * 8, 128, 0, st>>>(d_table, n_nodes);
  return cudaGetLastError();
}

void attach_tables(PointTable* T, cplx* d_mem, unsigned char* d_flags) {
  bool any = false;
  for (int ik = 0; ik < 4; ++ik) {
    bool used = false;
    for (int g = 0; g < T->ngroups; ++g) used |= (T->grp[g].km == ik);
    T->tab.data[ik] = used ? d_mem + (size_t)ik * TAB_NODES * TAB_SLOTS : nullptr;
    T->tab.bad[ik] = used ? d_flags + (size_t)ik * TAB_NODES : nullptr;
    any |= used;
  }
  T->tab.enabled = any ? 1 : 0;
}

// ------------------------------------------------------------------------------- finalize
__global__ void k_finalize(const Partial* parts, int n, double sum_w_mc, double sum_w_data, double nll_shift,
                           EvalResult* res) {
  // one warp; Neumaier compensated sums over the block partials
  __shared__ double s[4][32], c[4][32];
  const int l = threadIdx.x;
  double sum[4] = {0, 0, 0, 0}, comp[4] = {0, 0, 0, 0};
  for (int i = l; i < n; i += 32) {
    const double x[4] = {parts[i].data, parts[i].mc, parts[i].mc_noint, parts[i].n_nonpos};
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
    *res = r;
  }
}

// ------------------------------------------------------------------------------- host side
static int blocks_for(int64_t work, int per_block, int cap) {
  int64_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

int segment_blocks(const Segment& s, int sm_count) {
  const int64_t n = s.end - s.begin;
  if (s.kind == SMEAR_NONE) return blocks_for(n, UNSMEARED_THREADS, sm_count * 8);
  return blocks_for((n + TILE - 1) / TILE, 1, sm_count * 2);
}

static size_t smear_smem() { return sizeof(SmearShared); }

// A K-matrix group must have a channel layout (J^P in {1/2-, 3/2-, 1/2+, 3/2+}) and at most
// NPMAX + NKMC outputs.
static int G_valid_check(const KmGroup& G) { return (G.npole <= NPMAX) ? 0 : 1; }

cudaError_t launch_segment(const EventSet& ev, const Segment& seg, const PointTable* d_table, Partial* out,
                           double* fx_out, int sm_count, cudaStream_t st) {
  if (seg.end <= seg.begin) return cudaSuccess;
  const int nb = segment_blocks(seg, sm_count);
  const int band = (seg.kind == SMEAR_30 || seg.kind == SMEAR_150) ? 1 : 0;
  switch (seg.kind) {
    case SMEAR_NONE:
      k_unsmeared<<<nb, UNSMEARED_THREADS, 0, st>>>(ev, ev.nda, seg.begin, seg.end, seg.list, d_table, out, fx_out, 0);
      break;
    case SMEAR_20:
      k_smeared<20><<<nb, SMEAR_THREADS, smear_smem(), st>>>(ev, ev.nda, seg.begin, seg.end, seg.list, d_table, out,
                                                             fx_out, band);
      break;
    case SMEAR_30:
      k_smeared<30><<<nb, SMEAR_THREADS, smear_smem(), st>>>(ev, ev.nda, seg.begin, seg.end, seg.list, d_table, out,
                                                             fx_out, band);
      break;
    case SMEAR_150:
      k_smeared<150><<<nb, SMEAR_THREADS, smear_smem(), st>>>(ev, ev.nda, seg.begin, seg.end, seg.list, d_table, out,
                                                              fx_out, band);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t configure_kernels() {
  const int smem = (int)smear_smem();
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_smeared<20>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))) return e;
  if ((e = cudaFuncSetAttribute(k_smeared<30>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))) return e;
  if ((e = cudaFuncSetAttribute(k_smeared<150>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))) return e;
  return cudaSuccess;
}

cudaError_t launch_finalize(const Partial* parts, int nparts, double sum_w_mc, double sum_w_data, double nll_shift,
                            EvalResult* res, cudaStream_t st) {
  k_finalize<<<1, 32, 0, st>>>(parts, nparts, sum_w_mc, sum_w_data, nll_shift, res);
  return cudaGetLastError();
}

cudaError_t launch_amp2(const EventSet& ev, const PointTable* d_table, double* out, int sm_count, cudaStream_t st) {
  if (ev.n <= 0) return cudaSuccess;
  const int nb = blocks_for(ev.n, UNSMEARED_THREADS, sm_count * 8);
  k_unsmeared<<<nb, UNSMEARED_THREADS, 0, st>>>(ev, 0, 0, ev.n, nullptr, d_table, nullptr, out, 1);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------- point table
// Masses in the table range where the reference's complex square root (csqrt_branch) changes branch
// for one of the complex-mass channels (D* Sigma_c, D* Sigma_c*, D Sigma_c, D Sigma_c*): the lineshape
// jumps there, so interpolation must not straddle them.  Scan plus bisection, computed once.
static const std::vector<double>& complex_branch_masses() {
  static std::vector<double> out;
  static std::once_flag once;
  std::call_once(once, [] {
    const cplx ch[4][2] = {{mk(KM_DST, 0), mk(KM_SC, KM_SC_HW)}, {mk(KM_DST, 0), mk(KM_SCST, KM_SCST_HW)},
                           {mk(KM_D, 0), mk(KM_SC, KM_SC_HW)}, {mk(KM_D, 0), mk(KM_SCST, KM_SCST_HW)}};
    for (auto& c : ch) {
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
          out.push_back(0.5 * (a + b));
          prev = st;
        }
        prev_m = m;
      }
    }
  });
  return out;
}

// Decodes the float parameter block (layout of cu_init_data, RooDalitzAmplitude.cxx:3141-3210;
// coupling offsets of cuda_configure_ampcount, kernel_calEva.cu:1014-1098; K-matrix output slots
// of cuda_configure_Pc_KMatrix, :978-1010) and hoists every parameter-only constant.
int build_point_table(const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                      float ffr, float ffb, PointTable* T) {
  std::memset(T, 0, sizeof(PointTable));
  if (NX != 0) return 5;                       // PWA_E_UNSUPPORTED: Zcs chain
  if (NR > MAX_LSTAR || NZ > MAX_PC || NR < 0 || NZ < 0) return 4;  // PWA_E_SIZE
  if (para_size != NSET * (NR + NZ + NX)) return 3;                 // PWA_E_LAYOUT
  T->NR = NR;
  T->NZ = NZ;
  T->ffr = ffr;
  T->ffb = ffb;
  const double mmin = M_K + M_P, mmax = M_LB - M_JPSI;
  const double thr_pk = (double)(float)(M_P + M_K);
  const double thr_pz = (double)(float)(M_P + M_JPSI);
  int cnt = para_size;
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
    if (type == REF_BREITWIGNER)
      L.type = LT_BW;
    else if (type == REF_NONRESONANT)
      L.type = LT_NR;
    else
      return 5;
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
    // Lambda_b barrier constants (BTerm)
    const double J = 0.5 * S2;
    L.LB = (J <= 1) ? 0 : (int)(J - 1.5);
    double pB0 = -1;
    if (m_r < 0) pB0 = two_body_p(M_LB, M_JPSI, (mmin + mmax) / 2.0);
    if (m_r > 1e-10 && m_r + M_JPSI < M_LB) pB0 = two_body_p(M_LB, M_JPSI, m_r);
    if (m_r + M_JPSI > M_LB) pB0 = two_body_p(M_LB, M_JPSI, tanh_eff_mass(m_r, mmin, mmax));
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
    if (type == REF_BREITWIGNER)
      Z.type = LT_BW;
    else if (type == REF_KMATRIX)
      Z.type = LT_KM;
    else if (type == REF_NONRESONANT)
      Z.type = LT_NR;
    else
      return 5;
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
    double pB0 = -1;
    if (Z.m_r < 0) pB0 = two_body_p(M_LB, M_K, (M_JPSI + M_P + M_LB - M_K) / 2.0);
    if (Z.m_r > 1e-10 && Z.m_r + M_K < M_LB) pB0 = two_body_p(M_LB, M_K, Z.m_r);
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
  if (cnt != para_size + vamp_size) return 3;
  // K-matrix groups (Default_KMatrix pole scan and near-threshold mass shift, :674-746)
  const int kmcount = para_size + vamp_size + spline_size;
  for (int ik = 0; ik < 4; ++ik) {
    KmGroup& G = T->G[ik];
    G.J2 = (ik == 1 || ik == 3) ? 3 : 1;
    G.P = (ik >= 2) ? 1 : -1;
    G.Lna = (G.P == 1) ? 1 : 0;
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
      if (ich > 0) {
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
  // table grid and guard intervals (tables stay disabled until the caller attaches table memory)
  LineTables& tb = T->tab;
  tb.enabled = 0;
  tb.n_nodes = TAB_NODES;
  tb.m_lo = TAB_M_LO;
  tb.h = TAB_H;
  tb.inv_h = 1.0 / TAB_H;
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
  if (pos_parity) {  // real-mass channel thresholds of the positive-parity groups
    guard(KM_DST + KM_SC, cusp);
    guard(KM_D + KM_SC, cusp);
    guard(KM_D + KM_SCST, cusp);
  }
  if (neg_parity)
    for (double m : complex_branch_masses()) guard(m, step);
  if (tb.nguard >= MAX_GUARDS) return 4;
  return 0;
}

// Host evaluation of the decoded lineshapes (diagnostics and CPU tests of the point table): Lambda*
// lineshape x production barrier at mkp, and every Pc entry's lineshape x barrier at mz, entries in
// parameter-block order.
void host_lineshapes(const PointTable& T, double mkp, double mz, cplx* lstar, cplx* pc) {
  const LstarKin lk = lstar_kin(T, mkp);
  const PcKin pk = pc_kin(T, mz);
  for (int r = 0; r < T.NR; ++r) lstar[r] = lstar_lineshape(T.L[r], lk);
  for (int g = 0; g < T.ngroups; ++g) {
    const PcGroup& gr = T.grp[g];
    cplx kmo[NPMAX + NKMC];
    if (gr.km >= 0) km_solve(T.G[gr.km], mz, T.ffb, kmo);
    for (int q = 0; q < gr.count; ++q) {
      const int i = T.order[gr.first + q];
      const PcEntry& Z = T.Z[i];
      cplx v = (Z.type == LT_KM) ? kmo[Z.slot] : (Z.type == LT_BW) ? pc_bw(Z, pk) : mk(1, 0);
      pc[i] = v * pc_barrier(Z, pk);
    }
  }
}

}  // namespace pwa
