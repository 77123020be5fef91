// Device code shared by the likelihood kernels (pwa_kernels.cu) and the batched evaluator
// (pwa_batch.cu): per-event kinematics, lineshapes, the coupled-channel K-matrix, lookups of the
// per-point lineshape tables, SoA access, reductions and the event-range helpers.
#pragma once
#include <cmath>

#include "pwa_kernels.cuh"
#include "pwa_lineshapes.cuh"

namespace pwa {

// Resolution offsets in units of the mass resolution (reference data, Resonances.h:31-54).
#include "smear_tables.inc"

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

// Spline and revised K-matrix Lambda* lineshapes (GetAmpLz's MODELINDEPENDENT and REVISEDKMATRIX
// cases, kernel_calEva.cu:136-150).
static __host__ __device__ __forceinline__ cplx lstar_general(const PointTable& T, int r, double mkp) {
  const LstarEntry& L = T.L[r];
  if (L.type == LT_SPLINE) return spline_wave(T.spl + L.aux, SPL_KNOTS_L, SPL_L_LO, SPL_L_HI, mkp);
  return rkm_lineshape(T, 0, L.aux, mkp);
}

// Lambda* lineshape r times the Lambda_b -> Lambda* J/psi barrier (BW_AMP, cu_DPFPropogator.cu:248-314;
// BTerm :155-181; a spline wave takes the non-resonant barrier) with the parameter-only constants of
// the point table.
// GEN = false: the model has Breit-Wigner and non-resonant Lambda* entries only.
template <bool GEN = true>
__host__ __device__ inline cplx lstar_lineshape(const PointTable& T, int r, const LstarKin& k) {
  const LstarEntry& L = T.L[r];
  cplx bw = mk(1, 0);
  if (GEN && (L.type == LT_SPLINE || L.type == LT_RKM)) {
    bw = lstar_general(T, r, k.mkp);
  } else if (L.type == LT_BW) {
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

// Spline, revised K-matrix and triangle-cusp Pc lineshapes (GetAmp2s / TemplateGetAmp2s cases,
// kernel_calEva.cu:404-425, 708-730), out of line.
static __host__ __device__ __noinline__ cplx pc_general(const PointTable& T, const PcEntry& Z, double mz) {
  if (Z.type == LT_SPLINE) return spline_wave(T.spl + Z.aux, SPL_KNOTS_Z, SPL_Z_LO, SPL_Z_HI, mz);
  if (Z.type == LT_RKM) return rkm_lineshape(T, 1, Z.aux, mz);
  return cusp_lineshape(Z.m_r, Z.g_r, mz);
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

// Zcs -> J/psi K lineshapes at m(J/psi K): Breit-Wigner (BW_AMPX, cu_DPFPropogator.cu:226-246) times
// the Lambda_b -> Zcs p barrier (BTermX, :205-217).
struct XKin {
  double inv_m, s, pR, pBm;
  double rsR[6], rsB[6];
};

__host__ __device__ inline XKin x_kin(const PointTable& T, double mjk) {
  XKin k;
  k.inv_m = 1.0 / mjk;
  k.s = mjk * mjk;
  k.pR = two_body_p(mjk, M_K, M_JPSI);
  const double pB = two_body_p(M_LB, M_P, mjk);
  k.pBm = pB / M_LB;
  fill_rs(k.rsR, T.lmask_x_R, T.ffr, k.pR);
  fill_rs(k.rsB, T.lmask_x_B, T.ffb, pB);
  return k;
}

__host__ __device__ inline cplx x_lineshape(const XEntry& X, const XKin& k) {
  double FR = 1.0, gamma = X.g_r, ratio = 1.0;
  if (X.bw_above) {
    FR = X.sqrt_polyR0 * k.rsR[X.LR];
    ratio = k.pR * X.inv_pR0;
    gamma = X.g_r * ipow(ratio, 2 * X.LR + 1) * (X.m_r * k.inv_m) * FR * FR;
  }
  const double factor = FR * ipow(ratio, X.LR) * X.norm;
  const double de2 = X.m_r * X.m_r - k.s, gm = gamma * X.m_r;
  const double f = factor / (de2 * de2 + gm * gm);
  const double FB = (X.lb_mode != 0 || X.LB == 0) ? 1.0 : X.sqrt_polyB0 * k.rsB[X.LB];
  return mk(de2 * f, gm * f) * (FB * ipow(k.pBm, X.LB));
}

// One J^P group of the 7-channel isospin-split K-matrix (Isospin_KMatrix, cu_DPFPropogator.cu:
// 384-586): J/psi p and the charged / neutral partners of the three Sigma_c(*) D(*) channels, the
// 4 x 4 couplings and scattering terms spread over them with the isospin factors, a 7 x 7 solve, and
// the first row folded back onto the 4 production channels.  Outputs as km_solve's.  Kept out of line:
// only the isospin build calls it, and the default kernels keep their register allocation.
static __host__ __device__ __noinline__ void km_solve_iso(const KmGroup& G, double mz, double ffb, cplx* out) {
  const double s = mz * mz;
  cplx rho[7];
  rho[0] = rho_real(s, M_P, M_JPSI, G.Lna, ffb);
  const cplx dstm = mk(KMI_DSTM, 0), dst0 = mk(KMI_DST0, 0), dm = mk(KMI_DM, 0), d0 = mk(KMI_D0, 0);
  const cplx scpp = mk(KMI_SCPP, KMI_SCPP_HW), scp = mk(KMI_SCP, KMI_SCP_HW);
  const cplx scstpp = mk(KMI_SCSTPP, KMI_SCSTPP_HW), scstp = mk(KMI_SCSTP, KMI_SCSTP_HW);
  if (G.P == -1) {
    rho[1] = rho_complex(s, dstm, scpp);
    rho[2] = rho_complex(s, dst0, scp);
    rho[3] = rho_complex(s, dstm, scstpp);
    rho[4] = rho_complex(s, dst0, scstp);
    rho[5] = rho_complex(s, dm, G.J2 == 1 ? scpp : scstpp);
    rho[6] = rho_complex(s, d0, G.J2 == 1 ? scp : scstp);
  } else {
    rho[1] = rho_real(s, KMI_DSTM, KMI_SCPP, G.Lna, ffb);
    rho[2] = rho_real(s, KMI_DST0, KMI_SCP, G.Lna, ffb);
    rho[3] = rho_real(s, KMI_DM, KMI_SCPP, G.Lna, ffb);
    rho[4] = rho_real(s, KMI_D0, KMI_SCP, G.Lna, ffb);
    rho[5] = rho_real(s, KMI_DM, KMI_SCSTPP, G.Lna, ffb);
    rho[6] = rho_real(s, KMI_D0, KMI_SCSTP, G.Lna, ffb);
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
  // channel i >= 1 is production channel (i + 1) / 2 with isospin factor ISO0 (odd i) or ISO1
  auto iso = [](int i) { return i == 0 ? 1.0 : ((i + 1) % 2 == 0 ? KMI_ISO0 : KMI_ISO1); };
  cplx S[7][7];
#pragma unroll
  for (int i = 0; i < 7; ++i)
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      const int a = i < j ? i : j, b = i < j ? j : i;  // the reference fills the upper triangle
      const int ap = (a + 1) / 2, bp = (b + 1) / 2;
      const double f = iso(a) * iso(b);
      double v = f * (G.f[ap][bp] * ms[0]);
      for (int p = 0; p < G.npole; ++p) v += f * G.g[p][ap] * mg[p][bp];
      S[i][j] = mk(v * rho[j].im, -v * rho[j].re);
      if (i == j) S[i][j].re += ms[0];
    }
  cplx T7[7];
  first_row_inverse<7>(S, T7);
  const cplx T[NKMC] = {T7[0], T7[1] * KMI_ISO0 + T7[2] * KMI_ISO1, T7[3] * KMI_ISO0 + T7[4] * KMI_ISO1,
                        T7[5] * KMI_ISO0 + T7[6] * KMI_ISO1};
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

// One J^P group of the coupled-channel K-matrix at mass mz (Default_KMatrix,
// cu_DPFPropogator.cu:588-813): P-vector outputs, npole poles first then 4 production terms.
__host__ __device__ inline void km_solve(const KmGroup& G, double mz, double ffb, cplx* out) {
  if (G.iso) {
    km_solve_iso(G, mz, ffb, out);
    return;
  }
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

// ------------------------------------------------------------------------------- Pc entry tables
// Exact lineshapes (with production barrier) of the entries of Pc group g at the mass of k, written
// to raw[0 .. count) (order positions gr.first ...).
__host__ __device__ inline void pc_group_exact(const PointTable& T, int g, const PcKin& k, cplx* raw) {
  const PcGroup& gr = T.grp[g];
  cplx kmo[NPMAX + NKMC];
  if (gr.km >= 0) km_solve(T.G[gr.km], k.mz, T.ffb, kmo);
  for (int q = 0; q < gr.count; ++q) {
    const PcEntry& Z = T.Z[T.order[gr.first + q]];
    const cplx v = (Z.type == LT_KM)   ? kmo[Z.slot]
                   : (Z.type == LT_BW) ? pc_bw(Z, k)
                   : (Z.type == LT_NR) ? mk(1, 0)
                                       : pc_general(T, Z, k.mz);
    raw[q] = v * pc_barrier(Z, k);
  }
}

// Every Pc entry's lineshape at mass m, exactly, at raw[order position].  Kept out of line so that
// the rarely taken exact path does not set the register budget of the event kernels.
static __device__ __noinline__ void pc_entries_exact(const PointTable& T, double m, cplx* raw) {
  const PcKin kin = pc_kin(T, m);
  for (int g = 0; g < T.ngroups; ++g) pc_group_exact(T, g, kin, raw + T.grp[g].first);
}

// 6-point Lagrange weights for nodes j-2 .. j+3 at x = j + t (denominators -120, 24, -12, 12, -24, 120).
__host__ __device__ __forceinline__ void lagrange6(double t, double* w) {
  const double d0 = t + 2.0, d1 = t + 1.0, d2 = t, d3 = t - 1.0, d4 = t - 2.0, d5 = t - 3.0;
  const double p01 = d0 * d1, p012 = p01 * d2, p0123 = p012 * d3, p01234 = p0123 * d4;
  const double s45 = d4 * d5, s345 = d3 * s45, s2345 = d2 * s345, s12345 = d1 * s2345;
  w[0] = s12345 * (-1.0 / 120.0);
  w[1] = d0 * s2345 * (1.0 / 24.0);
  w[2] = p01 * s345 * (-1.0 / 12.0);
  w[3] = p012 * s45 * (1.0 / 12.0);
  w[4] = p0123 * d5 * (-1.0 / 24.0);
  w[5] = p01234 * (1.0 / 120.0);
}

struct TabAt {
  const double2* base;  // first stencil node, order position 0
  double w[6];
};

// Locates mass m on the per-point entry table: the level-1 grid, or the refined block of a flagged
// interval; false when neither can serve m (the caller then evaluates exactly).
__device__ __forceinline__ bool tab_at(const LineTables& tab, double m, TabAt& a) {
  if (!tab.enabled) return false;
  const double x = (m - tab.m_lo) * tab.inv_h;
  const double fj = floor(x);
  if (!(fj >= 2.0 && fj + 3.0 < (double)tab.n_nodes)) return false;
  const int j = (int)fj;
  const int c = __ldg(tab.cell + j);
  if (c == 0) {
    lagrange6(x - fj, a.w);
    a.base = reinterpret_cast<const double2*>(tab.data) + (size_t)(j - 2) * tab.stride;
    return true;
  }
  if (c < 0) return false;
  const double x2 = (x - fj) * (double)TAB_SUB;
  const double fi = fmin(floor(x2), (double)(TAB_SUB - 1));
  const int i = (int)fi;
  if (__ldg(tab.sub_bad + (size_t)(c - 1) * TAB_SUB + i)) return false;
  lagrange6(x2 - fi, a.w);
  a.base = reinterpret_cast<const double2*>(tab.sub) + ((size_t)(c - 1) * TAB_SUB_NODES + i) * tab.stride;
  return true;
}

__device__ __forceinline__ cplx tab_get(const TabAt& a, int stride, int pos) {
  cplx acc = mk(0, 0);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double2 v = __ldg(a.base + k * stride + pos);
    acc.re = fma(a.w[k], v.x, acc.re);
    acc.im = fma(a.w[k], v.y, acc.im);
  }
  return acc;
}

// All Pc entry lineshapes at mass m into out[order position] from a table of every group; false
// (and zeros) when the table cannot serve m.
__device__ __forceinline__ bool lookup_table(const PointTable& T, double m, cplx* out) {
  TabAt ta;
  const bool ok = tab_at(T.tab, m, ta);
#pragma unroll 2
  for (int q = 0; q < T.NZ; ++q) out[q] = ok ? tab_get(ta, T.tab.stride, q) : mk(0, 0);
  return ok;
}

// All Pc entry lineshapes at mass m into out[order position]: interpolated, or exact where the table
// cannot serve the mass.
__device__ __forceinline__ void lookup_entries(const PointTable& T, double m, cplx* out) {
  TabAt ta;
  if (tab_at(T.tab, m, ta)) {
#pragma unroll 2
    for (int q = 0; q < T.NZ; ++q) out[q] = tab_get(ta, T.tab.stride, q);
  } else {
    pc_entries_exact(T, m, out);
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

__device__ __forceinline__ bool nonzero(cplx c) { return c.re != 0.0 || c.im != 0.0; }

// Zcs planes of one event: pp3 plane 0 m(J/psi K), planes 1 + 2 (i*24 + j*12 + m) (+1) the angular
// factors AX; pp4 plane s*24 + k*12 + m the d-functions DX (GetAmpZcs, kernel_calEva.cu:192-286).
struct EvX {
  const float *pp3, *pp4;
  int64_t ns, e;
  __device__ __forceinline__ double mjk() const { return ldf(pp3, e); }
  __device__ __forceinline__ cplx AX(int i, int j, int m) const {
    const int a = 1 + (i * 24 + j * 12 + m) * 2;
    return mk(ldf(pp3, e + a * ns), ldf(pp3, e + (a + 1) * ns));
  }
  __device__ __forceinline__ double DX(int s, int k, int m) const { return ldf(pp4, e + (s * 24 + k * 12 + m) * ns); }
};

// One event's planes staged in shared memory as doubles (slots SLOT_*), with the accessors of Ev / EvX.
struct EvS {
  const double* p;
  __device__ __forceinline__ double mkp() const { return p[0]; }
  __device__ __forceinline__ double mz() const { return p[1]; }
  __device__ __forceinline__ cplx A(int i, int j, int m) const {
    const int a = 3 + (i * 12 + j * 6 + m) * 2;
    return mk(p[a], p[a + 1]);
  }
  __device__ __forceinline__ double DL(int s, int k, int m) const { return p[51 + s * 12 + k * 6 + m]; }
  __device__ __forceinline__ cplx AZ(int i, int j, int m) const {
    const int a = SLOT_PP1 + (i * 24 + j * 12 + m) * 2;
    return mk(p[a], p[a + 1]);
  }
  __device__ __forceinline__ double DZ(int s, int k, int m) const { return p[SLOT_PP2 + s * 24 + k * 12 + m]; }
  __device__ __forceinline__ double mjk() const { return p[SLOT_PP3]; }
  __device__ __forceinline__ cplx AX(int i, int j, int m) const {
    const int a = SLOT_PP3 + 1 + (i * 24 + j * 12 + m) * 2;
    return mk(p[a], p[a + 1]);
  }
  __device__ __forceinline__ double DX(int s, int k, int m) const { return p[SLOT_PP4 + s * 24 + k * 12 + m]; }
};

// Copies the plane slots point T reads of event e into dst (warp-cooperative, lane = 0 .. 31),
// converting to double; the caller synchronises the warp before reading.
__device__ __forceinline__ void stage_event(const PointTable& T, const EventSet& ev, int64_t e, double* dst,
                                            int lane) {
  for (int i = lane; i < T.nstage; i += 32) {
    const int s = T.stage[i];
    const float* src;
    int plane;
    if (s < SLOT_PP1) {
      src = ev.pp;
      plane = s;
    } else if (s < SLOT_PP2) {
      src = ev.pp1;
      plane = s - SLOT_PP1;
    } else if (s < SLOT_PP3) {
      src = ev.pp2;
      plane = s - SLOT_PP2;
    } else if (s < SLOT_PP4) {
      src = ev.pp3;
      plane = s - SLOT_PP3;
    } else {
      src = ev.pp4;
      plane = s - SLOT_PP4;
    }
    dst[s] = ldf(src, e + (int64_t)plane * ev.n_size);
  }
}

// Zcs chain amplitudes of proton helicity k for the helicities (i, j) in ij_lo .. ij_hi - 1
// (ij = 2 i + j), added to H[ij - ij_lo]: sum_x lineshape_x sum_m c_{x,k,m} DX AX.
template <int NIJ, class XA>
__device__ __forceinline__ void zcs_amplitudes(const PointTable& T, const XA& X, int k, int ij_lo, cplx* H) {
  const XKin xk = x_kin(T, X.mjk());
  for (int x = 0; x < T.NX; ++x) {
    const XEntry& Xe = T.X[x];
    const cplx bw = x_lineshape(Xe, xk);
#pragma unroll 1
    for (int m = 0; m < 12; ++m) {
      const cplx c = Xe.c[k * 12 + m];
      if (!nonzero(c)) continue;
      const cplx D = (bw * c) * X.DX(Xe.sidx, k, m);
#pragma unroll
      for (int q = 0; q < NIJ; ++q) {
        const int ij = ij_lo + q;
        cmac(H[q], X.AX(ij >> 1, ij & 1, m), D);
      }
    }
  }
}

__device__ __forceinline__ cplx shfl_xor(cplx v, int o) {
  return mk(__shfl_xor_sync(0xffffffffu, v.re, o), __shfl_xor_sync(0xffffffffu, v.im, o));
}

__device__ __forceinline__ cplx shfl(cplx v, int src) {
  return mk(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
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
  static_assert(sizeof(PointTable) % sizeof(int4) == 0, "PointTable must be a whole number of int4");
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

// ------------------------------------------------------------------------------- event kernels
constexpr int EV_THREADS = 256;
constexpr int EV_WARPS = EV_THREADS / 32;
constexpr int UNSMEARED_PER_WARP = 16;  // events per warp: lane = 16 * k + event

__device__ __forceinline__ int64_t event_index(const int32_t* list, int64_t begin, int64_t p) {
  return list ? (int64_t)list[begin + p] : begin + p;
}

// Work of this warp: groups warp0, warp0 + wstep, ... of positions [c0, c1).  Segments give each block
// a contiguous share, a whole number of rounds long, so consecutive rounds of a block take
// neighbouring events (masses) whose lineshape-table nodes stay in L1.  Deferred lists (few events,
// no mass order) are spread over all warps of the grid instead.
struct Chunk {
  int64_t c0, c1, warp0, wstep;
};
__device__ __forceinline__ Chunk block_chunk(int64_t count, int per_round, bool interleave) {
  if (interleave) return Chunk{0, count, (int64_t)blockIdx.x * EV_WARPS + threadIdx.x / 32, (int64_t)gridDim.x * EV_WARPS};
  int64_t chunk = (count + gridDim.x - 1) / gridDim.x;
  chunk = (chunk + per_round - 1) / per_round * per_round;
  const int64_t c0 = (int64_t)blockIdx.x * chunk;
  return Chunk{c0, min(count, c0 + chunk), threadIdx.x / 32, EV_WARPS};
}

template <int NB>
__device__ __forceinline__ const float* smear_table();
template <>
__device__ __forceinline__ const float* smear_table<20>() { return kSmear20; }
template <>
__device__ __forceinline__ const float* smear_table<30>() { return kSmear30; }
template <>
__device__ __forceinline__ const float* smear_table<150>() { return kSmear150; }
template <>
__device__ __forceinline__ const float* smear_table<0>() { return nullptr; }  // weighted grid scheme

}  // namespace pwa
