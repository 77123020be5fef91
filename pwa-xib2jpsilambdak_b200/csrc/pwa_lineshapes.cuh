// Lineshapes besides the Breit-Wigners and the coupled-channel K-matrix, in FP64 on the reference's
// float parameters: spline (model-independent) waves, the revised K-matrix, the triangle cusp
// (src/cu_DPFPropogator.cu:825-1343).  Used on the host (decoding, diagnostics) and on the device
// (per-event Lambda* lineshapes, Pc lineshape tables and their exact fallback).
#pragma once
#include <cmath>

#include "pwa_point.cuh"

namespace pwa {

// Domains of the spline waves: zero outside (float sums of the reference, ModelIndependentWave3 for
// the Lambda* chain, ModelIndependentWave for the Pc chain).
constexpr double SPL_L_LO = (double)(0.938272046f + 0.493677f - 0.002f);
constexpr double SPL_L_HI = (double)(5.61951f - 3.096916f + 0.002f);
constexpr double SPL_Z_LO = (double)(0.938272046f + 3.096916f - 0.002f);
constexpr double SPL_Z_HI = PWA_F(4.6f);

// Piecewise cubic of a spline block at x: the interval from the reference's bisection over the n
// knots (x above the last knot continues the last interval; x = hi uses the last knot's row).
__host__ __device__ inline cplx spline_wave(const float* poly, int n, double lo, double hi, double x) {
  if (x < lo || x > hi) return mk(0, 0);
  int klow = 0, khig = n - 1;
  if (x >= hi) {
    klow = khig;
  } else if (x > lo) {
    while (khig - klow > 1) {
      const int khalf = (klow + khig) / 2;
      if (x > (double)poly[khalf])
        klow = khalf;
      else
        khig = khalf;
    }
  }
  const double dx = x - (double)poly[klow];
  const float* a = poly + n + 4 * klow;
  const float* b = a + 4 * n;
  return mk(fma(dx, fma(dx, fma(dx, (double)a[3], (double)a[2]), (double)a[1]), (double)a[0]),
            fma(dx, fma(dx, fma(dx, (double)b[3], (double)b[2]), (double)b[1]), (double)b[0]));
}

// Revised K-matrix lineshape of entry i of chain c (0 Lambda*: p K system; 1 Pc: J/psi p system)
// at mass mpp (Revised_KMAMP, cu_DPFPropogator.cu:825-926).  The other entries of its set add their
// KMatrixTerm (:928-972) times the own denominator; the first non-resonant one fixes fsc, which the
// later ones return and which enters the own term below threshold.
__host__ __device__ inline cplx rkm_lineshape(const PointTable& T, int c, int i, double mpp) {
  const RkmEntry& R = T.rkm[c][i];
  const double s = mpp * mpp, ffr = T.ffr;
  double denorm = (R.m > 0) ? R.m * R.m - s : 1.0;
  double totG = 0, fsc = 0;
  const double pk = two_body_p(mpp, M_P, M_K);
  for (int j = 0; j < T.nrkm[c]; ++j) {
    const RkmEntry& E = T.rkm[c][j];
    if (j == i || E.set != R.set) continue;
    const double FR = barrier_ratio_pre(ffr, E.LR, pk, E.polyR0k);
    const double gamma = E.g * ipow(pk * E.inv_pR0k, 2 * E.LR + 1) * (E.m / mpp) * FR * FR;
    double term;
    if (E.m < 0) {
      if (fabs(fsc) < 1e-10) fsc = gamma;
      term = fsc;
    } else {
      const double d = E.m * E.m - s;
      term = (fabs(d) < 1e-10) ? 0.0 : E.m * gamma / d;
    }
    totG += term * denorm;
  }
  const double pR = (c == 0) ? pk : two_body_p(mpp, M_JPSI, M_P);
  const double FR = barrier_ratio_pre(ffr, R.LR, pR, R.polyR0c);
  const double ratio = pR * R.inv_pR0c;
  double factor = FR * ipow(ratio, R.LR);
  if (R.branch != 3) {
    double gamma = R.g;
    if (R.branch == 0) {
      gamma = R.g * ipow(ratio, 2 * R.LR + 1) * (R.m / mpp) * FR * FR;
    } else if (R.branch == 1) {  // the reference's Sigma pi channel (written for the Lambda(1405))
      const double pSP = two_body_p(mpp, PWA_F(1.18937f), PWA_F(0.13957018f));
      const double sp = PWA_F(0.0505f) * ipow(pSP * R.inv_pR0sp, 2 * R.LR + 1) * (R.m / mpp);
      gamma = R.g * ipow(pR * R.inv_pR0sp, 2 * R.LR + 1) * (R.m / mpp) + sp;
      denorm -= fsc * sp * R.m;
    }
    totG += R.m * gamma;
    factor *= R.factor;
  } else {
    totG += R.g * ipow(ratio, 2 * R.LR + 1) * (R.m / mpp) * FR * FR;
  }
  const double d2 = denorm * denorm + totG * totG;
  return mk(denorm / d2, totG / d2) * factor;
}

// Complex division and the reference's complex logarithm and arctangent (RooTDalitz/cuComplex.h:
// 660-676): the argument from acos(Re / |z|), negated for Im < 0; atan(z) = -i/2 log((1 + i z) / (1 - i z)).
// Re / |z| is clamped to [-1, 1]: rounding can push it just outside for a nearly real z, where acos
// would return NaN (the reference's float code has the same hazard).
__host__ __device__ inline cplx cdiv(cplx a, cplx b) {
  const double d = 1.0 / (b.re * b.re + b.im * b.im);
  return mk((a.re * b.re + a.im * b.im) * d, (a.im * b.re - a.re * b.im) * d);
}
__host__ __device__ inline cplx clog_ref(cplx x) {
  const double r = sqrt(x.re * x.re + x.im * x.im);
  double th = acos(fmin(1.0, fmax(-1.0, x.re / r)));
  if (x.im < 0) th = -th;
  return mk(log(r), th);
}
__host__ __device__ inline cplx catan_ref(cplx x) {
  const cplx ix = mk(-x.im, x.re);
  const cplx l = clog_ref(cdiv(mk(1.0 + ix.re, ix.im), mk(1.0 - ix.re, -ix.im)));
  return mk(0.5 * l.im, -0.5 * l.re);  // -i/2 * l
}

// Triangle cusp (GetCusp_AMP, cu_DPFPropogator.cu:1223-1343): midpoint rule over 100 bins of the
// loop-parameter integrand, each through the reference's complex square root.  m_r, gamma: mass and
// width of the particle in the loop; the other two are chi_c1 and the proton.
__host__ __device__ inline cplx cusp_lineshape(double m_r, double gamma, double mpp) {
  constexpr double P12 = M_LB, P13 = M_K, M2 = PWA_F(3.51067f), M3 = M_P;
  const cplx m1 = mk(m_r, -gamma / 2.0);
  const cplx m1sq = m1 * m1;
  const double inv_p2 = 1.0 / (mpp * mpp);
  const float dxf = (float)(1.0 / 100);
  const double dx = dxf;
  cplx acc = mk(0, 0);
  for (int i = 0; i < 100; ++i) {
    const double a = (double)((float)i * dxf + dxf / 2.0f);
    const cplx b = mk((a * (P12 * P12 - P13 * P13 - mpp * mpp) + M3 * M3 - M2 * M2) * inv_p2 + 1.0, -0.001);
    const cplx cc = mk((a * (m1sq.re - M3 * M3) + M3 * M3 - a * (1.0 - a) * P13 * P13) * inv_p2, a * m1sq.im * inv_p2);
    const cplx sv = csqrt_branch(4.0 * cc - b * b);
    const cplx t1 = catan_ref(cdiv(b, sv));
    const cplx t2 = catan_ref(cdiv(b + mk(2.0 * (a - 1.0), 0), sv));
    acc += dx * cdiv(t1 - t2, sv);
  }
  return acc * inv_p2;
}

}  // namespace pwa
