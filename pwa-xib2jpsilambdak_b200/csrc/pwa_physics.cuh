// Device physics of the Lambda_b -> J/psi p K- likelihood, FP64.
//
// Restates the lineshape library of the reference (src/cu_DPFPropogator.cu) for sm_100a:
// two-body momenta, Blatt-Weisskopf barriers, Breit-Wigners, channel phase space (real and
// complex-mass, with the reference's own complex square-root branch rule) and the 4-channel Pc
// K-matrix with its unpivoted first-row inverse.  Every float constant of the reference enters as
// the same float value promoted to double; everything is computed in double.
//
// Parameter-dependent constants (pole masses after the near-threshold shift, barrier constants at
// the resonance mass, Breit-Wigner normalisation) are computed once per parameter point in
// PointTable (pwa_point.cuh) and only event-dependent work remains here.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace pwa {

struct cplx {
  double re, im;
};
__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx& operator+=(cplx& a, cplx b) {
  a.re += b.re;
  a.im += b.im;
  return a;
}
__host__ __device__ __forceinline__ cplx& operator-=(cplx& a, cplx b) {
  a.re -= b.re;
  a.im -= b.im;
  return a;
}
__host__ __device__ __forceinline__ cplx conj(cplx a) { return {a.re, -a.im}; }
__host__ __device__ __forceinline__ double norm2(cplx a) { return a.re * a.re + a.im * a.im; }
__host__ __device__ __forceinline__ cplx recip(cplx a) {
  const double d = 1.0 / (a.re * a.re + a.im * a.im);
  return {a.re * d, -a.im * d};
}
// acc += a * b (complex multiply-add)
__host__ __device__ __forceinline__ void cmac(cplx& acc, cplx a, cplx b) {
  acc.re = fma(a.re, b.re, fma(-a.im, b.im, acc.re));
  acc.im = fma(a.re, b.im, fma(a.im, b.re, acc.im));
}

// Float constants of the reference (cu_DPFPropogator.cu:11-14, :590-595; Resonances.h:56-58).
#define PWA_F(x) ((double)(float)(x))
constexpr double M_LB = PWA_F(5.61951f);
constexpr double M_K = PWA_F(0.493677f);
constexpr double M_P = PWA_F(0.938272046f);
constexpr double M_JPSI = PWA_F(3.096916f);
constexpr double KM_D = PWA_F(1.86719f);
constexpr double KM_DST = PWA_F(2.008555f);
constexpr double KM_SC = PWA_F(2.453435f);
constexpr double KM_SCST = PWA_F(2.517955f);
constexpr double KM_SC_HW = PWA_F(-0.00105f);
constexpr double KM_SCST_HW = PWA_F(-0.00800f);
constexpr double MRES0 = PWA_F(-0.134064f);
constexpr double MRES1 = PWA_F(0.0599014f);
constexpr double MRES2 = PWA_F(-0.00655841f);
constexpr double BW_NORM_C = PWA_F(0.948850f);
constexpr double KM_DENORM_MIN = PWA_F(1e-3f);

__host__ __device__ __forceinline__ double sq(double x) { return x * x; }

__host__ __device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// Two-body breakup momentum (|.| inside the root, as the reference).
__host__ __device__ __forceinline__ double two_body_p(double M, double m1, double m2) {
  const double M2 = M * M;
  return sqrt(fabs((M2 - sq(m1 + m2)) * (M2 - sq(m1 - m2)))) / 2.0 / M;
}

// Blatt-Weisskopf polynomial |h_L(z)|^2 z^-L denominators for L <= 5 (Von Hippel-Quigg form).
__host__ __device__ __forceinline__ double bw_poly(int L, double z) {
  switch (L) {
    case 1: return 1.0 + z;
    case 2: return fma(z, z + 3.0, 9.0);
    case 3: return fma(z, fma(z, z + 6.0, 45.0), 225.0);
    case 4: return fma(z, fma(z, fma(z, z + 10.0, 135.0), 1575.0), 11025.0);
    case 5: return fma(z, fma(z, fma(z, fma(z, z + 15.0, 315.0), 6300.0), 99225.0), 893025.0);
  }
  return 1.0;
}

// F_L(p)/F_L(p0) given the precomputed polynomial at p0.
__host__ __device__ __forceinline__ double barrier_ratio_pre(double r, int L, double p, double poly0) {
  if (L < 1 || L > 5) return 1.0;
  return sqrt(poly0 / bw_poly(L, sq(r * p)));
}
__host__ __device__ __forceinline__ double barrier_ratio(double r, int L, double p, double p0) {
  if (L < 1 || L > 5) return 1.0;
  return sqrt(bw_poly(L, sq(r * p0)) / bw_poly(L, sq(r * p)));
}

// getFBW2: channel barrier at s relative to s = 25 GeV^2.
__host__ __device__ __forceinline__ double channel_barrier(double M2, double m1, double m2, int L, double ffb) {
  if (L == 0) return 1.0;
  const double p2 = (M2 - sq(m1 + m2)) * (M2 - sq(m1 - m2)) / M2 / 4.0;
  const double p20 = (25.0 - sq(m1 + m2)) * (25.0 - sq(m1 - m2)) / 25.0 / 4.0;
  const double z = ffb * ffb * p2, z0 = ffb * ffb * fabs(p20);
  double v = 1.0;
  if (L >= 1 && L <= 5) v = bw_poly(L, z0) / bw_poly(L, z);
  return ipow(p2 / p20, L) * v;
}

__host__ __device__ __forceinline__ cplx rho_real(double M2, double m1, double m2, int L, double ffb) {
  const double rho2 = (M2 - sq(m1 + m2)) * (M2 - sq(m1 - m2));
  const double rho = sqrt(fabs(rho2)) / M2 * channel_barrier(M2, m1, m2, L, ffb);
  return rho2 >= 0 ? mk(rho, 0) : mk(0, rho);
}

// Complex square root with the reference's branch rule (RooTDalitz/cuComplex.h:641-657):
// zero below 1e-6, imaginary part negated only when Im < 0 and |Im/Re| > 1e-3.
__host__ __device__ __forceinline__ cplx csqrt_branch(cplx x) {
  if (fabs(x.re) < PWA_F(0.000001f) && fabs(x.im) < PWA_F(0.000001f)) return mk(0, 0);
  const double radius = hypot(x.re, x.im);
  const double cosA = x.re / radius;
  double re = sqrt(radius * (cosA + 1.0) / 2.0);
  double im = sqrt(radius * (1.0 - cosA) / 2.0);
  if (signbit(x.im) && fabs(x.im / x.re) > PWA_F(0.001f)) im = -im;
  return mk(re, im);
}

// Phase space with complex (width-carrying) masses; the channel barrier is 1 there.
__host__ __device__ __forceinline__ cplx rho_complex(double M2, cplx m1, cplx m2) {
  const cplx a = m1 + m2, b = m1 - m2;
  const cplx part1 = a * a - mk(M2, 0), part2 = b * b - mk(M2, 0);
  const cplx r = csqrt_branch(part1 * part2);
  return r * (1.0 / M2);
}

__host__ __device__ __forceinline__ cplx breit_wigner(double m, double gamma, double e2) {
  const double de2 = m * m - e2, gm = gamma * m, d = de2 * de2 + gm * gm;
  return mk(de2 / d, gm / d);
}

__host__ __device__ __forceinline__ double bw_norm(double m_r, double gamma_r) {
  const double kr = sqrt(m_r * m_r + gamma_r * gamma_r);
  return BW_NORM_C * m_r * sqrt(gamma_r * kr / sqrt(m_r * (m_r + kr)));
}

// Effective resonance mass for out-of-range masses (tanh mapping into [mmin, mmax]).
__host__ __device__ __forceinline__ double tanh_eff_mass(double m, double mmin, double mmax) {
  return mmin + 0.5 * (mmax - mmin) * (1.0 + tanh((m - (mmin + mmax) / 2.0) / (mmax - mmin)));
}

// --------------------------------------------------------------------- K-matrix
constexpr int NKMC = 4;
constexpr int NPMAX = 4;

// First row of inv(S), S complex N x N row-major, by an unpivoted LU of S^T solved against e0
// (RooTDalitz/cuSolve4x4.h:278-353 for N = 4, solve_7x7 :463 for N = 7).
template <int N>
__host__ __device__ __forceinline__ void first_row_inverse(const cplx (&S)[N][N], cplx (&T)[N]) {
  // A = S^T: A[r][c] = S[c][r]
  cplx U[N][N], L[N][N], invU[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int c = 0; c < N; ++c) {
      if (c < i) continue;
      cplx u = S[c][i];
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (k < i) u -= L[i][k] * U[k][c];
      U[i][c] = u;
    }
    invU[i] = recip(U[i][i]);
#pragma unroll
    for (int r = 0; r < N; ++r) {
      if (r <= i) continue;
      cplx l = S[i][r];
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (k < i) l -= L[r][k] * U[k][i];
      L[r][i] = l * invU[i];
    }
  }
  cplx y[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    y[i] = (i == 0) ? mk(1, 0) : mk(0, 0);
#pragma unroll
    for (int j = 0; j < N; ++j)
      if (j < i) y[i] -= L[i][j] * y[j];
  }
#pragma unroll
  for (int i = N - 1; i >= 0; --i) {
    cplx x = y[i];
#pragma unroll
    for (int j = 0; j < N; ++j)
      if (j > i) x -= U[i][j] * T[j];
    T[i] = invU[i] * x;
  }
}
__host__ __device__ __forceinline__ void first_row_inverse4(const cplx (&S)[4][4], cplx (&T)[4]) {
  first_row_inverse<4>(S, T);
}

// Isospin-split channels of the 7-channel K-matrix (Isospin_KMatrix, cu_DPFPropogator.cu:384-586,
// the reference's ISOSPIN_SIGMACD build): charged and neutral D(*) and Sigma_c(*) masses, the
// Sigma_c(*) half-widths as complex masses, and the isospin factors sqrt(2/3), -sqrt(1/3) (floats).
constexpr double KMI_D0 = PWA_F(1.86484f), KMI_DST0 = PWA_F(2.00685f);
constexpr double KMI_SCP = PWA_F(2.45265f), KMI_SCSTP = PWA_F(2.5174f);
constexpr double KMI_SCP_HW = (double)(-2.3f / 1000.f / 2.f), KMI_SCSTP_HW = (double)(-17.2f / 1000.f / 2.f);
constexpr double KMI_DM = PWA_F(1.86966f), KMI_DSTM = PWA_F(2.01026f);
constexpr double KMI_SCPP = PWA_F(2.45397f), KMI_SCSTPP = PWA_F(2.51841f);
constexpr double KMI_SCPP_HW = (double)(-1.89f / 1000.f / 2.f), KMI_SCSTPP_HW = (double)(-14.78f / 1000.f / 2.f);
constexpr double KMI_ISO0 = PWA_F(0.816496580927726f), KMI_ISO1 = PWA_F(-0.5773502691896257f);

}  // namespace pwa
