// TEST INFRASTRUCTURE ONLY -- the FP64 CPU oracle for the unbinned amplitude likelihood.
//
// This file restates, in double precision and in plain scalar C++, the reference's GPU likelihood
// path (reference files src/kernel_calEva.cu and src/cu_DPFPropogator.cu).  It is used only by the
// tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, always as the checker; the
// product path never links or calls it.
//
// Inputs are exactly the reference's: the float SoA planes pp/pp1/pp2 (stride n_size), the float
// parameter block h_paraList, and the band counts.  Every float input and every float constant of
// the reference is promoted to double unchanged, so a difference between this oracle and a float
// implementation is arithmetic precision only.
//
// Parity is pinned against the reference's own code built for host cores (oracle/build_ref.py),
// see tests/test_oracle_vs_ref.py.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

using cd = std::complex<double>;

// A float literal of the reference promoted to double (the reference computes with floats).
constexpr double F(float x) { return (double)x; }

// Masses (cu_DPFPropogator.cu:11-14).
constexpr double M_LB = F(5.61951f);
constexpr double M_K = F(0.493677f);
constexpr double M_P = F(0.938272046f);
constexpr double M_JPSI = F(3.096916f);

// K-matrix channel masses, averaged isospin partners (cu_DPFPropogator.cu:590-595).
constexpr double KM_D = F(1.86719f);
constexpr double KM_DST = F(2.008555f);
constexpr double KM_SC = F(2.453435f);
constexpr double KM_SCST = F(2.517955f);
constexpr double KM_SC_HW = F(-0.00105f);
constexpr double KM_SCST_HW = F(-0.00800f);

// Resolution model (Resonances.h:56-58).
constexpr double MRES0 = F(-0.134064f);
constexpr double MRES1 = F(0.0599014f);
constexpr double MRES2 = F(-0.00655841f);

// Parameter table layout (Resonances.h:97-112).
constexpr int NSET = 6;
enum { P_MASS = 0, P_WIDTH, P_SPIN, P_LRESON, P_TYPE, P_PARITY };
enum { T_BREITWIGNER = 1, T_MODELINDEPENDENT = 3, T_TRIANGLE = 7, T_KMATRIX = 240, T_REVISEDKMATRIX = 360,
       T_NONRESONANT = 361 };
// Spline knots of the Lambda* and Pc model-independent waves (Resonances.h:5-6); a spline block holds
// the knots, then 4 coefficients per knot of the real part, then 4 of the imaginary part.
constexpr int NUMSP = 24;
constexpr int NUMSPZ = 11;
constexpr double M_CHIC1 = F(3.51067f);  // cu_DPFPropogator.cu:15
constexpr int NPMAX = 4;
constexpr int NKMC = 4;

// Offsets of the reference smearing schemes (Resonances.h:31-54); the values are data of the
// reference (rounded normal quantiles, not all symmetric) and are reproduced exactly.
const float kSmear30[30] = {-2.128f, -1.645f, -1.383f, -1.192f, -1.036f, -0.903f, -0.783f, -0.674f,
                            -0.573f, -0.477f, -0.385f, -0.297f, -0.210f, -0.126f, -0.042f, 0.042f,
                            0.126f,  0.210f,  0.297f,  0.385f,  0.477f,  0.573f,  0.675f,  0.784f,
                            0.903f,  1.037f,  1.192f,  1.383f,  1.645f,  2.128f};
const float kSmear20[20] = {-1.960f, -1.440f, -1.150f, -0.934f, -0.755f, -0.598f, -0.454f,
                            -0.319f, -0.189f, -0.063f, 0.063f,  0.189f,  0.319f,  0.454f,
                            0.598f,  0.755f,  0.935f,  1.150f,  1.440f,  1.960f};
const float kSmear150[150] = {
    -2.713f, -2.326f, -2.128f, -1.989f, -1.881f, -1.791f, -1.713f, -1.645f, -1.583f, -1.527f,
    -1.476f, -1.428f, -1.383f, -1.341f, -1.301f, -1.263f, -1.226f, -1.192f, -1.158f, -1.126f,
    -1.095f, -1.065f, -1.036f, -1.008f, -0.981f, -0.954f, -0.928f, -0.903f, -0.878f, -0.854f,
    -0.830f, -0.806f, -0.783f, -0.761f, -0.739f, -0.717f, -0.696f, -0.674f, -0.654f, -0.633f,
    -0.613f, -0.593f, -0.573f, -0.553f, -0.534f, -0.515f, -0.496f, -0.477f, -0.458f, -0.440f,
    -0.421f, -0.403f, -0.385f, -0.367f, -0.349f, -0.332f, -0.314f, -0.297f, -0.279f, -0.262f,
    -0.245f, -0.227f, -0.210f, -0.193f, -0.176f, -0.160f, -0.142f, -0.126f, -0.109f, -0.092f,
    -0.075f, -0.058f, -0.042f, -0.025f, -0.008f, 0.008f, 0.025f, 0.042f, 0.059f, 0.075f,
    0.092f, 0.109f, 0.126f, 0.143f, 0.160f, 0.176f, 0.193f, 0.210f, 0.228f, 0.245f,
    0.262f, 0.279f, 0.297f, 0.314f, 0.332f, 0.350f, 0.367f, 0.385f, 0.403f, 0.422f,
    0.440f, 0.458f, 0.477f, 0.496f, 0.515f, 0.534f, 0.553f, 0.573f, 0.593f, 0.613f,
    0.633f, 0.654f, 0.675f, 0.696f, 0.717f, 0.739f, 0.761f, 0.784f, 0.806f, 0.830f,
    0.854f, 0.878f, 0.903f, 0.928f, 0.954f, 0.981f, 1.008f, 1.037f, 1.066f, 1.096f,
    1.126f, 1.159f, 1.192f, 1.226f, 1.263f, 1.301f, 1.341f, 1.383f, 1.428f, 1.476f,
    1.527f, 1.583f, 1.645f, 1.713f, 1.791f, 1.881f, 1.989f, 2.128f, 2.326f, 2.713f,
};

inline double sq(double x) { return x * x; }

// ---------------------------------------------------------------- kinematics (cu_DPFPropogator.cu:33-153)
double two_body_p(double M, double m1, double m2) {  // getp
  const double M2 = M * M;
  return std::sqrt(std::fabs((M2 - sq(m1 + m2)) * (M2 - sq(m1 - m2)))) / 2.0 / M;
}

double bw_poly(int L, double z) {
  switch (L) {
    case 1: return 1.0 + z;
    case 2: return z * z + 3.0 * z + 9.0;
    case 3: return z * z * z + 6.0 * z * z + 45.0 * z + 225.0;
    case 4: return std::pow(z, 4) + 10.0 * std::pow(z, 3) + 135.0 * z * z + 1575.0 * z + 11025.0;
    case 5:
      return std::pow(z, 5) + 15.0 * std::pow(z, 4) + 315.0 * std::pow(z, 3) + 6300.0 * z * z +
             99225.0 * z + 893025.0;
  }
  return 1.0;
}

// Blatt-Weisskopf ratio F_L(p)/F_L(p0) (F_BW, cu_DPFPropogator.cu:69-97).
double barrier_ratio(double r, int L, double p, double p0) {
  if (L < 1 || L > 5) return 1.0;
  const double z = sq(r * p), z0 = sq(r * p0);
  return std::sqrt(bw_poly(L, z0) / bw_poly(L, z));
}

// Squared ratio with z from p^2 directly (F_BW2, cu_DPFPropogator.cu:99-127).
double barrier_ratio2(double r, int L, double p2, double p20) {
  if (L < 1 || L > 5) return 1.0;
  const double z = r * r * p2, z0 = r * r * std::fabs(p20);
  return bw_poly(L, z0) / bw_poly(L, z);
}

double channel_barrier(double M2, double m1, double m2, int L, double ffb) {  // getFBW2
  if (L == 0) return 1.0;
  const double p2 = (M2 - sq(m1 + m2)) * (M2 - sq(m1 - m2)) / M2 / 4.0;
  const double M20 = 25.0;
  const double p20 = (M20 - sq(m1 + m2)) * (M20 - sq(m1 - m2)) / M20 / 4.0;
  return std::pow(p2 / p20, L) * barrier_ratio2(ffb, L, p2, p20);
}

cd rho_real(double M2, double m1, double m2, int L, double ffb) {  // getrho
  const double rho2 = (M2 - sq(m1 + m2)) * (M2 - sq(m1 - m2));
  const double rho = std::sqrt(std::fabs(rho2)) / M2 * channel_barrier(M2, m1, m2, L, ffb);
  return rho2 >= 0 ? cd(rho, 0) : cd(0, rho);
}

// The reference's own complex square root (RooTDalitz/cuComplex.h:641-657): zero for tiny inputs,
// and the imaginary part takes the input's sign only when |Im/Re| > 1e-3.
cd csqrt_branch(cd x) {
  if (std::fabs(x.real()) < F(0.000001f) && std::fabs(x.imag()) < F(0.000001f)) return cd(0, 0);
  const double radius = std::abs(x);
  const double cosA = x.real() / radius;
  double re = std::sqrt(radius * (cosA + 1.0) / 2.0);
  double im = std::sqrt(radius * (1.0 - cosA) / 2.0);
  if (std::signbit(x.imag()) && std::fabs(x.imag() / x.real()) > F(0.001f)) im = -im;
  return cd(re, im);
}

cd rho_complex(double M2, cd m1, cd m2) {  // getrho_complexMass (barrier factor is 1 there)
  const cd part1 = (m1 + m2) * (m1 + m2) - M2;
  const cd part2 = (m1 - m2) * (m1 - m2) - M2;
  return csqrt_branch(part1 * part2) * (1.0 / M2);
}

// ---------------------------------------------------------------- production barriers (cu_DPFPropogator.cu:155-217)
double barrier_lb_lstar(double J, double mpp, double mr, double ffb) {  // BTerm
  const int LB = (J <= 1) ? 0 : (int)(J - 1.5);
  const double pB = two_body_p(M_LB, M_JPSI, mpp);
  double pB0 = pB;
  const double mmin = M_K + M_P, mmax = M_LB - M_JPSI;
  if (mr < 0) pB0 = two_body_p(M_LB, M_JPSI, (mmin + mmax) / 2.0);
  if (mr > 1e-10 && mr + M_JPSI < M_LB) pB0 = two_body_p(M_LB, M_JPSI, mr);
  if (mr + M_JPSI > M_LB) {
    const double mreff =
        mmin + 0.5 * (mmax - mmin) * (1.0 + std::tanh((mr - (mmin + mmax) / 2.0) / (mmax - mmin)));
    pB0 = two_body_p(M_LB, M_JPSI, mreff);
  }
  return barrier_ratio(ffb, LB, pB, pB0) * std::pow(pB / M_LB, LB) * std::pow(M_LB / pB0, LB);
}

double barrier_lb_pc(double J, double mpp, double mr, double ffb) {  // BTermZ
  const int LB = (int)(J - 0.5);
  const double pB = two_body_p(M_LB, M_K, mpp);
  double pB0 = pB;
  if (mr < 0) pB0 = two_body_p(M_LB, M_K, (M_JPSI + M_P + M_LB - M_K) / 2.0);
  if (mr > 1e-10 && mr + M_K < M_LB) pB0 = two_body_p(M_LB, M_K, mr);
  return barrier_ratio(ffb, LB, pB, pB0) * std::pow(pB / M_LB, LB);
}

double barrier_lb_x(double J, double mpp, double mr, double ffb) {  // BTermX (cu_DPFPropogator.cu:205-217)
  const int LB = (int)(J - 0.5);  // C truncation toward zero
  const double pB = two_body_p(M_LB, M_P, mpp);
  double pB0 = pB;
  if (mr < 0) return std::pow(pB / M_LB, LB);
  if (mr > 1e-10 && mr + M_P < M_LB) pB0 = two_body_p(M_LB, M_P, mr);
  return barrier_ratio(ffb, LB, pB, pB0) * std::pow(pB / M_LB, LB);
}

// ---------------------------------------------------------------- Breit-Wigners (cu_DPFPropogator.cu:219-336)
cd breit_wigner(double m, double gamma, double e2) {
  const double de2 = m * m - e2, gm = gamma * m, d = de2 * de2 + gm * gm;
  return cd(de2 / d, gm / d);
}

double bw_norm(double m_r, double gamma_r) {
  const double kr = std::sqrt(m_r * m_r + gamma_r * gamma_r);
  return F(0.948850f) * m_r * std::sqrt(gamma_r * kr / std::sqrt(m_r * (m_r + kr)));
}

cd bw_lstar(double m_r, double gamma_r, double mpp, int LR, double ffr) {  // BW_AMP
  const double pR = two_body_p(mpp, M_P, M_K);
  double pR0 = pR;
  const double mmin = M_K + M_P, mmax = M_LB - M_JPSI;
  const double thr = F(M_P + M_K);  // float sum in the reference
  if (m_r < 0) pR0 = two_body_p((mmin + mmax) / 2.0, M_P, M_K);
  if (m_r > thr) pR0 = two_body_p(m_r, M_P, M_K);
  if (m_r <= thr && m_r > 1e-10) {
    const double mreff =
        mmin + 0.5 * (mmax - mmin) * (1.0 + std::tanh((m_r - (mmin + mmax) / 2.0) / (mmax - mmin)));
    pR0 = two_body_p(mreff, M_P, M_K);
  }
  double FR = barrier_ratio(ffr, LR, pR, pR0);
  if (m_r < 0) return cd(std::pow(pR / pR0, LR), 0);
  double gamma = gamma_r;
  if (m_r > thr) {
    gamma = gamma_r * std::pow(pR / pR0, 2 * LR + 1) * (m_r / mpp) * FR * FR;
  } else if (m_r < F(1.43f) && m_r > 0) {
    const double msig = F(1.18937f), mpi0 = F(0.13957018f);
    const double pSP = two_body_p(mpp, msig, mpi0);
    pR0 = two_body_p(m_r, msig, mpi0);
    FR = 1.0;
    gamma = gamma_r * std::pow(pR / pR0, 2 * LR + 1) * (m_r / mpp);
    gamma += F(0.0505f) * std::pow(pSP / pR0, 2 * LR + 1) * (m_r / mpp);
  }
  const double factor = FR * std::pow(pR / pR0, LR) * bw_norm(m_r, gamma_r);
  return factor * breit_wigner(m_r, gamma, mpp * mpp);
}

cd bw_pc(double m_r, double gamma_r, double mpp, int LR, double ffr) {  // BW_AMPZ
  const double pR = two_body_p(mpp, M_P, M_JPSI);
  double pR0 = pR;
  const double thr = F(M_P + M_JPSI);
  if (m_r > thr) pR0 = two_body_p(m_r, M_P, M_JPSI);
  const double FR = barrier_ratio(ffr, LR, pR, pR0);
  double gamma = gamma_r;
  if (m_r > thr) gamma = gamma_r * std::pow(pR / pR0, 2 * LR + 1) * (m_r / mpp) * FR * FR;
  const double factor = FR * std::pow(pR / pR0, LR) * bw_norm(m_r, gamma_r);
  return factor * breit_wigner(m_r, gamma, mpp * mpp);
}

cd bw_x(double m_r, double gamma_r, double mpp, int LR, double ffr) {  // BW_AMPX (cu_DPFPropogator.cu:226-246)
  const double pR = two_body_p(mpp, M_K, M_JPSI);
  double pR0 = pR;
  const double thr = F(M_K + M_JPSI);
  if (m_r > thr) pR0 = two_body_p(m_r, M_K, M_JPSI);
  const double FR = barrier_ratio(ffr, LR, pR, pR0);
  double gamma = gamma_r;
  if (m_r > thr) gamma = gamma_r * std::pow(pR / pR0, 2 * LR + 1) * (m_r / mpp) * FR * FR;
  const double factor = FR * std::pow(pR / pR0, LR) * bw_norm(m_r, gamma_r);
  return factor * breit_wigner(m_r, gamma, mpp * mpp);
}

// ---------------------------------------------------------------- spline waves (cu_DPFPropogator.cu:1118-1221)
// Piecewise cubic in (x - knot) from a spline block: knots poly[0 .. n), real-part coefficients
// poly[n + 4k ..], imaginary-part coefficients poly[5n + 4k ..]; zero outside [xmin, xmax]; the
// interval is found by the reference's bisection over the knots (ModelIndependentWave3 for the
// Lambda* chain with n = NUMSP, ModelIndependentWave for the Pc chain with n = NUMSPZ).
cd spline_wave(const float* poly, int n, double xmin, double xmax, double x) {
  if (x < xmin || x > xmax) return cd(0, 0);
  int klow = 0, khig = n - 1;
  if (x <= xmin) {
    klow = 0;
  } else if (x >= xmax) {
    klow = khig;
  } else {
    while (khig - klow > 1) {
      const int khalf = (klow + khig) / 2;
      if (x > poly[khalf])
        klow = khalf;
      else
        khig = khalf;
    }
  }
  const double dx = x - poly[klow];
  const float* a = poly + n + 4 * klow;
  const float* b = a + 4 * n;
  return cd(a[0] + dx * (a[1] + dx * (a[2] + dx * a[3])), b[0] + dx * (b[1] + dx * (b[2] + dx * b[3])));
}
// Domains: float sums of the reference (m_p + m_k - 0.002f etc.).
const double SPL_LSTAR_LO = (double)(0.938272046f + 0.493677f - 0.002f);
const double SPL_LSTAR_HI = (double)(5.61951f - 3.096916f + 0.002f);
const double SPL_PC_LO = (double)(0.938272046f + 3.096916f - 0.002f);
const double SPL_PC_HI = F(4.6f);

// ---------------------------------------------------------------- revised K-matrix (cu_DPFPropogator.cu:825-1115)
// Effective mass of a resonance for its reference momentum (the tanh map below threshold, the
// midpoint for non-resonant entries).
double eff_mass(double m_r, double thr, double mmax) {
  if (m_r > thr) return m_r;
  if (m_r >= 0) return thr + 0.5 * (mmax - thr) * (1.0 + std::tanh((m_r - (thr + mmax) / 2.0) / (mmax - thr)));
  return (thr + mmax) / 2.0;
}

// KMatrixTerm: the term of another entry of the same J^P (always with the p K masses, whichever
// chain calls it).  The first non-resonant entry (m_r < 0) fixes fsc, which every later one returns.
double kmatrix_term(double m_r, double gamma_r, double mpp, int LR, double& fsc, double ffr) {
  const double s = mpp * mpp;
  const double pR = two_body_p(mpp, M_P, M_K);
  const double pR0 = two_body_p(eff_mass(m_r, M_P + M_K, M_LB - M_JPSI), M_P, M_K);
  const double FR = barrier_ratio(ffr, LR, pR, pR0);
  const double gamma = gamma_r * std::pow(pR / pR0, 2 * LR + 1) * (m_r / mpp) * FR * FR;
  if (m_r < 0) {
    if (std::fabs(fsc) < 1e-10) fsc = gamma;
    return fsc;
  }
  if (std::fabs(m_r * m_r - s) < 1e-10) return 0;
  return m_r * gamma / (m_r * m_r - s);
}

struct Entry {
  double m, g;
  int S2, LR, type, P;
};
inline Entry entry(const float* pl, int r) {
  const float* q = pl + r * NSET;
  return Entry{q[P_MASS], q[P_WIDTH], (int)q[P_SPIN], (int)q[P_LRESON], (int)q[P_TYPE], (int)q[P_PARITY]};
}

// Revised_KMAMP: entry nr coupled to the entries [irst, ired) of its type, spin and parity.
cd revised_km(const float* pl, double mpp, int nr, int irst, int ired, bool pc_chain, double ffr) {
  const double s = mpp * mpp;
  const double m1 = pc_chain ? M_JPSI : M_P, m2 = pc_chain ? M_P : M_K, m3 = pc_chain ? M_K : M_JPSI;
  const Entry R = entry(pl, nr);
  double totG = 0, fsc = 0, denorm = 1;
  if (R.m > 0) denorm = R.m * R.m - s;
  for (int ir = irst; ir < ired; ++ir) {
    const Entry E = entry(pl, ir);
    if (E.type == R.type && E.S2 == R.S2 && E.P == R.P) {
      if (ir == nr) continue;
      totG += kmatrix_term(E.m, E.g, mpp, E.LR, fsc, ffr) * denorm;
    }
  }
  const double pR = two_body_p(mpp, m1, m2);
  double pR0 = two_body_p(eff_mass(R.m, m1 + m2, M_LB - m3), m1, m2);
  double FR = barrier_ratio(ffr, R.LR, pR, pR0);
  double factor = FR * std::pow(pR / pR0, R.LR);
  if (R.m > 0) {
    double gamma = R.g;
    if (R.m > m1 + m2) gamma = R.g * std::pow(pR / pR0, 2 * R.LR + 1) * (R.m / mpp) * FR * FR;
    if (R.m < m1 + m2) {  // the Sigma pi channel of the reference (written for the Lambda(1405))
      const double msig = F(1.18937f), mpi0 = F(0.13957018f);
      const double pRSigPi = two_body_p(mpp, msig, mpi0);
      pR0 = two_body_p(R.m, msig, mpi0);
      FR = 1.0;
      gamma = R.g * std::pow(pR / pR0, 2 * R.LR + 1) * (R.m / mpp);
      const double sp = F(0.0505f) * std::pow(pRSigPi / pR0, 2 * R.LR + 1) * (R.m / mpp);
      gamma += sp;
      denorm -= fsc * sp * R.m;
    }
    totG += R.m * gamma;
    const double kr = std::sqrt(R.m * R.m + R.g * R.g);
    factor *= F(0.948850f) * R.m * std::sqrt(R.g * kr / std::sqrt(R.m * (R.m + kr)));
  } else {
    totG += R.g * std::pow(pR / pR0, 2 * R.LR + 1) * (R.m / mpp) * FR * FR;
  }
  const double d2 = denorm * denorm + totG * totG;
  return cd(denorm / d2, totG / d2) * factor;
}

// Revised_KMAMP_refactor (the form storeLineshapeLsKM evaluates): products of the other entries'
// (m_j^2 - s) instead of the per-term division.
cd revised_km_refactor(const float* pl, double mpp, int nr, int irst, int ired, bool pc_chain, double ffr) {
  const double s = mpp * mpp;
  const double m1 = pc_chain ? M_JPSI : M_P, m2 = pc_chain ? M_P : M_K, m3 = pc_chain ? M_K : M_JPSI;
  const Entry R = entry(pl, nr);
  auto prod_delta = [&](int ir, const Entry& X) {  // product_delta_S
    double pr = 1;
    for (int j = irst; j < ired; ++j) {
      if (j == ir) continue;
      const Entry E = entry(pl, j);
      if (E.type == X.type && E.S2 == X.S2 && E.P == X.P) pr *= E.m * E.m - s;
    }
    return pr;
  };
  double fsc = 0;
  const double pR = two_body_p(mpp, m1, m2);
  const double pR0 = two_body_p(eff_mass(R.m, m1 + m2, M_LB - m3), m1, m2);
  const double FR = barrier_ratio(ffr, R.LR, pR, pR0);
  const double gamma = R.g * std::pow(pR / pR0, 2 * R.LR + 1) * (R.m / mpp) * FR * FR;
  const double pds_r = prod_delta(nr, R);
  const double pds_all = pds_r * (R.m * R.m - s);
  double sum = pds_r * R.m * gamma;
  for (int ir = irst; ir < ired; ++ir) {
    if (ir == nr) continue;
    const Entry E = entry(pl, ir);
    if (E.S2 == R.S2 && E.P == R.P && E.type == R.type) {
      // m_gamma with the p K masses
      const double qR = two_body_p(mpp, M_P, M_K);
      const double qR0 = two_body_p(eff_mass(E.m, M_P + M_K, M_LB - M_JPSI), M_P, M_K);
      const double fr = barrier_ratio(ffr, E.LR, qR, qR0);
      const double g = E.g * std::pow(qR / qR0, 2 * E.LR + 1) * (E.m / mpp) * fr * fr;
      double mg;
      if (E.m < 0) {
        if (std::fabs(fsc) < 1e-10) fsc = g;
        mg = fsc * (E.m * E.m - mpp * mpp);
      } else {
        mg = E.m * g;
      }
      sum += mg * prod_delta(ir, E);
    }
  }
  const double den = pds_all * pds_all + sum * sum;
  const double kr = std::sqrt(R.m * R.m + R.g * R.g);
  const double factor = FR * std::pow(pR / pR0, R.LR) * F(0.948850f) * R.m * std::sqrt(R.g * kr / std::sqrt(R.m * (R.m + kr)));
  return cd(pds_r * pds_all / den, pds_r * sum / den) * factor;
}

// ---------------------------------------------------------------- triangle cusp (cu_DPFPropogator.cu:1223-1343)
// The reference's complex logarithm and arctangent (RooTDalitz/cuComplex.h:660-676): the argument
// from acos(Re / |z|), negative for Im < 0; atan(z) = -i/2 log((1 + i z) / (1 - i z)).
cd clog_ref(cd x) {
  const double r = std::sqrt(x.real() * x.real() + x.imag() * x.imag());
  double th = std::acos(std::min(1.0, std::max(-1.0, x.real() / r)));  // clamped against rounding
  if (x.imag() < 0) th = -th;
  return cd(std::log(r), th);
}
// complex division as a / b = a conj(b) / |b|^2 (the reference's own algorithm scales instead; the
// two agree to rounding, and this form is the one the device code uses)
cd cdiv(cd a, cd b) {
  const double d = 1.0 / (b.real() * b.real() + b.imag() * b.imag());
  return cd((a.real() * b.real() + a.imag() * b.imag()) * d, (a.imag() * b.real() - a.real() * b.imag()) * d);
}
cd catan_ref(cd x) {
  const cd ii(0, 1);
  return -0.5 * (ii * clog_ref(cdiv(1.0 + ii * x, 1.0 - ii * x)));
}

cd cusp_amp(double m_r, double gamma, double mpp) {  // GetCusp_AMP
  const cd ii(0, 1);
  const double p12 = M_LB, p13 = M_K;
  const cd m1(m_r, -gamma / 2.0);
  const double m2 = M_CHIC1, m3 = M_P;
  const double p23 = mpp;
  cd integral(0, 0);
  const int bins = 100;
  const double dx = F(1.f / bins);
  for (int i = 0; i < bins; ++i) {
    const double alpha = (double)((float)i * (float)dx + (float)dx / 2.0f);
    const cd b = (alpha * (p12 * p12 - p13 * p13 - p23 * p23) + m3 * m3 - m2 * m2) / p23 / p23 + 1.0 - 0.001 * ii;
    const cd c = (alpha * (m1 * m1 - m3 * m3) + m3 * m3 - alpha * (1.0 - alpha) * p13 * p13) / (p23 * p23);
    const cd sv = csqrt_branch(4.0 * c - b * b);
    const cd t1 = catan_ref(cdiv(b, sv));
    const cd t2 = catan_ref(cdiv(b + 2.0 * (alpha - 1.0), sv));
    integral += dx * cdiv(t1 - t2, sv);
  }
  return integral * (1.0 / mpp / mpp);
}

// ---------------------------------------------------------------- K-matrix (cu_DPFPropogator.cu:588-813)
// First row of the inverse of a complex n x n matrix S, via an unpivoted LU of S^T with b = e0
// (RooTDalitz/cuSolve4x4.h:278-353 uses this construction).
void first_row_of_inverse(const cd* S, int n, cd* out) {
  std::vector<cd> A(n * n), L(n * n, cd(0, 0)), U(n * n, cd(0, 0)), invU(n);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) A[r * n + c] = S[c * n + r];
  for (int i = 0; i < n; ++i) {
    for (int c = i; c < n; ++c) {
      cd u = A[i * n + c];
      for (int k = 0; k < i; ++k) u -= L[i * n + k] * U[k * n + c];
      U[i * n + c] = u;
    }
    invU[i] = 1.0 / U[i * n + i];
    for (int r = i + 1; r < n; ++r) {
      cd l = A[r * n + i];
      for (int k = 0; k < i; ++k) l -= L[r * n + k] * U[k * n + i];
      L[r * n + i] = l * invU[i];
    }
  }
  std::vector<cd> y(n);
  for (int i = 0; i < n; ++i) {
    y[i] = (i == 0) ? cd(1, 0) : cd(0, 0);
    for (int j = 0; j < i; ++j) y[i] -= L[i * n + j] * y[j];
  }
  for (int i = n - 1; i >= 0; --i) {
    cd x = y[i];
    for (int j = i + 1; j < n; ++j) x -= U[i * n + j] * out[j];
    out[i] = invU[i] * x;
  }
}

struct Model {
  const float* pl = nullptr;
  int para_size = 0, vamp_size = 0, spline_size = 0;
  int NR = 0, NZ = 0, NX = 0;
  double FFR = 3, FFB = 3;
  int kmcount = 0;
  std::vector<int> ampcount;  // first coupling index of each resonance
  std::vector<int> ikmslot;   // K-matrix output slot of each Pc entry
  std::vector<int> splcount;  // first float of each resonance's spline block
  bool swap_coupling_parts = false;
};

// Coupling offsets (kernel_calEva.cu:1014-1098) and K-matrix output slots (:978-1010).
void configure(Model& m) {
  const float* pl = m.pl;
  int cnt = m.para_size;
  m.ampcount.assign(m.NR + m.NZ + m.NX, 0);
  for (int r = 0; r < m.NR; ++r) {
    m.ampcount[r] = cnt;
    const int S2 = (int)pl[r * NSET + P_SPIN];
    cnt += 2 * ((S2 == 1) ? 8 : 12);
  }
  for (int i = 0; i < m.NZ; ++i) {
    const int r = m.NR + i;
    m.ampcount[r] = cnt;
    const double S = (int)pl[r * NSET + P_SPIN] / 2.0;
    for (int k = 0; k < 2; ++k)
      for (int hpsi = -1; hpsi <= 1; ++hpsi)
        for (int ihz = 0; ihz < 2; ++ihz)
          for (int ihp = 0; ihp < 2; ++ihp)
            if (!(std::fabs(hpsi - (ihp ? 0.5 : -0.5)) > S)) cnt += 2;
  }
  for (int i = 0; i < m.NX; ++i) {
    const int r = m.NR + m.NZ + i;
    m.ampcount[r] = cnt;
    const double S = (int)pl[r * NSET + P_SPIN] / 2.0;
    for (int k = 0; k < 2; ++k)
      for (int hpsi = -1; hpsi <= 1; ++hpsi) {
        if (std::abs(hpsi) > S) continue;
        for (int ihp = 0; ihp < 2; ++ihp) {
          const double hp = ihp ? 0.5 : -0.5;
          for (int ihz = 0; ihz < 2; ++ihz) {
            const double hz = ihz ? hp + 0.5 : hp - 0.5;
            if (std::fabs(hz) > S) continue;
            cnt += 2;
          }
        }
      }
  }
  int per_group[4] = {0, 0, 0, 0};
  m.ikmslot.assign(m.NZ, 0);
  for (int i = 0; i < m.NZ; ++i) {
    const int r = m.NR + i;
    const int S2 = (int)pl[r * NSET + P_SPIN], LR = (int)pl[r * NSET + P_LRESON];
    if ((int)pl[r * NSET + P_TYPE] == T_KMATRIX) {
      const int ik = (LR > 0) ? ((S2 == 3) ? 3 : 2) : ((S2 == 3) ? 1 : 0);
      m.ikmslot[i] = per_group[ik]++;
    }
  }
  m.kmcount = m.para_size + m.vamp_size + m.spline_size;
  // spline blocks follow the couplings (cuda_configure_splcount, kernel_calEva.cu:1100-1135)
  m.splcount.assign(m.NR + m.NZ, 0);
  int sc = m.para_size + m.vamp_size;
  for (int r = 0; r < m.NR + m.NZ; ++r) {
    m.splcount[r] = sc;
    if ((int)pl[r * NSET + P_TYPE] == T_MODELINDEPENDENT) sc += 9 * (r < m.NR ? NUMSP : NUMSPZ);
  }
}

// The reference's ISOSPIN_SIGMACD build (RooTDalitz/Resonances.h:17, compile-time there) replaces the
// 4-channel K-matrix by Isospin_KMatrix; a run-time switch here (oracle_set_kmatrix_isospin).
static bool g_kmatrix_isospin = false;

// Isospin_KMatrix (cu_DPFPropogator.cu:384-586): 7 channels -- J/psi p and the charged (D- / D*-
// with Sigma_c++ / Sigma_c*++) and neutral (D0 / D*0 with Sigma_c+ / Sigma_c*+) partners of the three
// Sigma_c(*) D(*) channels -- with the 4 x 4 couplings and scattering terms spread by the isospin
// factors sqrt(2/3) (charged) and -sqrt(1/3) (neutral), the poles of channels 1 and 3 shifted by
// Re(i g^2 / 3 (2 rho_charged + rho_neutral)), a 7 x 7 first-row inverse, and its row folded back onto
// the 4 production channels.  Same outputs as kmatrix_group.
int kmatrix_group_isospin(const Model& md, double mpp, int J_r, int P_r, int ik, cd* Mtr) {
  constexpr double D0 = F(1.86484f), DST0 = F(2.00685f), SCP = F(2.45265f), SCSTP = F(2.5174f);
  constexpr double SCP_HW = (double)(-2.3f / 1000.f / 2.f), SCSTP_HW = (double)(-17.2f / 1000.f / 2.f);
  constexpr double DM = F(1.86966f), DSTM = F(2.01026f), SCPP = F(2.45397f), SCSTPP = F(2.51841f);
  constexpr double SCPP_HW = (double)(-1.89f / 1000.f / 2.f), SCSTPP_HW = (double)(-14.78f / 1000.f / 2.f);
  const double iso_f[2] = {F(0.816496580927726f), F(-0.5773502691896257f)};
  const float* pl = md.pl;
  const double ffb = md.FFB;
  const int Lna = (P_r == 1) ? 1 : 0;
  const double s = mpp * mpp;
  cd rho[7];
  rho[0] = rho_real(s, M_P, M_JPSI, Lna, ffb);
  if (J_r == 1 && P_r == -1) {
    rho[1] = rho_complex(s, cd(DSTM, 0), cd(SCPP, SCPP_HW));
    rho[2] = rho_complex(s, cd(DST0, 0), cd(SCP, SCP_HW));
    rho[3] = rho_complex(s, cd(DSTM, 0), cd(SCSTPP, SCSTPP_HW));
    rho[4] = rho_complex(s, cd(DST0, 0), cd(SCSTP, SCSTP_HW));
    rho[5] = rho_complex(s, cd(DM, 0), cd(SCPP, SCPP_HW));
    rho[6] = rho_complex(s, cd(D0, 0), cd(SCP, SCP_HW));
  } else if (J_r == 3 && P_r == -1) {
    rho[1] = rho_complex(s, cd(DSTM, 0), cd(SCPP, SCPP_HW));
    rho[2] = rho_complex(s, cd(DST0, 0), cd(SCP, SCP_HW));
    rho[3] = rho_complex(s, cd(DSTM, 0), cd(SCSTPP, SCSTPP_HW));
    rho[4] = rho_complex(s, cd(DST0, 0), cd(SCSTP, SCSTP_HW));
    rho[5] = rho_complex(s, cd(DM, 0), cd(SCSTPP, SCSTPP_HW));
    rho[6] = rho_complex(s, cd(D0, 0), cd(SCSTP, SCSTP_HW));
  } else if (P_r == 1) {
    rho[1] = rho_real(s, DSTM, SCPP, Lna, ffb);
    rho[2] = rho_real(s, DST0, SCP, Lna, ffb);
    rho[3] = rho_real(s, DM, SCPP, Lna, ffb);
    rho[4] = rho_real(s, D0, SCP, Lna, ffb);
    rho[5] = rho_real(s, DM, SCSTPP, Lna, ffb);
    rho[6] = rho_real(s, D0, SCSTP, Lna, ffb);
  } else {
    return -1;
  }
  const float* g_alpha = &pl[md.kmcount + ik * (NPMAX + NKMC) * NKMC];
  const float* f_scat = &pl[md.kmcount + NPMAX * NKMC + ik * (NPMAX + NKMC) * NKMC];
  int Npole = 0, ikm = 1;
  double ms[NPMAX + 1] = {1, 1, 1, 1, 1};
  for (int r = md.NR; r < md.NR + md.NZ; ++r) {
    const double mfit = pl[r * NSET + P_MASS];
    const int iChannel = (int)pl[r * NSET + P_WIDTH];
    const int S = (int)pl[r * NSET + P_SPIN];
    const int type = (int)pl[r * NSET + P_TYPE];
    const int parity = (int)pl[r * NSET + P_PARITY];
    if (!(type == T_KMATRIX && S == J_r && parity == P_r && mfit > 0)) continue;
    if (Npole >= NPMAX) return -2;
    double m0 = mfit;
    if (iChannel == 1 || iChannel == 3) {
      const double mfit2 = mfit * mfit;
      const cd ra = iChannel == 1 ? rho_complex(mfit2, cd(DSTM, 0), cd(SCPP, SCPP_HW))
                                  : rho_complex(mfit2, cd(DM, 0), cd(SCPP, SCPP_HW));
      const cd rb = iChannel == 1 ? rho_complex(mfit2, cd(DST0, 0), cd(SCP, SCP_HW))
                                  : rho_complex(mfit2, cd(D0, 0), cd(SCP, SCP_HW));
      const double g = g_alpha[Npole * NKMC + iChannel];
      const cd shift = cd(0, g * g / 3.0) * (2.0 * ra + rb);
      m0 = std::sqrt(mfit2 + shift.real());
    } else if (iChannel != 0) {
      return -3;  // the reference prints "An unacceptable channel" and uses an unset mass
    }
    double denorm = m0 * m0 - s;
    if (std::fabs(denorm) < F(1e-3f)) denorm = F(1e-3f);
    ++Npole;
    ms[0] *= denorm;
    for (int ip = 1; ip <= NPMAX; ++ip)
      if (ip != ikm) ms[ip] *= denorm;
    ++ikm;
  }
  double mg[NPMAX][NKMC], fs[NKMC][NKMC], kma[7][7];
  for (int i = 0; i < Npole; ++i)
    for (int j = 0; j < NKMC; ++j) mg[i][j] = g_alpha[i * NKMC + j] * ms[i + 1];
  for (int i = 0; i < NKMC; ++i)
    for (int j = 0; j < NKMC; ++j) fs[i][j] = f_scat[i * NKMC + j] * ms[0];
  for (int i = 0; i < 7; ++i) {
    const double fi = (i == 0) ? 1.0 : iso_f[(i + 1) % 2];
    const int ip = (i + 1) / 2;
    for (int j = i; j < 7; ++j) {
      const double fj = (j == 0) ? 1.0 : iso_f[(j + 1) % 2];
      const int jp = (j + 1) / 2;
      double v = fi * fj * fs[ip][jp];
      for (int k = 0; k < Npole; ++k) v += fi * fj * (double)g_alpha[k * NKMC + ip] * mg[k][jp];
      kma[i][j] = kma[j][i] = v;
    }
  }
  cd KK[49];
  for (int i = 0; i < 7; ++i)
    for (int j = 0; j < 7; ++j) {
      KK[i * 7 + j] = cd(0, -1) * (kma[i][j] * rho[j]);
      if (i == j) KK[i * 7 + j] += ms[0];
    }
  cd T7[7];
  first_row_of_inverse(KK, 7, T7);
  const cd T[NKMC] = {T7[0], iso_f[0] * T7[1] + iso_f[1] * T7[2], iso_f[0] * T7[3] + iso_f[1] * T7[4],
                      iso_f[0] * T7[5] + iso_f[1] * T7[6]};
  const double na = (Lna >= 1) ? channel_barrier(s, M_P, M_JPSI, Lna, ffb) : 1.0;
  for (int p = 0; p < Npole; ++p) {
    cd acc(0, 0);
    for (int i = 0; i < NKMC; ++i) acc += T[i] * mg[p][i];
    Mtr[p] = acc * na;
  }
  for (int i = 0; i < NKMC; ++i) Mtr[Npole + i] = T[i] * (ms[0] * na);
  return Npole + NKMC;
}

// One J^P group of the coupled-channel Pc K-matrix at invariant mass mpp.  Writes Npole + 4 P-vector
// outputs (poles first, then the four non-resonant production terms).
int kmatrix_group(const Model& md, double mpp, int J_r, int P_r, int ik, cd* Mtr) {
  if (g_kmatrix_isospin) return kmatrix_group_isospin(md, mpp, J_r, P_r, ik, Mtr);
  const float* pl = md.pl;
  const double ffb = md.FFB;
  const int Lna = (P_r == 1) ? 1 : 0;
  const double s = mpp * mpp;
  cd rho[NKMC];
  rho[0] = rho_real(s, M_P, M_JPSI, Lna, ffb);
  if (J_r == 1 && P_r == -1) {
    rho[1] = rho_complex(s, cd(KM_DST, 0), cd(KM_SC, KM_SC_HW));
    rho[3] = rho_complex(s, cd(KM_D, 0), cd(KM_SC, KM_SC_HW));
    rho[2] = rho_complex(s, cd(KM_DST, 0), cd(KM_SCST, KM_SCST_HW));
  } else if (J_r == 3 && P_r == -1) {
    rho[1] = rho_complex(s, cd(KM_DST, 0), cd(KM_SC, KM_SC_HW));
    rho[2] = rho_complex(s, cd(KM_DST, 0), cd(KM_SCST, KM_SCST_HW));
    rho[3] = rho_complex(s, cd(KM_D, 0), cd(KM_SCST, KM_SCST_HW));
  } else if (P_r == 1) {
    rho[1] = rho_real(s, KM_DST, KM_SC, Lna, ffb);
    rho[2] = rho_real(s, KM_D, KM_SC, Lna, ffb);
    rho[3] = rho_real(s, KM_D, KM_SCST, Lna, ffb);
  } else {
    return -1;  // channel phase space undefined in the reference for this J^P
  }
  const float* g_alpha = &pl[md.kmcount + ik * (NPMAX + NKMC) * NKMC];
  const float* f_scat = &pl[md.kmcount + NPMAX * NKMC + ik * (NPMAX + NKMC) * NKMC];
  int Npole = 0, ikm = 1;
  double ms[NPMAX + 1] = {1, 1, 1, 1, 1};
  for (int r = md.NR; r < md.NR + md.NZ; ++r) {
    const double mfit = pl[r * NSET + P_MASS];
    const int iChannel = (int)pl[r * NSET + P_WIDTH];
    const int S = (int)pl[r * NSET + P_SPIN];
    const int type = (int)pl[r * NSET + P_TYPE];
    const int parity = (int)pl[r * NSET + P_PARITY];
    if (!(type == T_KMATRIX && S == J_r && parity == P_r && mfit > 0)) continue;
    if (Npole >= NPMAX) return -2;
    double m0 = mfit;
    if (iChannel > 0) {
      const double mfit2 = mfit * mfit;
      cd rch;
      if (iChannel == 1)
        rch = rho_complex(mfit2, cd(KM_DST, 0), cd(KM_SC, KM_SC_HW));
      else if (iChannel == 2)
        rch = rho_complex(mfit2, cd(KM_D, 0), cd(KM_SCST, KM_SCST_HW));
      else if (iChannel == 3)
        rch = rho_complex(mfit2, cd(KM_D, 0), cd(KM_SC, KM_SC_HW));
      else
        return -3;
      const double g = g_alpha[Npole * NKMC + iChannel];
      const cd shift = cd(0, g * g) * rch;
      m0 = std::sqrt(mfit2 + shift.real());
    } else if (iChannel < 0) {
      return -3;
    }
    double denorm = m0 * m0 - s;
    if (std::fabs(denorm) < F(1e-3f)) denorm = F(1e-3f);
    ++Npole;
    ms[0] *= denorm;
    for (int ip = 1; ip <= NPMAX; ++ip)
      if (ip != ikm) ms[ip] *= denorm;
    ++ikm;
  }
  double mg[NPMAX][NKMC], fs[NKMC][NKMC], kma[NKMC][NKMC];
  for (int i = 0; i < Npole; ++i)
    for (int j = 0; j < NKMC; ++j) mg[i][j] = g_alpha[i * NKMC + j] * ms[i + 1];
  for (int i = 0; i < NKMC; ++i)
    for (int j = 0; j < NKMC; ++j) fs[i][j] = f_scat[i * NKMC + j] * ms[0];
  for (int i = 0; i < NKMC; ++i)
    for (int j = i; j < NKMC; ++j) {
      double v = fs[i][j];
      for (int k = 0; k < Npole; ++k) v += (double)g_alpha[k * NKMC + i] * mg[k][j];
      kma[i][j] = kma[j][i] = v;
    }
  cd KK[NKMC * NKMC];
  for (int i = 0; i < NKMC; ++i)
    for (int j = 0; j < NKMC; ++j) {
      KK[i * NKMC + j] = cd(0, -1) * (kma[i][j] * rho[j]);
      if (i == j) KK[i * NKMC + j] += ms[0];
    }
  cd T[NKMC];
  first_row_of_inverse(KK, NKMC, T);
  const double na = (Lna >= 1) ? channel_barrier(s, M_P, M_JPSI, Lna, ffb) : 1.0;
  for (int ip = 0; ip < Npole; ++ip) {
    cd acc(0, 0);
    for (int i = 0; i < NKMC; ++i) acc += T[i] * mg[ip][i];
    Mtr[ip] = acc * na;
  }
  for (int i = 0; i < NKMC; ++i) Mtr[Npole + i] = T[i] * (ms[0] * na);
  return Npole + NKMC;
}

// ---------------------------------------------------------------- per-event amplitudes (kernel_calEva.cu:85-811)
struct Ev {
  const float *pp, *pp1, *pp2;
  long n;  // plane stride
  long i;  // event index
  const float *pp3 = nullptr, *pp4 = nullptr;  // Zcs chain planes (NX > 0)
  double p0(int plane) const { return pp[i + plane * n]; }
  double p1(int plane) const { return pp1[i + plane * n]; }
  double p2(int plane) const { return pp2[i + plane * n]; }
  double p3(int plane) const { return pp3[i + plane * n]; }
  double p4(int plane) const { return pp4[i + plane * n]; }
};

inline cd read_coupling(const Model& md, int& cnt) {
  const double a = md.pl[cnt], b = md.pl[cnt + 1];
  cnt += 2;
  return md.swap_coupling_parts ? cd(b, a) : cd(a, b);
}

inline int pc_group(int S2, int LR) { return (LR > 0) ? ((S2 == 3) ? 3 : 2) : ((S2 == 3) ? 1 : 0); }

// Lambda* chain contribution to the 8 helicity amplitudes H[4*dmu + 2*lb + p] (GetAmpLz).
bool amp_lstar(const Model& md, const Ev& e, cd* H) {
  const double mkp = e.p0(0);
  for (int r = 0; r < md.NR; ++r) {
    const float* q = &md.pl[r * NSET];
    double m0 = q[P_MASS];
    const double g0 = q[P_WIDTH];
    const int S2 = (int)q[P_SPIN], LR = (int)q[P_LRESON], type = (int)q[P_TYPE];
    const double S = 0.5 * S2;
    cd bw(0, 0);
    if (type == T_BREITWIGNER) {
      bw = bw_lstar(m0, g0, mkp, LR, md.FFR);
    } else if (type == T_NONRESONANT) {
      bw = cd(1, 0);
    } else if (type == T_MODELINDEPENDENT) {
      bw = spline_wave(md.pl + md.splcount[r], NUMSP, SPL_LSTAR_LO, SPL_LSTAR_HI, mkp);
      m0 = -0.5;  // the production barrier of a spline wave is the non-resonant one
    } else if (type == T_REVISEDKMATRIX) {
      bw = revised_km(md.pl, mkp, r, 0, md.NR, false, md.FFR);
    } else {
      return false;
    }
    bw *= barrier_lb_lstar(S, mkp, m0, md.FFB);
    int cnt = md.ampcount[r];
    const int s = (S2 - 1) / 2;
    for (int k = 0; k < 2; ++k)
      for (int m = 0; m < 6; ++m) {
        if (S2 == 1 && m >= 4) continue;
        const cd c = read_coupling(md, cnt);
        if (std::abs(c) < 1e-10) continue;
        const double dl = e.p0(51 + s * 12 + k * 6 + m);
        for (int i = 0; i < 2; ++i)
          for (int j = 0; j < 2; ++j) {
            const int a = 3 + (i * 12 + j * 6 + m) * 2;
            const cd A(e.p0(a), e.p0(a + 1));
            H[4 * i + 2 * j + k] += dl * (A * bw) * c;
          }
      }
  }
  return true;
}

// Zcs chain contribution to H[8] (GetAmpZcs, kernel_calEva.cu:192-286), reproducing how that kernel
// walks the couplings: per proton helicity it reads consecutive couplings for (lambda_psi in -1..1,
// lambda_p in {0, 1}, lambda_Zcs = lambda_p -+ 1/2) with |lambda_psi|, |lambda_Zcs| <= J, and the
// running index m of those combinations selects the AX / DX planes.  (ConfigureCouplings wrote the
// couplings for lambda_p = -+1/2 instead; the kernel's reading is what enters the likelihood.)
void amp_zcs(const Model& md, const Ev& e, cd* H) {
  const double mjk = e.p3(0);
  for (int x = 0; x < md.NX; ++x) {
    const int r = md.NR + md.NZ + x;
    const float* q = &md.pl[r * NSET];
    const double m0 = q[P_MASS], g0 = q[P_WIDTH];
    const int S2 = (int)q[P_SPIN], LR = (int)q[P_LRESON];
    const double S = 0.5 * S2;
    const cd bw = barrier_lb_x(S, mjk, m0, md.FFB) * bw_x(m0, g0, mjk, LR, md.FFR);
    int cnt = md.ampcount[r];
    const int s = S2 / 2;
    for (int k = 0; k < 2; ++k) {
      int m = 0;
      for (int hpsi = -1; hpsi <= 1; ++hpsi) {
        if (std::fabs((double)hpsi) > S) continue;
        for (int hp = 0; hp <= 1; ++hp)
          for (int iz = 0; iz < 2; ++iz) {
            const double hz = hp - 0.5 + iz;
            if (std::fabs(hz) > S) continue;
            const cd c = read_coupling(md, cnt);
            if (std::abs(c) < 1e-10) {
              ++m;
              continue;
            }
            const double dx = e.p4(s * 24 + k * 12 + m);
            for (int i = 0; i < 2; ++i)
              for (int j = 0; j < 2; ++j) {
                const int a = 1 + (i * 24 + j * 12 + m) * 2;
                const cd A(e.p3(a), e.p3(a + 1));
                H[4 * i + 2 * j + k] += dx * (A * bw) * c;
              }
            ++m;
          }
      }
    }
  }
}

// Angular part of one Pc entry times its couplings (no lineshape), added into HZ[8].
void amp_pc_angular(const Model& md, const Ev& e, int iPc, cd scale, cd* HZ) {
  const int r = md.NR + iPc;
  const int S2 = (int)md.pl[r * NSET + P_SPIN];
  const double S = 0.5 * S2;
  int cnt = md.ampcount[r];
  const int s = (S2 - 1) / 2;
  for (int k = 0; k < 2; ++k) {
    int m = 0;
    for (int hpsi = -1; hpsi <= 1; ++hpsi)
      for (int ihz = 0; ihz < 2; ++ihz)
        for (int ihp = 0; ihp < 2; ++ihp) {
          const double hp = ihp ? 0.5 : -0.5;
          if (std::fabs(hpsi - hp) > S) { ++m; continue; }
          const cd c = read_coupling(md, cnt);
          if (std::abs(c) < 1e-10) { ++m; continue; }
          const double dz = e.p2(s * 24 + k * 12 + m);
          for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
              const int a = (i * 24 + j * 12 + m) * 2;
              const cd A(e.p1(a), e.p1(a + 1));
              HZ[4 * i + 2 * j + k] += dz * (A * scale) * c;
            }
          ++m;
        }
  }
}

// Lineshapes of all Pc entries at mass mz (K-matrix groups solved once each).  Returns false if a
// J^P group cannot be evaluated.
bool pc_lineshapes(const Model& md, double mz, double weight, cd* bw) {
  cd akm[4][NPMAX + NKMC];
  bool have[4] = {false, false, false, false};
  for (int i = 0; i < md.NZ; ++i) {
    const float* q = &md.pl[(md.NR + i) * NSET];
    double m0 = q[P_MASS];
    const double g0 = q[P_WIDTH];
    const int S2 = (int)q[P_SPIN], LR = (int)q[P_LRESON], type = (int)q[P_TYPE];
    cd b(0, 0);
    if (type == T_BREITWIGNER) {
      b = bw_pc(m0, g0, mz, LR, md.FFR);
    } else if (type == T_MODELINDEPENDENT) {
      b = spline_wave(md.pl + md.splcount[md.NR + i], NUMSPZ, SPL_PC_LO, SPL_PC_HI, mz);
      m0 = -0.5;
    } else if (type == T_REVISEDKMATRIX) {
      b = revised_km(md.pl, mz, md.NR + i, md.NR, md.NR + md.NZ, true, md.FFR);
    } else if (type == T_TRIANGLE) {
      b = cusp_amp(m0, g0, mz);
    } else if (type == T_KMATRIX) {
      const int ik = pc_group(S2, LR);
      if (!have[ik]) {
        if (kmatrix_group(md, mz, S2, (LR > 0) ? 1 : -1, ik, akm[ik]) < 0) return false;
        have[ik] = true;
      }
      b = akm[ik][md.ikmslot[i]];
    } else if (type == T_NONRESONANT) {
      b = cd(1, 0);
    } else {
      return false;
    }
    bw[i] = b * (barrier_lb_pc(0.5 * S2, mz, m0, md.FFB) * weight);
  }
  return true;
}

// Unsmeared |A|^2 (GetAmp2s): coherent sum, or the sum of the chains' separate |A|^2.
double amp2_unsmeared(const Model& md, const Ev& e, bool interference) {
  cd HL[8] = {}, HX[8] = {}, HZ[8] = {};
  if (!amp_lstar(md, e, HL)) return std::nan("");
  if (md.NX > 0) amp_zcs(md, e, HX);
  std::vector<cd> bw(std::max(md.NZ, 1));
  if (md.NZ > 0 && !pc_lineshapes(md, e.p0(1), 1.0, bw.data())) return std::nan("");
  for (int i = 0; i < md.NZ; ++i) amp_pc_angular(md, e, i, bw[i], HZ);
  double tot = 0;
  for (int h = 0; h < 8; ++h)
    tot += interference ? std::norm(HL[h] + HX[h] + HZ[h]) : std::norm(HL[h]) + std::norm(HX[h]) + std::norm(HZ[h]);
  return tot;
}

// Smeared |A|^2 (TemplateGetAmp2s): the Pc lineshapes are averaged over nbins mass offsets
// scheme[b]*mres(m), bilinearly in the amplitude.  The per-bin weight is the float 1/nbins and the
// Pc-Pc accumulator is rescaled by its float reciprocal, exactly as the reference does
// (kernel_calEva.cu:676,771-783), so the effective weights match to the last bit of the constants.
double amp2_smeared(const Model& md, const Ev& e, int nbins, const float* scheme) {
  cd HL[8] = {};  // Lambda* and Zcs (H_L_Zcs of the reference)
  if (!amp_lstar(md, e, HL)) return std::nan("");
  if (md.NX > 0) amp_zcs(md, e, HL);
  const int NZ = md.NZ;
  std::vector<cd> HZ(NZ * 8, cd(0, 0)), BW1(NZ, cd(0, 0)), BW2(NZ * NZ, cd(0, 0)), bw(std::max(NZ, 1));
  for (int i = 0; i < NZ; ++i) amp_pc_angular(md, e, i, cd(1, 0), &HZ[i * 8]);
  const double mz = e.p0(1);
  const double mres = MRES0 + mz * (MRES1 + mz * MRES2);
  const float wf = (float)(1.0 / nbins);
  const double w = wf;
  const double unscale = (double)(1.f / wf);
  for (int b = 0; b < nbins; ++b) {
    const double off = (double)scheme[b] * mres;
    if (NZ > 0 && !pc_lineshapes(md, mz + off, w, bw.data())) return std::nan("");
    for (int i = 0; i < NZ; ++i) {
      BW1[i] += bw[i];
      for (int j = 0; j < NZ; ++j) BW2[i * NZ + j] += bw[i] * std::conj(bw[j] * unscale);
    }
  }
  double tot = 0;
  for (int h = 0; h < 8; ++h) {
    tot += std::norm(HL[h]);
    for (int i = 0; i < NZ; ++i) {
      tot += 2.0 * (std::conj(HL[h]) * (BW1[i] * HZ[i * 8 + h])).real();
      for (int j = 0; j < NZ; ++j) tot += (BW2[i * NZ + j] * HZ[i * 8 + h] * std::conj(HZ[j * 8 + h])).real();
    }
  }
  return tot;
}

// Weighted grid smearing (fixed-width Gaussian on a mass grid; no counterpart in the reference):
// sum_b w_b |A(m + off_b)|^2 evaluated as that sum, helicity by helicity (independent of the
// expanded BW1/BW2-like form the kernels use).
double amp2_smeared_grid(const Model& md, const Ev& e, int nb, const double* off, const double* wt) {
  cd HL[8] = {};
  if (!amp_lstar(md, e, HL)) return std::nan("");
  if (md.NX > 0) amp_zcs(md, e, HL);
  const int NZ = md.NZ;
  std::vector<cd> HZ(NZ * 8, cd(0, 0)), bw(std::max(NZ, 1));
  for (int i = 0; i < NZ; ++i) amp_pc_angular(md, e, i, cd(1, 0), &HZ[i * 8]);
  const double mz = e.p0(1);
  double tot = 0;
  for (int b = 0; b < nb; ++b) {
    if (NZ > 0 && !pc_lineshapes(md, mz + off[b], 1.0, bw.data())) return std::nan("");
    double s = 0;
    for (int h = 0; h < 8; ++h) {
      cd a = HL[h];
      for (int i = 0; i < NZ; ++i) a += bw[i] * HZ[i * 8 + h];
      s += std::norm(a);
    }
    tot += wt[b] * s;
  }
  return tot;
}

// In the reference the 3/2-band and 20-bin windows are tested on the float mass.
bool in_mc_smear_window(float mz) { return (mz > 4.4 && mz < 4.48) || (mz > 4.27 && mz < 4.34); }

}  // namespace

extern "C" {

void oracle_set_kmatrix_isospin(int on) { g_kmatrix_isospin = on != 0; }

// Per-event |A|^2 with the reference's band dispatch (kernel_calEva.cu:819-961):
//   [0, nda_smr)                     30-offset smearing
//   [nda_smr, nda_smr + nda_fine)    150-offset smearing
//   [nda_smr + nda_fine, n_events)   20-offset smearing inside the MC windows, else unsmeared,
//                                    times the event weight w unless w <= -1000 (data sentinel).
// fx_noint receives w*|A|^2 without Pc/Lambda* interference (0 for data).  Returns 0 on success.
// pp3 / pp4: the Zcs chain planes (mJ/psi K, AX; DX), required when NX > 0.
int oracle_eval_fx_x(const float* pp, const float* pp1, const float* pp2, const float* pp3, const float* pp4,
                     long n_size, long n_events, long nda_smr, long nda_fine, const float* paraList, int para_size,
                     int vamp_size, int spline_size, int NR, int NZ, int NX, float FFR, float FFB,
                     int swap_coupling_parts, double* fx, double* fx_noint, int nthreads) {
  if (NX > 0 && (!pp3 || !pp4)) return -10;
  Model md;
  md.pl = paraList;
  md.para_size = para_size;
  md.vamp_size = vamp_size;
  md.spline_size = spline_size;
  md.NR = NR;
  md.NZ = NZ;
  md.NX = NX;
  md.FFR = FFR;
  md.FFB = FFB;
  md.swap_coupling_parts = swap_coupling_parts != 0;
  configure(md);
  const long b1 = std::max(0L, nda_smr);
  const long b2 = std::max(0L, nda_smr + nda_fine);
  int err = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) reduction(| : err)
  for (long i = 0; i < n_events; ++i) {
    Ev e{pp, pp1, pp2, n_size, i, pp3, pp4};
    double v;
    if (i < b1) {
      v = amp2_smeared(md, e, 30, kSmear30);
      fx[i] = v;
      if (fx_noint) fx_noint[i] = 0;
    } else if (i < b2) {
      v = amp2_smeared(md, e, 150, kSmear150);
      fx[i] = v;
      if (fx_noint) fx_noint[i] = 0;
    } else {
      const float mz = pp[i + n_size];
      v = in_mc_smear_window(mz) ? amp2_smeared(md, e, 20, kSmear20) : amp2_unsmeared(md, e, true);
      const double w = pp[i + 2 * n_size];
      const bool data = pp[i + 2 * n_size] <= -1000.f;
      fx[i] = data ? v : v * w;
      if (fx_noint) fx_noint[i] = data ? 0.0 : amp2_unsmeared(md, e, false) * w;
    }
    if (std::isnan(v)) err |= 1;
  }
  return err ? -12 : 0;
}

// Every event smeared with the weighted grid (off[b] GeV, weight wt[b]); fx weighted by w for MC,
// fx_noint the unsmeared non-interfering w|A|^2 of MC events (0 for data).
int oracle_eval_fx_grid(const float* pp, const float* pp1, const float* pp2, const float* pp3, const float* pp4,
                        long n_size, long n_events, int nb, const double* off, const double* wt,
                        const float* paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                        int NX, float FFR, float FFB, double* fx, double* fx_noint, int nthreads) {
  if (NX > 0 && (!pp3 || !pp4)) return -10;
  if (nb < 1 || !off || !wt) return -11;
  Model md;
  md.pl = paraList;
  md.para_size = para_size;
  md.vamp_size = vamp_size;
  md.spline_size = spline_size;
  md.NR = NR;
  md.NZ = NZ;
  md.NX = NX;
  md.FFR = FFR;
  md.FFB = FFB;
  configure(md);
  int err = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) reduction(| : err)
  for (long i = 0; i < n_events; ++i) {
    Ev e{pp, pp1, pp2, n_size, i, pp3, pp4};
    const double v = amp2_smeared_grid(md, e, nb, off, wt);
    const double w = pp[i + 2 * n_size];
    const bool data = pp[i + 2 * n_size] <= -1000.f;
    fx[i] = data ? v : v * w;
    if (fx_noint) fx_noint[i] = data ? 0.0 : amp2_unsmeared(md, e, false) * w;
    if (std::isnan(v)) err |= 1;
  }
  return err ? -12 : 0;
}

int oracle_eval_fx(const float* pp, const float* pp1, const float* pp2, long n_size, long n_events,
                   long nda_smr, long nda_fine, const float* paraList, int para_size, int vamp_size,
                   int spline_size, int NR, int NZ, int NX, float FFR, float FFB, int swap_coupling_parts,
                   double* fx, double* fx_noint, int nthreads) {
  return oracle_eval_fx_x(pp, pp1, pp2, nullptr, nullptr, n_size, n_events, nda_smr, nda_fine, paraList,
                          para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, swap_coupling_parts, fx,
                          fx_noint, nthreads);
}

// Per-event unsmeared coherent |A|^2 without weights (GetAmp2s_NoSMR as used by
// kernel_store_amp2s, kernel_calEva.cu:1365-1373).
int oracle_amp2_x(const float* pp, const float* pp1, const float* pp2, const float* pp3, const float* pp4,
                  long n_size, long n_events, const float* paraList, int para_size, int vamp_size, int spline_size,
                  int NR, int NZ, int NX, float FFR, float FFB, double* out, int nthreads) {
  if (NX > 0 && (!pp3 || !pp4)) return -10;
  Model md;
  md.pl = paraList;
  md.para_size = para_size;
  md.vamp_size = vamp_size;
  md.spline_size = spline_size;
  md.NR = NR;
  md.NZ = NZ;
  md.NX = NX;
  md.FFR = FFR;
  md.FFB = FFB;
  configure(md);
  int err = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) reduction(| : err)
  for (long i = 0; i < n_events; ++i) {
    Ev e{pp, pp1, pp2, n_size, i, pp3, pp4};
    out[i] = amp2_unsmeared(md, e, true);
    if (std::isnan(out[i])) err |= 1;
  }
  return err ? -12 : 0;
}

int oracle_amp2(const float* pp, const float* pp1, const float* pp2, long n_size, long n_events,
                const float* paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                float FFR, float FFB, double* out, int nthreads) {
  return oracle_amp2_x(pp, pp1, pp2, nullptr, nullptr, n_size, n_events, paraList, para_size, vamp_size,
                       spline_size, NR, NZ, NX, FFR, FFB, out, nthreads);
}

// NLL assembly of host_store_fx (kernel_calEva.cu:1296-1362) from per-event values, with
// compensated sums.  Returns the MC normalisation sum; writes the NLL (including the
// +1000 interference guard) to *nll.
double oracle_assemble_nll(const double* fx, const double* fx_noint, const float* sw, long nda,
                           long n_events, double sum_w_mc, double sum_w_data, double nll_shift,
                           double* nll) {
  auto kahan = [](double& s, double& c, double x) {
    const double y = x - c, t = s + y;
    c = (t - s) - y;
    s = t;
  };
  double si = 0, ci = 0, sn = 0, cn = 0, sd = 0, cdd = 0;
  for (long i = nda; i < n_events; ++i) {
    kahan(si, ci, fx[i]);
    kahan(sn, cn, fx_noint[i]);
  }
  for (long i = 0; i < nda; ++i) kahan(sd, cdd, fx[i] > 0 ? std::log(fx[i]) * (double)sw[i] : -1e12);
  double v = nll_shift + sum_w_data * std::log(si / sum_w_mc) - sd;
  if (std::fabs(sn / si - 1.0) > F(0.3f)) v += 1000.0;
  *nll = v;
  return si;
}

// Lineshape probes for unit tests.
void oracle_bw_lstar(double m_r, double gamma_r, double mpp, int LR, double ffr, double* out) {
  const cd v = bw_lstar(m_r, gamma_r, mpp, LR, ffr);
  out[0] = v.real();
  out[1] = v.imag();
}
void oracle_bw_pc(double m_r, double gamma_r, double mpp, int LR, double ffr, double* out) {
  const cd v = bw_pc(m_r, gamma_r, mpp, LR, ffr);
  out[0] = v.real();
  out[1] = v.imag();
}
double oracle_barrier_lb_lstar(double J, double mpp, double mr, double ffb) {
  return barrier_lb_lstar(J, mpp, mr, ffb);
}
double oracle_barrier_lb_pc(double J, double mpp, double mr, double ffb) { return barrier_lb_pc(J, mpp, mr, ffb); }

// P-vector outputs of K-matrix group ik at mass mpp; out holds 2*(Npole+4) doubles.  Returns the
// number of complex outputs or a negative error.
int oracle_kmatrix(const float* paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                   double FFB, double mpp, int ik, double* out) {
  Model md;
  md.pl = paraList;
  md.para_size = para_size;
  md.vamp_size = vamp_size;
  md.spline_size = spline_size;
  md.NR = NR;
  md.NZ = NZ;
  md.FFB = FFB;
  configure(md);
  const int J = (ik == 1 || ik == 3) ? 3 : 1;
  const int P = (ik >= 2) ? 1 : -1;
  cd M[NPMAX + NKMC];
  const int n = kmatrix_group(md, mpp, J, P, ik, M);
  for (int i = 0; i < n; ++i) {
    out[2 * i] = M[i].real();
    out[2 * i + 1] = M[i].imag();
  }
  return n;
}

// host_store_lineshapeLsKM (kernel_calEva.cu:1490-1584): for every Lambda* entry iLz < NR and mass
// h_mkp[i], the revised K-matrix lineshape in its refactored form times the Lambda_b barrier, and the
// Breit-Wigner times the same barrier; both barriers with radius FFR, as the reference calls them.
// Outputs [iLz * n_points + i].
int oracle_lineshapes_lstar_km(const float* h_mkp, int n_points, int NR, float FFR, const float* paraList,
                               double* km_re, double* km_im, double* bw_re, double* bw_im) {
  for (int i = 0; i < n_points; ++i) {
    const double mkp = h_mkp[i];
    for (int r = 0; r < NR; ++r) {
      const Entry E = entry(paraList, r);
      const double bt = barrier_lb_lstar(0.5 * E.S2, mkp, E.m, FFR);
      const cd km = revised_km_refactor(paraList, mkp, r, 0, NR, false, FFR) * bt;
      const cd bw = bw_lstar(E.m, E.g, mkp, E.LR, FFR) * bt;
      km_re[r * n_points + i] = km.real();
      km_im[r * n_points + i] = km.imag();
      bw_re[r * n_points + i] = bw.real();
      bw_im[r * n_points + i] = bw.imag();
    }
  }
  return 0;
}

// Every Lambda* lineshape times its production barrier at mkp (lstar: 2 NR doubles) and every Pc
// lineshape times its barrier at mz (pc: 2 NZ doubles), as the amplitude kernels use them.
int oracle_lineshapes(const float* paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                      float FFR, float FFB, double mkp, double mz, double* lstar, double* pc) {
  Model md;
  md.pl = paraList;
  md.para_size = para_size;
  md.vamp_size = vamp_size;
  md.spline_size = spline_size;
  md.NR = NR;
  md.NZ = NZ;
  md.FFR = FFR;
  md.FFB = FFB;
  configure(md);
  for (int r = 0; r < NR; ++r) {
    const Entry E = entry(paraList, r);
    double m0 = E.m;
    cd bw(1, 0);
    if (E.type == T_BREITWIGNER) {
      bw = bw_lstar(E.m, E.g, mkp, E.LR, FFR);
    } else if (E.type == T_MODELINDEPENDENT) {
      bw = spline_wave(paraList + md.splcount[r], NUMSP, SPL_LSTAR_LO, SPL_LSTAR_HI, mkp);
      m0 = -0.5;
    } else if (E.type == T_REVISEDKMATRIX) {
      bw = revised_km(paraList, mkp, r, 0, NR, false, FFR);
    } else if (E.type != T_NONRESONANT) {
      return -1;
    }
    bw *= barrier_lb_lstar(0.5 * E.S2, mkp, m0, FFB);
    lstar[2 * r] = bw.real();
    lstar[2 * r + 1] = bw.imag();
  }
  if (NZ > 0) {
    std::vector<cd> b(NZ);
    if (!pc_lineshapes(md, mz, 1.0, b.data())) return -2;
    for (int i = 0; i < NZ; ++i) {
      pc[2 * i] = b[i].real();
      pc[2 * i + 1] = b[i].imag();
    }
  }
  return 0;
}

}  // extern "C"
