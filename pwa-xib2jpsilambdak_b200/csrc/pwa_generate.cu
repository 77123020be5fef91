// On-device synthetic events: flat Lambda_b -> J/psi(-> mu mu) p K- phase space, the helicity angles
// of the ntuple maker (gen_toys/phsp_toys/tree.C:127-406) and the per-event angular basis of
// RooDalitzAmplitude::filldlz (src/RooDalitzAmplitude.cxx:7086-7308), written straight into the
// reference SoA planes.  One thread per event; random numbers come from a counter-based Philox4x32-10
// generator keyed by (seed, event id), so any event can be regenerated independently.
//
// Rounding points of the reference basis are reproduced: angles are float(acos(cos)), the phase sums
// are formed in float without contraction, products in double, stored as float.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/pwa_b200.h"
#include "pwa_physics.cuh"

namespace pwa {
namespace gen {

constexpr double MU = 0.105658;  // muon mass of the toy generator (gentoy_formhj.C:11)

// ------------------------------------------------------------------ Philox4x32-10 (Salmon et al. 2011)
struct u32x4 {
  uint32_t x, y, z, w;
};
__device__ __forceinline__ u32x4 philox(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}
struct Rng {
  uint64_t id;
  uint32_t k0, k1, ctr = 0;
  u32x4 buf{};
  int left = 0;
  __device__ uint32_t next32() {
    if (left == 0) {
      buf = philox(u32x4{(uint32_t)id, (uint32_t)(id >> 32), ctr++, 0x5057u}, k0, k1);
      left = 4;
    }
    const uint32_t v = (left == 4) ? buf.x : (left == 3) ? buf.y : (left == 2) ? buf.z : buf.w;
    --left;
    return v;
  }
  // uniform in (0, 1) with 53 random bits
  __device__ double uni() {
    const uint64_t a = next32() >> 5, b = next32() >> 6;
    return ((double)(a * 67108864ull + b) + 0.5) * (1.0 / 9007199254740992.0);
  }
};

// ------------------------------------------------------------------ small vector algebra (FP64)
struct V3 {
  double x, y, z;
};
struct V4 {
  V3 p;
  double e;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 unit(V3 a) {
  const double n = sqrt(dot(a, a));
  return n > 0 ? (1.0 / n) * a : a;
}
__device__ __forceinline__ V4 operator+(V4 a, V4 b) { return {a.p + b.p, a.e + b.e}; }
__device__ __forceinline__ V4 boost(V4 v, V3 b) {
  const double b2 = dot(b, b);
  const double g = 1.0 / sqrt(1.0 - b2);
  const double bp = dot(b, v.p);
  const double g2 = b2 > 0 ? (g - 1.0) / b2 : 0.0;
  return {v.p + (g2 * bp + g * v.e) * b, g * (v.e + bp)};
}
// into the rest frame of `parent`
__device__ __forceinline__ V4 to_rest(V4 v, V4 parent) { return boost(v, (-1.0 / parent.e) * parent.p); }
__device__ __forceinline__ double mass(V4 v) { return sqrt(fmax(v.e * v.e - dot(v.p, v.p), 0.0)); }
__device__ __forceinline__ double clamp1(double c) { return fmin(1.0, fmax(-1.0, c)); }

struct Angles {
  double cLb, cL, cPsi, phiK, phiMu;                    // Lambda* chain
  double zcLb, zcZ, zcPsi, zphiZ, zphiPsi, zphiMu;      // Pc chain
  double cP, alphaMu;                                   // alignment
  double mkp, mz, mpsik;
};

// Flat phase space in the Lambda_b rest frame (Dalitz-plane rejection, isotropic orientation and
// J/psi decay).  Returns false if the bounded rejection loop did not accept.
__device__ bool phase_space(Rng& R, V4& p, V4& k, V4& mup, V4& mum) {
  const double M = M_LB;
  const double s1lo = sq(M_P + M_K), s1hi = sq(M - M_JPSI);
  const double s2lo = sq(M_JPSI + M_P), s2hi = sq(M - M_K);
  double s1 = 0, s2 = 0;
  bool ok = false;
  for (int t = 0; t < 256 && !ok; ++t) {
    s1 = s1lo + (s1hi - s1lo) * R.uni();
    s2 = s2lo + (s2hi - s2lo) * R.uni();
    const double m1 = sqrt(s1);
    const double ep = (s1 - M_K * M_K + M_P * M_P) / (2 * m1);
    const double epsi = (M * M - s1 - M_JPSI * M_JPSI) / (2 * m1);
    const double qp = sqrt(fmax(ep * ep - M_P * M_P, 0.0)), qpsi = sqrt(fmax(epsi * epsi - M_JPSI * M_JPSI, 0.0));
    const double lo = sq(ep + epsi) - sq(qp + qpsi), hi = sq(ep + epsi) - sq(qp - qpsi);
    ok = (s2 > lo) && (s2 < hi);
  }
  if (!ok) return false;
  const double s3 = M * M + M_JPSI * M_JPSI + M_P * M_P + M_K * M_K - s1 - s2;
  const double Epsi = (M * M + M_JPSI * M_JPSI - s1) / (2 * M);
  const double Ek = (M * M + M_K * M_K - s2) / (2 * M);
  const double Ep = (M * M + M_P * M_P - s3) / (2 * M);
  const double qpsi = sqrt(fmax(Epsi * Epsi - M_JPSI * M_JPSI, 0.0));
  const double qk = sqrt(fmax(Ek * Ek - M_K * M_K, 0.0));
  const double qp = sqrt(fmax(Ep * Ep - M_P * M_P, 0.0));
  const double ca = clamp1((qpsi * qpsi + qp * qp - qk * qk) / (2 * qpsi * qp));
  const double sa = sqrt(fmax(1 - ca * ca, 0.0));
  V3 psi3{qpsi, 0, 0}, p3{-qp * ca, qp * sa, 0};
  V3 k3 = -(psi3 + p3);
  // uniform rotation from a uniform unit quaternion (Shoemake)
  const double u1 = R.uni(), u2 = R.uni(), u3 = R.uni();
  const double a = sqrt(1 - u1), b = sqrt(u1);
  const double w = a * sin(2 * M_PI * u2), x = a * cos(2 * M_PI * u2), y = b * sin(2 * M_PI * u3),
               z = b * cos(2 * M_PI * u3);
  auto rot = [&](V3 v) -> V3 {
    return {(1 - 2 * (y * y + z * z)) * v.x + 2 * (x * y - z * w) * v.y + 2 * (x * z + y * w) * v.z,
            2 * (x * y + z * w) * v.x + (1 - 2 * (x * x + z * z)) * v.y + 2 * (y * z - x * w) * v.z,
            2 * (x * z - y * w) * v.x + 2 * (y * z + x * w) * v.y + (1 - 2 * (x * x + y * y)) * v.z};
  };
  V4 psi{rot(psi3), Epsi};
  p = V4{rot(p3), Ep};
  k = V4{rot(k3), Ek};
  const double qmu = two_body_p(M_JPSI, MU, MU);
  const double c = 2 * R.uni() - 1, ph = 2 * M_PI * R.uni() - M_PI;
  const double sn = sqrt(fmax(1 - c * c, 0.0));
  const V3 mu3{qmu * sn * cos(ph), qmu * sn * sin(ph), qmu * c};
  const double emu = sqrt(qmu * qmu + MU * MU);
  const V3 bpsi = (1.0 / psi.e) * psi.p;
  mup = boost(V4{mu3, emu}, bpsi);
  mum = boost(V4{-mu3, emu}, bpsi);
  return true;
}

// Helicity angles with the ntuple maker's conventions; the Lambda_b flight direction is +z.
__device__ Angles helicity_angles(V4 p, V4 k, V4 mup, V4 mum) {
  Angles A;
  const V4 psi = mup + mum, lam = p + k, zc = psi + p;
  const V3 zh{0, 0, 1};
  {  // helicityJpsiLam
    const V3 L = unit(lam.p), psiU = unit(psi.p);
    A.cLb = dot(zh, L);
    const V3 U = unit(to_rest(p, lam).p);
    A.cL = -dot(psiU, U);
    V3 ab = -unit(zh - dot(zh, L) * L);
    A.phiK = atan2(dot(unit(cross(-psiU, ab)), U), dot(ab, U));
    ab = -ab;
    const V3 U2 = unit(to_rest(mum, psi).p);
    A.cPsi = dot(psiU, U2);
    A.phiMu = atan2(dot(unit(cross(psiU, ab)), U2), dot(ab, U2));
  }
  {  // helicityZK
    const V3 ZU = unit(zc.p);
    A.zcLb = dot(zh, ZU);
    V3 ab = unit(lam.p - dot(lam.p, zh) * zh);
    A.zphiZ = atan2(dot(unit(cross(zh, ab)), ZU), dot(ab, ZU));
    const V4 psiz = to_rest(psi, zc), kz = to_rest(k, zc), mumz = to_rest(mum, zc);
    const V3 U = unit(psiz.p), kU = unit(kz.p);
    A.zcZ = -dot(kU, U);
    ab = -unit(zh - dot(zh, ZU) * ZU);
    A.zphiPsi = atan2(dot(unit(cross(-kU, ab)), U), dot(ab, U));
    const V3 U2 = unit(to_rest(mumz, psiz).p);
    A.zcPsi = dot(U, U2);
    ab = -unit(-kz.p + dot(kz.p, U) * U);
    A.zphiMu = atan2(dot(unit(cross(U, ab)), U2), dot(ab, U2));
  }
  {  // helicityTwoFrame
    A.cP = dot(unit(to_rest(k, p).p), unit(to_rest(psi, p).p));
    const V3 z3 = unit(to_rest(mum, psi).p);
    const V4 pps = to_rest(p, psi), lps = to_rest(lam, psi);
    const V3 x3z = -unit(-pps.p + dot(pps.p, z3) * z3);
    const V3 x3l = -unit(-lps.p + dot(lps.p, z3) * z3);
    A.alphaMu = atan2(dot(unit(cross(z3, x3z)), x3l), dot(x3z, x3l));
  }
  A.cLb = clamp1(A.cLb);
  A.cL = clamp1(A.cL);
  A.cPsi = clamp1(A.cPsi);
  A.zcLb = clamp1(A.zcLb);
  A.zcZ = clamp1(A.zcZ);
  A.zcPsi = clamp1(A.zcPsi);
  A.cP = clamp1(A.cP);
  A.mkp = mass(lam);
  A.mz = mass(zc);
  A.mpsik = mass(psi + k);
  return A;
}

// ------------------------------------------------------------------ d-functions
__constant__ double kLnFact[64];

__device__ __forceinline__ double d_half(double beta, int am, int an) {
  if (am == an) return cos(0.5 * beta);
  return (am == 1) ? -sin(0.5 * beta) : sin(0.5 * beta);
}
__device__ __forceinline__ double d_one(double beta, int am, int an) {
  if (am == an) return (cos(beta) + 1.0) / 2.0;
  if (am != 0) return (1.0 - cos(beta)) / 2.0;
  return sin(beta) * 7.07106781186547461715e-01 * (an == 1 ? 1.0 : -1.0);
}
// d^j_{mn}(beta), all arguments doubled; log-factorial sum of Varshalovich 4.3.1(3).
__device__ double d_j(double beta, int j2, int m2, int n2) {
  const int jpm = (j2 + m2) / 2, jpn = (j2 + n2) / 2, jmm = (j2 - m2) / 2, jmn = (j2 - n2) / 2, mpn = (m2 + n2) / 2;
  if (jpm < 0 || jpn < 0 || jmm < 0 || jmn < 0) return 0.0;
  const double pi = 3.141592653589793116, pi2 = 6.283185307179586232;
  if (fabs(beta) < 1e-10) return (jpm == jpn) ? 1.0 : 0.0;
  if (fabs(beta - pi) < 1e-10) return (jpm == jmn) ? ((abs(jpm) % 2 == 1) ? -1.0 : 1.0) : 0.0;
  if (fabs(beta - pi2) < 1e-10) return (jpm == jpn) ? ((abs(mpn) % 2 == 1) ? -1.0 : 1.0) : 0.0;
  const double b = 0.5 * beta;
  const double s = log(sin(b)), c = log(fabs(cos(b)));
  const double rt = 0.5 * (kLnFact[jpm] + kLnFact[jmm] + kLnFact[jpn] + kLnFact[jmn]);
  const int k0 = max(0, mpn);
  int kq = k0 + jpm;
  if (beta > pi) kq += mpn;
  double q = (kq % 2 == 1) ? -1.0 : 1.0;
  double cx = 2 * k0 - mpn, sx = jpm + jpn - 2 * k0, r = 0.0;
  for (int k = k0; k <= min(jpm, jpn); ++k) {
    r += q * exp(rt - kLnFact[k] - kLnFact[jpm - k] - kLnFact[jpn - k] - kLnFact[k - mpn] + cx * c + sx * s);
    cx += 2;
    sx -= 2;
    q = -q;
  }
  return r;
}

// ------------------------------------------------------------------ basis
__device__ void write_basis(const Angles& A, float* pp, float* pp1, float* pp2, int64_t ns, int64_t e, float w) {
  const double th = (float)acos(A.cLb), th1 = (float)acos(A.cL), th2 = (float)acos(A.cPsi);
  const double thB = (float)acos(A.zcLb), thZ = (float)acos(A.zcZ), thPsi = (float)acos(A.zcPsi);
  const double thp = (float)acos(A.cP);
  const float phi1 = (float)A.phiK, phi2 = (float)A.phiMu, phiZ = (float)A.zphiZ, phiPsi = (float)A.zphiPsi,
              phiMu = (float)A.zphiMu, alphaMu = (float)A.alphaMu;
  pp[e] = (float)A.mkp;
  pp[e + ns] = (float)A.mz;
  pp[e + 2 * ns] = w;
  const int HEL1T[6] = {1, 1, -1, -1, 3, -3}, HEL2[6] = {1, 0, 0, -1, 1, -1};
  for (int i = 0; i < 2; ++i) {
    const int dmu = i ? 1 : -1;
    for (int j = 0; j < 2; ++j) {
      const int h0t = j ? 1 : -1;  // 2 x hel0
      for (int m = 0; m < 6; ++m) {
        const float part = __fadd_rn(__fmul_rn(0.5f * HEL1T[m], phi1), __fmul_rn((float)HEL2[m], phi2));
        const double dh = d_half(th, h0t, HEL1T[m] - 2 * HEL2[m]);
        const double d1 = d_one(th2, HEL2[m], dmu);
        double sn, cs;
        sincos((double)part, &sn, &cs);
        const int a = 3 + (i * 12 + j * 6 + m) * 2;
        pp[e + a * ns] = (float)((cs * dh) * d1);
        pp[e + (a + 1) * ns] = (float)((sn * dh) * d1);
      }
    }
  }
  for (int s = 0; s < 5; ++s)
    for (int k = 0; k < 2; ++k)
      for (int m = 0; m < 6; ++m) {
        const float v = (s == 0 && m >= 4) ? 0.f : (float)d_j(th1, 2 * s + 1, HEL1T[m], k ? 1 : -1);
        pp[e + (51 + s * 12 + k * 6 + m) * ns] = v;
      }
  for (int i = 0; i < 2; ++i) {
    const int dmu = i ? 1 : -1;
    for (int j = 0; j < 2; ++j) {
      const float h0 = j ? 0.5f : -0.5f;
      int m = 0;
      for (int hpsi = -1; hpsi <= 1; ++hpsi)
        for (int ihz = 0; ihz < 2; ++ihz) {
          const float hz = ihz ? 0.5f : -0.5f;
          float part = __fadd_rn(__fmul_rn(h0, phiZ), __fmul_rn((float)hpsi, phiMu));
          part = __fadd_rn(part, __fmul_rn(hz, phiPsi));
          part = __fadd_rn(part, __fmul_rn((float)dmu, alphaMu));
          const double d1 = d_one(thPsi, hpsi, dmu);
          const double dh = d_half(thB, j ? 1 : -1, ihz ? 1 : -1);
          double sn, cs;
          sincos((double)part, &sn, &cs);
          const float re = (float)((cs * d1) * dh), im = (float)((sn * d1) * dh);
          for (int ihp = 0; ihp < 2; ++ihp, ++m) {
            const int a = (i * 24 + j * 12 + m) * 2;
            pp1[e + a * ns] = re;
            pp1[e + (a + 1) * ns] = im;
          }
        }
    }
  }
  for (int s = 0; s < 4; ++s)
    for (int k = 0; k < 2; ++k) {
      int m = 0;
      for (int hpsi = -1; hpsi <= 1; ++hpsi)
        for (int ihz = 0; ihz < 2; ++ihz)
          for (int ihp = 0; ihp < 2; ++ihp, ++m) {
            const int hp2 = ihp ? 1 : -1;  // 2 x help
            float v = 0.f;
            if (!(abs(2 * hpsi - hp2) > 2 * s + 1))
              v = (float)(d_half(thp, hp2, k ? 1 : -1) * d_j(thZ, 2 * s + 1, ihz ? 1 : -1, 2 * hpsi - hp2));
            pp2[e + (s * 24 + k * 12 + m) * ns] = v;
          }
    }
}

__global__ void k_generate(float* pp, float* pp1, float* pp2, int64_t ns, int64_t col0, int64_t n, uint64_t seed,
                           uint64_t first_id, float w_lo, float w_hi, int data, int* n_failed) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  Rng R;
  R.id = first_id + (uint64_t)t;
  R.k0 = (uint32_t)seed;
  R.k1 = (uint32_t)(seed >> 32);
  V4 p, k, mup, mum;
  if (!phase_space(R, p, k, mup, mum)) {
    atomicAdd(n_failed, 1);
    p = V4{{0.1, 0.2, 0.3}, 0}, k = p, mup = p, mum = p;
    p.e = sqrt(dot(p.p, p.p) + M_P * M_P);
  }
  const Angles A = helicity_angles(p, k, mup, mum);
  const float w = data ? -1001.f : (float)(w_lo + (w_hi - w_lo) * R.uni());
  write_basis(A, pp, pp1, pp2, ns, col0 + t, w);
}

// angles[16][n] in the order: mLk, mjpsiL, cosTheta_Lb, cosTheta_L, cosTheta_Jpsi, phiK, phiMu,
// Z_cosTheta_Lb, Z_cosTheta_Z, Z_cosTheta_Jpsi, Z_phiZ, Z_phiJpsi, Z_phiMu, cosTheta_Lambda, alpha_Mu, w
__global__ void k_basis_from_angles(const double* ang, int64_t n, float* pp, float* pp1, float* pp2, int64_t ns) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  Angles A;
  A.mkp = ang[t];
  A.mz = ang[n + t];
  A.cLb = ang[2 * n + t];
  A.cL = ang[3 * n + t];
  A.cPsi = ang[4 * n + t];
  A.phiK = ang[5 * n + t];
  A.phiMu = ang[6 * n + t];
  A.zcLb = ang[7 * n + t];
  A.zcZ = ang[8 * n + t];
  A.zcPsi = ang[9 * n + t];
  A.zphiZ = ang[10 * n + t];
  A.zphiPsi = ang[11 * n + t];
  A.zphiMu = ang[12 * n + t];
  A.cP = ang[13 * n + t];
  A.alphaMu = ang[14 * n + t];
  write_basis(A, pp, pp1, pp2, ns, t, (float)ang[15 * n + t]);
}

// four-vectors[16][n] (p, k, mu+, mu-: px py pz E) -> angles[15][n] (same order as above, no w)
__global__ void k_angles_from_vectors(const double* v, int64_t n, double* ang) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  auto ld = [&](int q) { return V4{{v[(4 * q) * n + t], v[(4 * q + 1) * n + t], v[(4 * q + 2) * n + t]}, v[(4 * q + 3) * n + t]}; };
  const Angles A = helicity_angles(ld(0), ld(1), ld(2), ld(3));
  const double out[15] = {A.mkp, A.mz, A.cLb, A.cL, A.cPsi, A.phiK, A.phiMu, A.zcLb, A.zcZ, A.zcPsi, A.zphiZ,
                          A.zphiPsi, A.zphiMu, A.cP, A.alphaMu};
  for (int q = 0; q < 15; ++q) ang[q * n + t] = out[q];
}

int init_tables() {
  static bool done = false;
  if (done) return 0;
  double lf[64];
  for (int i = 0; i < 64; ++i) lf[i] = std::lgamma((double)i + 1.0);
  if (cudaMemcpyToSymbol(kLnFact, lf, sizeof(lf)) != cudaSuccess) return PWA_E_CUDA;
  done = true;
  return 0;
}

// ------------------------------------------------------------------ unit coordinates
// The phase space as a map from x in [0,1]^7 (the coordinates of the learned proposal density):
// s2 = m^2(J/psi p) linear in x0 over [(m_J/psi + m_p)^2, (m_Lb - m_K)^2] (so that the Pc bands lie at
// fixed x0) and s1 = m^2(Kp) linear in x1 across the Dalitz row at that s2 (so that the region's
// boundary is x1 = 0 and x1 = 1); the decay's orientation in the Lambda_b rest frame from the J/psi
// direction (cos theta = 2 x2 - 1 to the flight axis, azimuth 2 pi x3) and the roll 2 pi x4 of the
// decay plane about it (together a uniform rotation); the mu+ direction in the J/psi rest frame
// (cos = 2 x5 - 1, phi = 2 pi x6 - pi), as the flat generator above draws it.  Flat phase space has
// density (s2 range) (row length at s2) / (Dalitz area) in these coordinates.
//
// Range of s1 = m^2(Kp) at s2 = m^2(J/psi p): the p and K- energies and momenta in the J/psi p rest
// frame give the extremes (E_p + E_K)^2 - (q_p -+ q_K)^2.
__host__ __device__ inline void dalitz_row(double s2, double& lo, double& hi) {
  const double M = M_LB, m2 = sqrt(s2);
  const double ep = (s2 - M_JPSI * M_JPSI + M_P * M_P) / (2 * m2);
  const double ek = (M * M - s2 - M_K * M_K) / (2 * m2);
  const double qp = sqrt(fmax(ep * ep - M_P * M_P, 0.0)), qk = sqrt(fmax(ek * ek - M_K * M_K, 0.0));
  lo = sq(ep + ek) - sq(qp + qk);
  hi = sq(ep + ek) - sq(qp - qk);
}
constexpr double S2_LO = (M_JPSI + M_P) * (M_JPSI + M_P), S2_HI = (M_LB - M_K) * (M_LB - M_K);

__device__ void event_from_unit(const double* x, V4& p, V4& k, V4& mup, V4& mum, double& row_len) {
  const double M = M_LB;
  const double s2 = S2_LO + (S2_HI - S2_LO) * x[0];
  double lo, hi;
  dalitz_row(s2, lo, hi);
  row_len = hi - lo;
  const double s1 = lo + (hi - lo) * x[1];
  const double s3 = M * M + M_JPSI * M_JPSI + M_P * M_P + M_K * M_K - s1 - s2;
  const double Epsi = (M * M + M_JPSI * M_JPSI - s1) / (2 * M);
  const double Ek = (M * M + M_K * M_K - s2) / (2 * M);
  const double Ep = (M * M + M_P * M_P - s3) / (2 * M);
  const double qpsi = sqrt(fmax(Epsi * Epsi - M_JPSI * M_JPSI, 0.0));
  const double qk = sqrt(fmax(Ek * Ek - M_K * M_K, 0.0));
  const double qp = sqrt(fmax(Ep * Ep - M_P * M_P, 0.0));
  const double ca = clamp1((qpsi * qpsi + qp * qp - qk * qk) / (2 * qpsi * qp));
  const double sa = sqrt(fmax(1 - ca * ca, 0.0));
  const V3 psi3{qpsi, 0, 0}, p3{-qp * ca, qp * sa, 0};
  const V3 k3 = -(psi3 + p3);
  const double ct = 2 * x[2] - 1, st = sqrt(fmax(1 - ct * ct, 0.0));
  const double ph = 2 * M_PI * x[3], chi = 2 * M_PI * x[4];
  const V3 e1{st * cos(ph), st * sin(ph), ct};
  const V3 e2{-sin(ph), cos(ph), 0.0};
  const V3 e3{-ct * cos(ph), -ct * sin(ph), st};
  const V3 f2 = cos(chi) * e2 + sin(chi) * e3, f3 = cos(chi) * e3 - sin(chi) * e2;
  auto rot = [&](V3 v) { return v.x * e1 + v.y * f2 + v.z * f3; };
  const V4 psi{rot(psi3), Epsi};
  p = V4{rot(p3), Ep};
  k = V4{rot(k3), Ek};
  const double qmu = two_body_p(M_JPSI, MU, MU);
  const double c = 2 * x[5] - 1, phm = 2 * M_PI * x[6] - M_PI;
  const double sn = sqrt(fmax(1 - c * c, 0.0));
  const V3 mu3{qmu * sn * cos(phm), qmu * sn * sin(phm), qmu * c};
  const double emu = sqrt(qmu * qmu + MU * MU);
  const V3 bpsi = (1.0 / psi.e) * psi.p;
  mup = boost(V4{mu3, emu}, bpsi);
  mum = boost(V4{-mu3, emu}, bpsi);
}

__global__ void k_events_from_unit(const double* __restrict__ x, int64_t ldx, int64_t n, float* pp, float* pp1,
                                   float* pp2, int64_t ns, int64_t col0, float w, int data, double* flat,
                                   double norm) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double u[7];
  for (int d = 0; d < 7; ++d) u[d] = x[d * ldx + t];
  V4 p, k, mup, mum;
  double row_len;
  event_from_unit(u, p, k, mup, mum, row_len);
  write_basis(helicity_angles(p, k, mup, mum), pp, pp1, pp2, ns, col0 + t, data ? -1001.f : w);
  if (flat) flat[t] = row_len * norm;
}

// Flat phase space in unit coordinates: x0 by rejection against the Dalitz row length (max_len
// bounds it), the other coordinates uniform.
__global__ void k_unit_flat(int64_t n, uint64_t seed, uint64_t first_id, double* x, int64_t ldx, double max_len) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  Rng R;
  R.id = first_id + (uint64_t)t;
  R.k0 = (uint32_t)seed ^ 0x75u;
  R.k1 = (uint32_t)(seed >> 32);
  double x0 = R.uni();
  for (int it = 0; it < 1000; ++it) {  // acceptance is above one half: 1000 tries never run out in practice
    double lo, hi;
    dalitz_row(S2_LO + (S2_HI - S2_LO) * x0, lo, hi);
    if (R.uni() * max_len < hi - lo) break;
    x0 = R.uni();
  }
  x[t] = x0;
  for (int d = 1; d < 7; ++d) x[d * ldx + t] = R.uni();
}

// Dalitz area in (s1, s2) (Simpson's rule on the row length over s2) and the largest row length.
static void dalitz_area(double* area, double* max_len) {
  const int n = 20000;
  const double h = (S2_HI - S2_LO) / n;
  double a = 0, mx = 0;
  for (int i = 0; i <= n; ++i) {
    double lo, hi;
    dalitz_row(S2_LO + i * h, lo, hi);
    const double len = hi - lo;
    a += len * ((i == 0 || i == n) ? 1 : (i % 2 ? 4 : 2));
    mx = fmax(mx, len);
  }
  *area = a * h / 3;
  *max_len = mx * 1.001;
}

}  // namespace gen
}  // namespace pwa

extern "C" {

int pwa_generate_events(float* d_pp, float* d_pp1, float* d_pp2, int64_t n_size, int64_t col0, int64_t n,
                        uint64_t seed, uint64_t first_id, float w_lo, float w_hi, int data, void* stream) {
  if (!d_pp || !d_pp1 || !d_pp2 || n < 0 || col0 < 0 || col0 + n > n_size) return PWA_E_ARG;
  if (n == 0) return PWA_OK;
  if (pwa::gen::init_tables()) return PWA_E_CUDA;
  int* d_fail = nullptr;
  if (cudaMalloc(&d_fail, sizeof(int)) != cudaSuccess) return PWA_E_NOMEM;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(d_fail, 0, sizeof(int), st);
  pwa::gen::k_generate<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_pp, d_pp1, d_pp2, n_size, col0, n, seed,
                                                                     first_id, w_lo, w_hi, data, d_fail);
  int failed = 0;
  cudaError_t e = cudaMemcpyAsync(&failed, d_fail, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_fail);
  if (e != cudaSuccess) return PWA_E_CUDA;
  return failed ? PWA_E_PARAM : PWA_OK;
}

int pwa_basis_from_angles(const double* d_angles, int64_t n, float* d_pp, float* d_pp1, float* d_pp2,
                          int64_t n_size, void* stream) {
  if (!d_angles || !d_pp || !d_pp1 || !d_pp2 || n < 0 || n > n_size) return PWA_E_ARG;
  if (n == 0) return PWA_OK;
  if (pwa::gen::init_tables()) return PWA_E_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  pwa::gen::k_basis_from_angles<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_angles, n, d_pp, d_pp1, d_pp2,
                                                                              n_size);
  return cudaStreamSynchronize(st) == cudaSuccess ? PWA_OK : PWA_E_CUDA;
}

int pwa_angles_from_vectors(const double* d_vectors, int64_t n, double* d_angles, void* stream) {
  if (!d_vectors || !d_angles || n < 0) return PWA_E_ARG;
  if (n == 0) return PWA_OK;
  cudaStream_t st = (cudaStream_t)stream;
  pwa::gen::k_angles_from_vectors<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(d_vectors, n, d_angles);
  return cudaStreamSynchronize(st) == cudaSuccess ? PWA_OK : PWA_E_CUDA;
}
int pwa_events_from_unit(const double* d_x, int64_t ldx, int64_t n, float* d_pp, float* d_pp1, float* d_pp2,
                         int64_t n_size, int64_t col0, float w, int data, double* d_flat, void* stream) {
  if (!d_x || !d_pp || !d_pp1 || !d_pp2 || n < 0 || ldx < n || col0 < 0 || col0 + n > n_size) return PWA_E_ARG;
  if (n == 0) return PWA_OK;
  if (pwa::gen::init_tables()) return PWA_E_CUDA;
  double area, max_len;
  pwa::gen::dalitz_area(&area, &max_len);
  cudaStream_t st = (cudaStream_t)stream;
  pwa::gen::k_events_from_unit<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
      d_x, ldx, n, d_pp, d_pp1, d_pp2, n_size, col0, w, data, d_flat, (pwa::gen::S2_HI - pwa::gen::S2_LO) / area);
  return cudaStreamSynchronize(st) == cudaSuccess ? PWA_OK : PWA_E_CUDA;
}

int pwa_unit_flat(int64_t n, uint64_t seed, uint64_t first_id, double* d_x, int64_t ldx, void* stream) {
  if (!d_x || n < 0 || ldx < n) return PWA_E_ARG;
  if (n == 0) return PWA_OK;
  double area, max_len;
  pwa::gen::dalitz_area(&area, &max_len);
  cudaStream_t st = (cudaStream_t)stream;
  pwa::gen::k_unit_flat<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, seed, first_id, d_x, ldx, max_len);
  return cudaStreamSynchronize(st) == cudaSuccess ? PWA_OK : PWA_E_CUDA;
}
}
