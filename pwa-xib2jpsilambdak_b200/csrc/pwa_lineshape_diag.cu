// Lambda* lineshape diagnostic: for every Lambda* entry and mass, the revised K-matrix lineshape (in
// the refactored form of Revised_KMAMP_refactor, cu_DPFPropogator.cu:998-1063) and the Breit-Wigner
// (BW_AMP, :248-314), each times the Lambda_b -> Lambda* J/psi barrier (BTerm, :155-181) with radius
// FFR, exactly as the reference's storeLineshapeLsKM / GetLineshapeLsKM / GetLineshapeLsBW compute them
// (kernel_calEva.cu:1490-1584), for every entry whatever its type.  FP64 on the float parameters.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/pwa_b200.h"
#include "pwa_kernels.cuh"

namespace pwa {
cudaError_t configure_kernels();
}

namespace {

using namespace pwa;

struct Row {
  double m, g;
  int S2, LR, type, P;
};

// The resonance table rows of the Lambda* entries, passed by value.
struct LstarRows {
  float q[MAX_LSTAR * NSET];
};

__device__ __forceinline__ Row row(const LstarRows& t, int r) {
  const float* q = t.q + r * NSET;
  return Row{q[0], q[1], (int)q[2], (int)q[3], (int)q[4], (int)q[5]};
}

__device__ double eff_mass(double m, double thr, double hi) {
  if (m > thr) return m;
  if (m >= 0) return tanh_eff_mass(m, thr, hi);
  return (thr + hi) / 2.0;
}

// BTerm(J, mpp, mr, radius)
__device__ double lb_barrier(int S2, double mpp, double mr, double radius) {
  const double J = 0.5 * S2;
  const int LB = (J <= 1) ? 0 : (int)(J - 1.5);
  const double pB = two_body_p(M_LB, M_JPSI, mpp);
  const double mmin = M_K + M_P, mmax = M_LB - M_JPSI;
  double pB0 = pB;
  if (mr < 0) pB0 = two_body_p(M_LB, M_JPSI, (mmin + mmax) / 2.0);
  if (mr > 1e-10 && mr + M_JPSI < M_LB) pB0 = two_body_p(M_LB, M_JPSI, mr);
  if (mr + M_JPSI > M_LB) pB0 = two_body_p(M_LB, M_JPSI, tanh_eff_mass(mr, mmin, mmax));
  return barrier_ratio(radius, LB, pB, pB0) * ipow(pB / M_LB, LB) * ipow(M_LB / pB0, LB);
}

// BW_AMP
__device__ cplx bw_amp(double m_r, double g_r, double mpp, int LR, double ffr) {
  const double pR = two_body_p(mpp, M_P, M_K);
  const double mmin = M_K + M_P, mmax = M_LB - M_JPSI;
  const double thr = (double)(float)(M_P + M_K);
  double pR0 = pR;
  if (m_r < 0) pR0 = two_body_p((mmin + mmax) / 2.0, M_P, M_K);
  if (m_r > thr) pR0 = two_body_p(m_r, M_P, M_K);
  if (m_r <= thr && m_r > 1e-10) pR0 = two_body_p(tanh_eff_mass(m_r, mmin, mmax), M_P, M_K);
  double FR = barrier_ratio(ffr, LR, pR, pR0);
  if (m_r < 0) return mk(ipow(pR / pR0, LR), 0);
  double gamma = g_r;
  if (m_r > thr) {
    gamma = g_r * ipow(pR / pR0, 2 * LR + 1) * (m_r / mpp) * FR * FR;
  } else if (m_r < PWA_F(1.43f) && m_r > 0) {
    const double pSP = two_body_p(mpp, PWA_F(1.18937f), PWA_F(0.13957018f));
    pR0 = two_body_p(m_r, PWA_F(1.18937f), PWA_F(0.13957018f));
    FR = 1.0;
    gamma = g_r * ipow(pR / pR0, 2 * LR + 1) * (m_r / mpp) + PWA_F(0.0505f) * ipow(pSP / pR0, 2 * LR + 1) * (m_r / mpp);
  }
  return breit_wigner(m_r, gamma, mpp * mpp) * (FR * ipow(pR / pR0, LR) * bw_norm(m_r, g_r));
}

// Revised_KMAMP_refactor for entry nr of the NR Lambda* entries (p K system).
__device__ cplx rkm_refactor(const LstarRows& t, int NR, int nr, double mpp, double ffr) {
  const double s = mpp * mpp, thr = M_P + M_K, hi = M_LB - M_JPSI;
  const Row R = row(t, nr);
  auto prod_delta = [&](int ir, const Row& X) {  // product_delta_S
    double pr = 1;
    for (int j = 0; j < NR; ++j) {
      if (j == ir) continue;
      const Row E = row(t, j);
      if (E.type == X.type && E.S2 == X.S2 && E.P == X.P) pr *= E.m * E.m - s;
    }
    return pr;
  };
  const double pR = two_body_p(mpp, M_P, M_K);
  const double pR0 = two_body_p(eff_mass(R.m, thr, hi), M_P, M_K);
  const double FR = barrier_ratio(ffr, R.LR, pR, pR0);
  const double gamma = R.g * ipow(pR / pR0, 2 * R.LR + 1) * (R.m / mpp) * FR * FR;
  const double pds_r = prod_delta(nr, R);
  const double pds_all = pds_r * (R.m * R.m - s);
  double sum = pds_r * R.m * gamma, fsc = 0;
  for (int ir = 0; ir < NR; ++ir) {
    if (ir == nr) continue;
    const Row E = row(t, ir);
    if (!(E.S2 == R.S2 && E.P == R.P && E.type == R.type)) continue;
    const double q0 = two_body_p(eff_mass(E.m, thr, hi), M_P, M_K);
    const double fr = barrier_ratio(ffr, E.LR, pR, q0);
    const double g = E.g * ipow(pR / q0, 2 * E.LR + 1) * (E.m / mpp) * fr * fr;
    double mg;
    if (E.m < 0) {  // m_gamma of a non-resonant entry: the first one fixes fsc
      if (fabs(fsc) < 1e-10) fsc = g;
      mg = fsc * (E.m * E.m - mpp * mpp);
    } else {
      mg = E.m * g;
    }
    sum += mg * prod_delta(ir, E);
  }
  const double den = pds_all * pds_all + sum * sum;
  const double kr = sqrt(R.m * R.m + R.g * R.g);
  const double factor = FR * ipow(pR / pR0, R.LR) * BW_NORM_C * R.m * sqrt(R.g * kr / sqrt(R.m * (R.m + kr)));
  return mk(pds_r * pds_all / den, pds_r * sum / den) * factor;
}

__global__ void k_lineshapes_lstar(LstarRows t, int NR, double ffr, const float* __restrict__ mkp, int n,
                                   double* km_re, double* km_im, double* bw_re, double* bw_im) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = mkp[i];
  for (int r = 0; r < NR; ++r) {
    const Row R = row(t, r);
    const double bt = lb_barrier(R.S2, m, R.m, ffr);
    const cplx km = rkm_refactor(t, NR, r, m, ffr) * bt;
    const cplx bw = bw_amp(R.m, R.g, m, R.LR, ffr) * bt;
    const size_t o = (size_t)r * n + i;
    km_re[o] = km.re;
    km_im[o] = km.im;
    bw_re[o] = bw.re;
    bw_im[o] = bw.im;
  }
}

}  // namespace

extern "C" int pwa_lineshapes_lstar_km(int device, const float* h_mkp, int n_points, int NR, float FFR,
                                       const float* h_paraList, int para_size, double* km_re, double* km_im,
                                       double* bw_re, double* bw_im) {
  if (!h_mkp || !h_paraList || !km_re || !km_im || !bw_re || !bw_im || n_points < 0 || NR < 0) return PWA_E_ARG;
  if (NR > MAX_LSTAR) return PWA_E_SIZE;
  if (para_size < NSET * NR) return PWA_E_LAYOUT;
  if (n_points == 0 || NR == 0) return PWA_OK;
  LstarRows t{};
  for (int i = 0; i < NSET * NR; ++i) t.q[i] = h_paraList[i];
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e);
  float* d_m = nullptr;
  double* d_out = nullptr;
  const size_t nout = (size_t)NR * n_points;
  if ((e = cudaMalloc(&d_m, n_points * sizeof(float))) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMalloc(&d_out, 4 * nout * sizeof(double))) != cudaSuccess) {
    cudaFree(d_m);
    return cuda_fail(e);
  }
  e = cudaMemcpy(d_m, h_mkp, n_points * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_lineshapes_lstar<<<(n_points + 127) / 128, 128>>>(t, NR, FFR, d_m, n_points, d_out, d_out + nout,
                                                        d_out + 2 * nout, d_out + 3 * nout);
    e = cudaGetLastError();
  }
  double* outs[4] = {km_re, km_im, bw_re, bw_im};
  for (int k = 0; k < 4 && e == cudaSuccess; ++k)
    e = cudaMemcpy(outs[k], d_out + k * nout, nout * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_m);
  cudaFree(d_out);
  return e == cudaSuccess ? PWA_OK : cuda_fail(e);
}
