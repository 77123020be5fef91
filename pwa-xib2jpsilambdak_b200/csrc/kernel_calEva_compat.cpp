// The reference's GPU boundary with its exact C++ signatures (RooTDalitz/kernel_calEva.h:20-27),
// implemented on the C ABI of pwa_b200.h.  See include/kernel_calEva_compat.h for semantics.
#include "../../include/kernel_calEva_compat.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <map>
#include <mutex>

#include "../../include/pwa_b200.h"

namespace {

// One context per device, re-bound when the caller passes different planes or band counts
// (the reference keeps these as file-scope globals, kernel_calEva.cu:76-80).
struct Bound {
  pwa_ctx* ctx = nullptr;
  const float *pp = nullptr, *pp1 = nullptr, *pp2 = nullptr, *sw = nullptr;
  const float *pp3 = nullptr, *pp4 = nullptr;
  long n = -1, nda = -1, smr = -1, fine = -1;
};
std::mutex g_mu;
std::map<int, Bound> g_bound;

// DEVICE_NUM = 1 and iDevice = 0, as the reference's Makefile builds it (Makefile:11-13); the
// device is the caller's current device.
int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

void report(const char* where, int rc) {
  std::fprintf(stderr, "%s: %s (%s)\n", where, pwa_error_string(rc), pwa_last_cuda_error());
}

Bound* bind(const float* pp, const float* pp1, const float* pp2, const float* sw, long n, long nda, long smr,
            long fine, int* rc) {
  const int dev = current_device();
  Bound& b = g_bound[dev];
  if (!b.ctx) {
    *rc = pwa_ctx_create(dev, &b.ctx);
    if (*rc) return nullptr;
  }
  if (b.pp != pp || b.pp1 != pp1 || b.pp2 != pp2 || b.sw != sw || b.n != n || b.nda != nda || b.smr != smr ||
      b.fine != fine) {
    const long n_size = (n / 32 + 1) * 32;
    *rc = pwa_ctx_set_device_events(b.ctx, pp, pp1, pp2, sw, n, n_size, nda, smr, fine);
    if (*rc) {
      b.pp = nullptr;
      return nullptr;
    }
    b.pp3 = b.pp4 = nullptr;
    b.pp = pp;
    b.pp1 = pp1;
    b.pp2 = pp2;
    b.sw = sw;
    b.n = n;
    b.nda = nda;
    b.smr = smr;
    b.fine = fine;
  }
  *rc = 0;
  return &b;
}

// Zcs planes (the reference's d_float_pp3 / d_float_pp4), attached when the model has Zcs entries.
int bind_zcs(Bound* b, const std::vector<float*>& pp3, const std::vector<float*>& pp4, int NUMZcs) {
  if (NUMZcs <= 0) return 0;
  if (pp3.size() != 1 || pp4.size() != 1 || !pp3[0] || !pp4[0]) return PWA_E_ARG;
  if (b->pp3 == pp3[0] && b->pp4 == pp4[0]) return 0;
  const int rc = pwa_ctx_set_device_zcs_events(b->ctx, pp3[0], pp4[0]);
  if (rc) return rc;
  b->pp3 = pp3[0];
  b->pp4 = pp4[0];
  return 0;
}

}  // namespace

void cu_malloc_h_pp(float* h_float_pp, float*& d_float_pp, int mem_length, int device) {
  d_float_pp = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return;
  if (cudaMalloc((void**)&d_float_pp, mem_length > 0 ? mem_length : 1) != cudaSuccess) {
    d_float_pp = nullptr;
    std::fprintf(stderr, "cu_malloc_h_pp: allocation of %d bytes failed\n", mem_length);
    return;
  }
  if (mem_length > 0) cudaMemcpy(d_float_pp, h_float_pp, mem_length, cudaMemcpyHostToDevice);
}

void cu_Free_pp(std::vector<float*> a, std::vector<float*> b, std::vector<float*> c, std::vector<float*> d,
                std::vector<float*> e) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto* v : {&a, &b, &c, &d, &e})
    for (float* p : *v)
      if (p) cudaFree(p);
  for (auto& kv : g_bound) pwa_ctx_destroy(kv.second.ctx);
  g_bound.clear();
}

double host_store_fx(std::vector<float*> d_float_pp, std::vector<float*> d_float_pp1,
                     std::vector<float*> d_float_pp2, std::vector<float*> d_float_pp3,
                     std::vector<float*> d_float_pp4, std::vector<float*> d_float_sw, float* h_paraList, int para_size, int vamp_size,
                     int paraSpline_size, double* h_fx, int end, int begin, int Nda, int Nda_SMR,
                     int Nda_SMR_finebinning, int NUMLz, int NUMPc, int NUMZcs, double& mynll, double SumW,
                     double sumW_data, float _FFR, float _FFB, bool store_h_fx) {
  const double nan = std::numeric_limits<double>::quiet_NaN();
  std::lock_guard<std::mutex> lk(g_mu);
  if (d_float_pp.size() != 1 || d_float_pp1.size() != 1 || d_float_pp2.size() != 1 || d_float_sw.size() != 1 ||
      begin != 0) {
    std::fprintf(stderr, "host_store_fx: one device and begin = 0 are supported\n");
    mynll = nan;
    return nan;
  }
  int rc = 0;
  Bound* b = bind(d_float_pp[0], d_float_pp1[0], d_float_pp2[0], d_float_sw[0], end, Nda, Nda_SMR,
                  Nda_SMR_finebinning, &rc);
  if (b) rc = bind_zcs(b, d_float_pp3, d_float_pp4, NUMZcs);
  if (!b || rc) {
    report("host_store_fx", rc);
    mynll = nan;
    return nan;
  }
  pwa_result r;
  rc = pwa_ctx_eval_nll(b->ctx, h_paraList, para_size, vamp_size, paraSpline_size, NUMLz, NUMPc, NUMZcs, _FFR,
                        _FFB, SumW, sumW_data, 10000000.0, &r, (store_h_fx && h_fx) ? h_fx : nullptr);
  if (rc) {
    report("host_store_fx", rc);
    mynll = nan;
    return nan;
  }
  if (std::getenv("PWA_COMPAT_PRINT_SUMINT")) std::printf("SUMINT:%g\n", r.sumint);
  mynll = r.nll;
  return r.sumint;
}

void cuda_configure_Pc_KMatrix(const float*) {}
void cuda_configure_ampcount(const float*, const int) {}
void cuda_configure_smear() {}

void host_store_amp2s(std::vector<float*> d_float_pp, std::vector<float*> d_float_pp1,
                      std::vector<float*> d_float_pp2, std::vector<float*> d_float_pp3,
                      std::vector<float*> d_float_pp4, float* h_paraList,
                      int para_size, int vamp_size, int paraSpline_size, double* h_amp2s, int end, int begin,
                      int NUMLz, int NUMPc, int NUMZcs, float _FFR, float _FFB) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (d_float_pp.size() != 1 || begin != 0) {
    std::fprintf(stderr, "host_store_amp2s: one device and begin = 0 are supported\n");
    return;
  }
  pwa_ctx* ctx = nullptr;
  int rc = pwa_ctx_create(current_device(), &ctx);
  if (!rc) {
    const long n_size = (end / 32 + 1) * 32;
    rc = pwa_ctx_set_device_events(ctx, d_float_pp[0], d_float_pp1[0], d_float_pp2[0], nullptr, end, n_size, 0, -1,
                                   0);
  }
  if (!rc && NUMZcs > 0) {
    if (d_float_pp3.size() != 1 || d_float_pp4.size() != 1)
      rc = PWA_E_ARG;
    else
      rc = pwa_ctx_set_device_zcs_events(ctx, d_float_pp3[0], d_float_pp4[0]);
  }
  if (!rc)
    rc = pwa_ctx_amp2(ctx, h_paraList, para_size, vamp_size, paraSpline_size, NUMLz, NUMPc, NUMZcs, _FFR, _FFB,
                      h_amp2s);
  if (rc) report("host_store_amp2s", rc);
  pwa_ctx_destroy(ctx);
}

void host_store_lineshapeLsKM(const float* h_mkp, float* h_KM_real, float* h_KM_imag, float* h_BW_real,
                              float* h_BW_imag, const int n_points, const int NR, const int nLz, const float _FFR,
                              float* h_paraList, const int para_size, const int vamp_size,
                              const int paraSpline_size) {
  (void)vamp_size;
  (void)paraSpline_size;
  if (nLz < NR) {
    std::fprintf(stderr, "host_store_lineshapeLsKM: %d output rows for %d Lambda* entries\n", nLz, NR);
    return;
  }
  const size_t n = (size_t)n_points * (size_t)(NR > 0 ? NR : 0);
  std::vector<double> buf(4 * n);
  const int rc = pwa_lineshapes_lstar_km(current_device(), h_mkp, n_points, NR, _FFR, h_paraList, para_size,
                                         buf.data(), buf.data() + n, buf.data() + 2 * n, buf.data() + 3 * n);
  if (rc) {
    report("host_store_lineshapeLsKM", rc);
    return;
  }
  float* outs[4] = {h_KM_real, h_KM_imag, h_BW_real, h_BW_imag};
  for (int k = 0; k < 4; ++k)
    for (size_t i = 0; i < n; ++i) outs[k][i] = (float)buf[k * n + i];
}
