// C ABI (include/pwa_b200.h): contexts, event upload and one-call likelihood evaluation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pwa_b200.h"
#include "pwa_kernels.cuh"

using namespace pwa;

namespace pwa {
cudaError_t configure_kernels();
}

namespace {
thread_local std::string g_last_cuda = "no error";
}  // namespace

namespace pwa {
// Records the message of a failed CUDA call for pwa_last_cuda_error and maps it to a status code.
int cuda_fail(cudaError_t e) {
  g_last_cuda = cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? PWA_E_NOMEM : PWA_E_CUDA;
}
}  // namespace pwa

namespace {
#define PWA_CUDA(x)                      \
  do {                                   \
    cudaError_t _e = (x);                \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)

// m(J/psi p) windows of the 20-offset smearing of the normalisation kernel
// (kernel_calEva.cu:874), tested on the float mass as the reference does.
inline bool in_window(float mz) { return (mz > 4.4 && mz < 4.48) || (mz > 4.27 && mz < 4.34); }
}  // namespace

struct pwa_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // events
  const float *pp = nullptr, *pp1 = nullptr, *pp2 = nullptr, *sw = nullptr;
  float *own_pp = nullptr, *own_pp1 = nullptr, *own_pp2 = nullptr, *own_sw = nullptr;
  const float *pp3 = nullptr, *pp4 = nullptr;  // Zcs chain planes (models with Zcs entries)
  float *own_pp3 = nullptr, *own_pp4 = nullptr;
  int64_t n = 0, n_size = 0, nda = 0, nda_smr = 0, nda_fine = 0;
  // selected data events [win_first, win_first + win_n) (win_n < 0: all data, the default); the band
  // arguments then count from win_first
  int64_t win_first = 0, win_n = -1;
  // resolution model: PWA_SMEAR_REFERENCE, or PWA_SMEAR_GAUSS with (offset, weight) pairs on the device
  int smear_mode = PWA_SMEAR_REFERENCE;
  double* d_grid = nullptr;
  int grid_nb = 0;
  int32_t* d_lists = nullptr;
  std::vector<Segment> segs;
  std::vector<int> seg_off;
  std::vector<int64_t> seg_defer_off;  // segment's region of d_defer
  // events the table-only pass defers to the exact pass: n slots, one counter per segment (+ amp2)
  int32_t* d_defer = nullptr;
  int* d_defer_cnt = nullptr;
  int total_parts = 0;
  // per evaluation
  PointTable* d_table = nullptr;
  PointTable* h_table = nullptr;
  Partial* d_parts = nullptr;
  EvalResult* d_res = nullptr;
  EvalResult* h_res = nullptr;
  double* d_fx = nullptr;
  int64_t fx_cap = 0;
  double last_ms = 0;
  int last_launches = 0;
  // K-matrix lineshape tables (on by default)
  int use_tables = 1;
  // order of the per-class event lists (MC window / tail): 1 by m(J/psi p), 0 by event index
  int mass_order = 0;
  // build_point_table flags (K-matrix variant)
  int build_flags = 0;
  // launch shape of the batched passes per event class (Smear kind): waves of resident blocks
  int batch_waves[SMEAR_KINDS] = {1, 1, 1, 1, 1};
  void* d_tab = nullptr;  // TAB_BYTES of two-level lineshape tables
  // optional per-segment timing
  int timing = 0;
  std::vector<cudaEvent_t> seg_ev;
  std::vector<double> seg_ms;
  int h_defer_cnt[8] = {};  // deferred events per segment of the last timed evaluation
  // data uploaded unsorted: device position i < nda holds the caller's data event order[i]
  std::vector<int32_t> order;
  // batched evaluation (grow-only buffers)
  std::vector<void*> bt_tabs;        // lineshape tables of points that move a Pc lineshape
  PointTable* d_btables = nullptr;   // decoded tables of the points of one launch
  BatchPoint* d_bpts = nullptr;
  cplx* d_bdc = nullptr;             // coupling differences, 8 x 24 per point
  EvalResult* d_bres = nullptr;
  EvalResult* h_bres = nullptr;      // pinned
  Partial* d_bparts = nullptr;
  size_t bparts_cap = 0;
  double last_batch_ms = 0;
  std::vector<cudaEvent_t> bseg_ev;  // batched evaluation timing: start and end event per segment
  std::vector<double> bseg_ms;       // device time per segment of the last batch call (timing on)
};

namespace {

// Segment lists and the buffers sized by the segments.
void free_segments(pwa_ctx* c) {
  cudaFree(c->d_lists);
  cudaFree(c->d_parts);
  cudaFree(c->d_defer);
  cudaFree(c->d_defer_cnt);
  c->d_lists = nullptr;
  c->d_parts = nullptr;
  c->d_defer = nullptr;
  c->d_defer_cnt = nullptr;
  c->segs.clear();
  c->seg_off.clear();
  c->seg_defer_off.clear();
}

void free_events(pwa_ctx* c) {
  cudaFree(c->own_pp);
  cudaFree(c->own_pp1);
  cudaFree(c->own_pp2);
  cudaFree(c->own_sw);
  cudaFree(c->own_pp3);
  cudaFree(c->own_pp4);
  c->own_pp3 = c->own_pp4 = nullptr;
  c->pp3 = c->pp4 = nullptr;
  free_segments(c);
  c->own_pp = c->own_pp1 = c->own_pp2 = c->own_sw = nullptr;
  c->pp = c->pp1 = c->pp2 = c->sw = nullptr;
  c->order.clear();
  c->n = 0;
  c->win_first = 0;
  c->win_n = -1;
}

// Per-event outputs of the device order back into the caller's order (data uploaded unsorted).
void to_caller_order(const pwa_ctx* c, double* h) {
  if (c->order.empty()) return;
  std::vector<double> t(h, h + c->order.size());
  for (size_t i = 0; i < c->order.size(); ++i) h[c->order[i]] = t[i];
}

int build_reference_segments(pwa_ctx* c, const float* h_mz);

// Splits the events into the reference's kernel ranges (fake_kernel_store_fx,
// kernel_calEva.cu:920-961, begin = 0) and classifies the tail by the 20-offset window; with the
// Gaussian resolution model, one segment of all events on the weighted grid.
int build_segments(pwa_ctx* c, const float* h_mz) {
  const int64_t n = c->n;
  if (c->smear_mode == PWA_SMEAR_GAUSS) {
    c->segs.clear();
    auto grid_segment = [&](int64_t b, int64_t e) {
      if (e <= b) return;
      Segment g{SMEAR_GRID, b, e, nullptr};
      g.grid = c->d_grid;
      g.grid_nb = c->grid_nb;
      c->segs.push_back(g);
    };
    if (c->win_n < 0) {
      grid_segment(0, n);
    } else {
      grid_segment(c->win_first, c->win_first + c->win_n);
      grid_segment(c->nda, n);
    }
  } else {
    const int rc = build_reference_segments(c, h_mz);
    if (rc) return rc;
  }
  c->seg_off.clear();
  c->seg_defer_off.clear();
  int tot = 0;
  int64_t doff = 0;
  for (auto& s : c->segs) {
    c->seg_off.push_back(tot);
    tot += segment_parts(s, c->sm_count, true);
    c->seg_defer_off.push_back(doff);
    doff += s.end - s.begin;
  }
  c->total_parts = std::max(tot, 1);
  PWA_CUDA(cudaMalloc(&c->d_parts, c->total_parts * sizeof(Partial)));
  PWA_CUDA(cudaMemset(c->d_parts, 0, c->total_parts * sizeof(Partial)));
  PWA_CUDA(cudaMalloc(&c->d_defer, std::max<int64_t>(n, 1) * sizeof(int32_t)));
  PWA_CUDA(cudaMalloc(&c->d_defer_cnt, 8 * sizeof(int)));
  return PWA_OK;
}

int build_reference_segments(pwa_ctx* c, const float* h_mz) {
  const int64_t n = c->n;
  std::vector<int32_t> lw, lu;
  int64_t b1s = 0, b1e, b2s, b2e;
  if (c->win_n < 0) {
    b1e = std::max<int64_t>(0, std::min(n, c->nda_smr));
    b2s = std::max<int64_t>(0, c->nda_smr);
    b2e = std::max<int64_t>(b2s, std::min(n, c->nda_smr + c->nda_fine));
    const int64_t r0 = std::min(n, std::max<int64_t>(0, c->nda_smr + c->nda_fine));
    lw.reserve(n / 4);
    lu.reserve(n - r0);
    for (int64_t e = r0; e < n; ++e) (in_window(h_mz[e]) ? lw : lu).push_back((int32_t)e);
  } else {
    // a window of the data: its bands counted from its first event, its tail with all MC events
    const int64_t f = c->win_first, wn = c->win_n;
    b1s = f;
    b1e = f + std::max<int64_t>(0, std::min(wn, c->nda_smr));
    b2s = f + std::max<int64_t>(0, std::min(wn, c->nda_smr));
    b2e = std::max<int64_t>(b2s, f + std::min(wn, c->nda_smr + c->nda_fine));
    const int64_t r0 = f + std::min(wn, std::max<int64_t>(0, c->nda_smr + c->nda_fine));
    for (int64_t e = r0; e < f + wn; ++e) (in_window(h_mz[e]) ? lw : lu).push_back((int32_t)e);
    for (int64_t e = c->nda; e < n; ++e) (in_window(h_mz[e]) ? lw : lu).push_back((int32_t)e);
  }
  if (c->mass_order) {
    // neighbouring list positions then read neighbouring nodes of the lineshape tables
    auto by_mass = [&](int32_t x, int32_t y) { return h_mz[x] < h_mz[y]; };
    std::stable_sort(lw.begin(), lw.end(), by_mass);
    std::stable_sort(lu.begin(), lu.end(), by_mass);
  }
  const size_t nl = lw.size() + lu.size();
  if (nl) {
    PWA_CUDA(cudaMalloc(&c->d_lists, nl * sizeof(int32_t)));
    if (!lw.empty()) PWA_CUDA(cudaMemcpy(c->d_lists, lw.data(), lw.size() * 4, cudaMemcpyHostToDevice));
    if (!lu.empty())
      PWA_CUDA(cudaMemcpy(c->d_lists + lw.size(), lu.data(), lu.size() * 4, cudaMemcpyHostToDevice));
  }
  c->segs.clear();
  // heaviest work first so the long tiles start early
  if (b2e > b2s) c->segs.push_back({SMEAR_150, b2s, b2e, nullptr});
  if (b1e > b1s) c->segs.push_back({SMEAR_30, b1s, b1e, nullptr});
  if (!lw.empty()) c->segs.push_back({SMEAR_20, 0, (int64_t)lw.size(), c->d_lists});
  if (!lu.empty()) c->segs.push_back({SMEAR_NONE, 0, (int64_t)lu.size(), c->d_lists + lw.size()});
  return PWA_OK;
}

}  // namespace

int pwa::ctx_view(const pwa_ctx* c, CtxView* v) {
  if (!c || !v) return PWA_E_ARG;
  *v = CtxView{c->device, c->sm_count, c->st, c->pp, c->pp1, c->pp2, c->sw, c->pp3, c->pp4, c->n, c->n_size,
               c->nda, c->smear_mode == PWA_SMEAR_GAUSS ? 1 : 0, c->d_grid, c->grid_nb, c->use_tables,
               c->build_flags};
  return c->pp ? PWA_OK : PWA_E_STATE;
}

namespace {

int check_events(int64_t n, int64_t n_size, int64_t nda) {
  if (n < 0 || nda < 0 || nda > n || n_size < n || n > INT32_MAX) return PWA_E_ARG;
  return PWA_OK;
}

}  // namespace

extern "C" {

const char* pwa_error_string(int code) {
  switch (code) {
    case PWA_OK: return "ok";
    case PWA_E_CUDA: return "CUDA runtime error";
    case PWA_E_ARG: return "invalid argument";
    case PWA_E_LAYOUT: return "parameter block layout inconsistent with the resonance table";
    case PWA_E_SIZE: return "model size exceeds the compiled maximum";
    case PWA_E_UNSUPPORTED: return "lineshape type or decay chain not supported";
    case PWA_E_PARAM: return "invalid resonance parameters";
    case PWA_E_STATE: return "no events uploaded (or no Zcs planes for a model with Zcs entries)";
    case PWA_E_NOMEM: return "device allocation failed";
  }
  return "unknown error";
}

const char* pwa_last_cuda_error(void) { return g_last_cuda.c_str(); }

int pwa_ctx_create(int device, pwa_ctx** out) {
  if (!out) return PWA_E_ARG;
  *out = nullptr;
  pwa_ctx* c = new pwa_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = configure_kernels();
  // a blocking stream: ordered with the legacy default stream, on which callers (torch by default)
  // write the device events a context borrows and free the memory it reads
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamDefault);
  if (e == cudaSuccess) e = cudaEventCreate(&c->e0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->e1);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_table, sizeof(PointTable));
  if (e == cudaSuccess) e = cudaMallocHost(&c->h_table, sizeof(PointTable));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_res, sizeof(EvalResult));
  if (e == cudaSuccess) e = cudaMallocHost(&c->h_res, sizeof(EvalResult));
  if (e != cudaSuccess) {
    pwa_ctx_destroy(c);
    return cuda_fail(e);
  }
  *out = c;
  return PWA_OK;
}

int pwa_ctx_destroy(pwa_ctx* c) {
  if (!c) return PWA_OK;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  for (void* t : c->bt_tabs) cudaFree(t);
  cudaFree(c->d_btables);
  cudaFree(c->d_bpts);
  cudaFree(c->d_bdc);
  cudaFree(c->d_bres);
  cudaFree(c->d_bparts);
  cudaFreeHost(c->h_bres);
  free_events(c);
  cudaFree(c->d_grid);
  cudaFree(c->d_table);
  cudaFreeHost(c->h_table);
  cudaFree(c->d_res);
  cudaFreeHost(c->h_res);
  cudaFree(c->d_fx);
  cudaFree(c->d_tab);
  for (auto e : c->seg_ev) cudaEventDestroy(e);
  for (auto e : c->bseg_ev) cudaEventDestroy(e);
  if (c->e0) cudaEventDestroy(c->e0);
  if (c->e1) cudaEventDestroy(c->e1);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return PWA_OK;
}

int pwa_ctx_upload_events(pwa_ctx* c, const float* pp, const float* pp1, const float* pp2, const float* sw,
                          int64_t n, int64_t n_size, int64_t nda, int64_t nda_smr, int64_t nda_fine) {
  if (!c || !pp || !pp1 || !pp2 || (nda > 0 && !sw)) return PWA_E_ARG;
  int rc = check_events(n, n_size, nda);
  if (rc) return rc;
  PWA_CUDA(cudaSetDevice(c->device));
  free_events(c);
  const size_t ns = (size_t)n_size;
  PWA_CUDA(cudaMalloc(&c->own_pp, 111 * ns * sizeof(float)));
  PWA_CUDA(cudaMalloc(&c->own_pp1, 96 * ns * sizeof(float)));
  PWA_CUDA(cudaMalloc(&c->own_pp2, 96 * ns * sizeof(float)));
  PWA_CUDA(cudaMalloc(&c->own_sw, ns * sizeof(float)));
  PWA_CUDA(cudaMemcpy(c->own_pp, pp, 111 * ns * sizeof(float), cudaMemcpyHostToDevice));
  PWA_CUDA(cudaMemcpy(c->own_pp1, pp1, 96 * ns * sizeof(float), cudaMemcpyHostToDevice));
  PWA_CUDA(cudaMemcpy(c->own_pp2, pp2, 96 * ns * sizeof(float), cudaMemcpyHostToDevice));
  if (sw)
    PWA_CUDA(cudaMemcpy(c->own_sw, sw, ns * sizeof(float), cudaMemcpyHostToDevice));
  else
    PWA_CUDA(cudaMemset(c->own_sw, 0, ns * sizeof(float)));
  c->pp = c->own_pp;
  c->pp1 = c->own_pp1;
  c->pp2 = c->own_pp2;
  c->sw = c->own_sw;
  c->n = n;
  c->n_size = n_size;
  c->nda = nda;
  c->nda_smr = nda_smr;
  c->nda_fine = nda_fine;
  return build_segments(c, pp + n_size);
}

int pwa_band_order(const float* mz, int64_t nda, int32_t* order, int64_t* n_band1, int64_t* n_band2) {
  if ((nda > 0 && (!mz || !order)) || nda < 0 || !n_band1 || !n_band2) return PWA_E_ARG;
  // reOrder.C: (4.2, 4.43) U (4.47, 4.6), then (4.43, 4.47), then the rest, order kept inside each
  auto band = [](double m) {
    if ((m > 4.2 && m < 4.43) || (m > 4.47 && m < 4.6)) return 1;
    if (m > 4.43 && m < 4.47) return 2;
    return 3;
  };
  int64_t k = 0, n1 = 0, n2 = 0;
  for (int b = 1; b <= 3; ++b)
    for (int64_t i = 0; i < nda; ++i)
      if (band((double)mz[i]) == b) {
        order[k++] = (int32_t)i;
        n1 += b == 1;
        n2 += b == 2;
      }
  *n_band1 = n1;
  *n_band2 = n2;
  return PWA_OK;
}

int pwa_ctx_upload_events_unsorted(pwa_ctx* c, const float* pp, const float* pp1, const float* pp2, const float* sw,
                                   int64_t n, int64_t n_size, int64_t nda) {
  if (!c || !pp || !pp1 || !pp2 || (nda > 0 && !sw)) return PWA_E_ARG;
  int rc = check_events(n, n_size, nda);
  if (rc) return rc;
  std::vector<int32_t> order((size_t)nda);
  int64_t n1 = 0, n2 = 0;
  if ((rc = pwa_band_order(pp + n_size, nda, order.data(), &n1, &n2))) return rc;
  // host copies with the data columns in band order (MC columns as given)
  auto permute = [&](const float* src, int planes) {
    std::vector<float> dst(src, src + (size_t)planes * n_size);
    for (int p = 0; p < planes; ++p)
      for (int64_t i = 0; i < nda; ++i) dst[(size_t)p * n_size + i] = src[(size_t)p * n_size + order[i]];
    return dst;
  };
  const std::vector<float> a = permute(pp, 111), b = permute(pp1, 96), d = permute(pp2, 96);
  std::vector<float> w;
  if (sw) w = permute(sw, 1);
  // the reference's caller passes the band-1 count minus one (RooDalitzAmplitude.cxx:1943-1946)
  if ((rc = pwa_ctx_upload_events(c, a.data(), b.data(), d.data(), sw ? w.data() : nullptr, n, n_size, nda,
                                  n1 - 1, n2)))
    return rc;
  c->order = std::move(order);
  return PWA_OK;
}

int pwa_ctx_set_device_events(pwa_ctx* c, const float* d_pp, const float* d_pp1, const float* d_pp2,
                              const float* d_sw, int64_t n, int64_t n_size, int64_t nda, int64_t nda_smr,
                              int64_t nda_fine) {
  if (!c || !d_pp || !d_pp1 || !d_pp2 || (nda > 0 && !d_sw)) return PWA_E_ARG;
  int rc = check_events(n, n_size, nda);
  if (rc) return rc;
  PWA_CUDA(cudaSetDevice(c->device));
  free_events(c);
  c->pp = d_pp;
  c->pp1 = d_pp1;
  c->pp2 = d_pp2;
  c->sw = d_sw;
  c->n = n;
  c->n_size = n_size;
  c->nda = nda;
  c->nda_smr = nda_smr;
  c->nda_fine = nda_fine;
  std::vector<float> mz((size_t)std::max<int64_t>(n, 1));
  if (n) PWA_CUDA(cudaMemcpy(mz.data(), d_pp + n_size, n * sizeof(float), cudaMemcpyDeviceToHost));
  return build_segments(c, mz.data());
}

int pwa_ctx_set_smearing(pwa_ctx* c, int mode, double sigma, double step, int half_bins) {
  if (!c) return PWA_E_ARG;
  if (mode != PWA_SMEAR_REFERENCE && mode != PWA_SMEAR_GAUSS) return PWA_E_ARG;
  PWA_CUDA(cudaSetDevice(c->device));
  if (mode == PWA_SMEAR_GAUSS) {
    if (!(sigma > 0) || !(step > 0) || half_bins < 0 || 2 * half_bins + 1 > GRID_MAX_NB) return PWA_E_ARG;
    const int nb = 2 * half_bins + 1;
    std::vector<double> g(2 * nb);
    double sum = 0;
    for (int b = 0; b < nb; ++b) {
      const double off = (b - half_bins) * step;
      g[2 * b] = off;
      g[2 * b + 1] = std::exp(-0.5 * (off / sigma) * (off / sigma));
      sum += g[2 * b + 1];
    }
    for (int b = 0; b < nb; ++b) g[2 * b + 1] /= sum;
    if (!c->d_grid) PWA_CUDA(cudaMalloc(&c->d_grid, 2 * GRID_MAX_NB * sizeof(double)));
    PWA_CUDA(cudaMemcpy(c->d_grid, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->grid_nb = nb;
  }
  c->smear_mode = mode;
  if (!c->pp) return PWA_OK;
  // re-split the uploaded events for the new model
  free_segments(c);
  std::vector<float> mz((size_t)std::max<int64_t>(c->n, 1));
  if (c->n) PWA_CUDA(cudaMemcpy(mz.data(), c->pp + c->n_size, c->n * sizeof(float), cudaMemcpyDeviceToHost));
  return build_segments(c, mz.data());
}

int pwa_ctx_set_batch_waves(pwa_ctx* c, int kind, int waves) {
  if (!c || kind < 0 || kind >= SMEAR_KINDS || waves < 1 || waves > 64) return PWA_E_ARG;
  c->batch_waves[kind] = waves;
  return PWA_OK;
}

int pwa_ctx_set_kmatrix(pwa_ctx* c, int kmatrix) {
  if (!c) return PWA_E_ARG;
  if (kmatrix != PWA_KMATRIX_DEFAULT && kmatrix != PWA_KMATRIX_ISOSPIN) return PWA_E_ARG;
  c->build_flags = kmatrix == PWA_KMATRIX_ISOSPIN ? BUILD_KM_ISOSPIN : 0;
  return PWA_OK;
}

int pwa_ctx_set_event_order(pwa_ctx* c, int by_mass) {
  if (!c) return PWA_E_ARG;
  c->mass_order = by_mass ? 1 : 0;
  if (!c->pp) return PWA_OK;
  PWA_CUDA(cudaSetDevice(c->device));
  free_segments(c);
  std::vector<float> mz((size_t)std::max<int64_t>(c->n, 1));
  if (c->n) PWA_CUDA(cudaMemcpy(mz.data(), c->pp + c->n_size, c->n * sizeof(float), cudaMemcpyDeviceToHost));
  return build_segments(c, mz.data());
}

int pwa_ctx_select_data(pwa_ctx* c, int64_t first, int64_t n_data, int64_t nda_smr, int64_t nda_fine) {
  if (!c) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  if (n_data >= 0 && (first < 0 || first + n_data > c->nda)) return PWA_E_ARG;
  PWA_CUDA(cudaSetDevice(c->device));
  c->win_first = n_data >= 0 ? first : 0;
  c->win_n = n_data;
  c->nda_smr = nda_smr;
  c->nda_fine = nda_fine;
  free_segments(c);
  std::vector<float> mz((size_t)std::max<int64_t>(c->n, 1));
  if (c->n) PWA_CUDA(cudaMemcpy(mz.data(), c->pp + c->n_size, c->n * sizeof(float), cudaMemcpyDeviceToHost));
  return build_segments(c, mz.data());
}

int pwa_ctx_upload_zcs_events(pwa_ctx* c, const float* pp3, const float* pp4) {
  if (!c || !pp3 || !pp4) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  PWA_CUDA(cudaSetDevice(c->device));
  cudaFree(c->own_pp3);
  cudaFree(c->own_pp4);
  c->own_pp3 = c->own_pp4 = nullptr;
  c->pp3 = c->pp4 = nullptr;
  const size_t ns = (size_t)c->n_size;
  std::vector<float> a, b;
  if (!c->order.empty()) {  // data uploaded unsorted: the same band order for the Zcs planes
    auto permute = [&](const float* src, int planes, std::vector<float>& dst) {
      dst.assign(src, src + (size_t)planes * ns);
      for (int p = 0; p < planes; ++p)
        for (size_t i = 0; i < c->order.size(); ++i) dst[(size_t)p * ns + i] = src[(size_t)p * ns + c->order[i]];
    };
    permute(pp3, PWA_PP3_PLANES, a);
    permute(pp4, PWA_PP4_PLANES, b);
    pp3 = a.data();
    pp4 = b.data();
  }
  PWA_CUDA(cudaMalloc(&c->own_pp3, PWA_PP3_PLANES * ns * sizeof(float)));
  PWA_CUDA(cudaMalloc(&c->own_pp4, PWA_PP4_PLANES * ns * sizeof(float)));
  PWA_CUDA(cudaMemcpy(c->own_pp3, pp3, PWA_PP3_PLANES * ns * sizeof(float), cudaMemcpyHostToDevice));
  PWA_CUDA(cudaMemcpy(c->own_pp4, pp4, PWA_PP4_PLANES * ns * sizeof(float), cudaMemcpyHostToDevice));
  c->pp3 = c->own_pp3;
  c->pp4 = c->own_pp4;
  return PWA_OK;
}

int pwa_ctx_set_device_zcs_events(pwa_ctx* c, const float* d_pp3, const float* d_pp4) {
  if (!c || !d_pp3 || !d_pp4) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  PWA_CUDA(cudaSetDevice(c->device));
  cudaFree(c->own_pp3);
  cudaFree(c->own_pp4);
  c->own_pp3 = c->own_pp4 = nullptr;
  c->pp3 = d_pp3;
  c->pp4 = d_pp4;
  return PWA_OK;
}

// The event set of an evaluation: the Zcs planes go with it only for a model with Zcs entries
// (they select the kernels with the Zcs terms).
static int event_set(const pwa_ctx* c, int NX, const PointTable& T, EventSet* ev) {
  *ev = EventSet{c->pp, c->pp1, c->pp2, c->sw, c->n_size, c->n, c->nda};
  ev->lgen = lstar_has_general(T);
  if (NX > 0) {
    if (!c->pp3 || !c->pp4) return PWA_E_STATE;
    ev->pp3 = c->pp3;
    ev->pp4 = c->pp4;
  }
  return PWA_OK;
}

// Copies the decoded point table to the device and, with tables on, builds the lineshape tables
// for it on the context's stream.
static int upload_point(pwa_ctx* c, int* launches) {
  if (c->use_tables) {
    if (!c->d_tab) PWA_CUDA(cudaMalloc(&c->d_tab, TAB_BYTES));
    attach_tables(c->h_table, c->d_tab);
  }
  PWA_CUDA(cudaMemcpyAsync(c->d_table, c->h_table, sizeof(PointTable), cudaMemcpyHostToDevice, c->st));
  if (c->h_table->tab.enabled) {
    PWA_CUDA(launch_build_tables(c->d_table, TAB_NODES, c->sm_count, c->st));
    *launches += 4;
  }
  return PWA_OK;
}

int pwa_ctx_eval_nll(pwa_ctx* c, const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                     int NX, float FFR, float FFB, double sum_w_mc, double sum_w_data, double nll_shift,
                     pwa_result* out, double* h_fx) {
  if (!c || !pl || !out) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  int rc = build_point_table(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, c->h_table, c->build_flags);
  if (rc) return rc;
  PWA_CUDA(cudaSetDevice(c->device));
  if (h_fx && c->fx_cap < c->n) {
    cudaFree(c->d_fx);
    c->d_fx = nullptr;
    PWA_CUDA(cudaMalloc(&c->d_fx, std::max<int64_t>(c->n, 1) * sizeof(double)));
    c->fx_cap = c->n;
  }
  EventSet ev;
  if ((rc = event_set(c, NX, *c->h_table, &ev))) return rc;
  PWA_CUDA(cudaEventRecord(c->e0, c->st));
  int launches = 0;
  if ((rc = upload_point(c, &launches))) return rc;
  if (c->timing) {
    while (c->seg_ev.size() < c->segs.size()) {
      cudaEvent_t e;
      PWA_CUDA(cudaEventCreate(&e));
      c->seg_ev.push_back(e);
    }
  }
  const bool defer = c->h_table->tab.enabled != 0;
  // slots of passes that do not run this time must read as zero
  PWA_CUDA(cudaMemsetAsync(c->d_parts, 0, c->total_parts * sizeof(Partial), c->st));
  PWA_CUDA(cudaMemsetAsync(c->d_defer_cnt, 0, 8 * sizeof(int), c->st));
  for (size_t i = 0; i < c->segs.size(); ++i) {
    int32_t* dq = defer ? c->d_defer + c->seg_defer_off[i] : nullptr;
    int* dc = defer ? c->d_defer_cnt + i : nullptr;
    PWA_CUDA(launch_segment(ev, c->segs[i], c->d_table, c->d_parts + c->seg_off[i], h_fx ? c->d_fx : nullptr, dq, dc,
                            c->sm_count, c->st));
    if (c->timing) PWA_CUDA(cudaEventRecord(c->seg_ev[i], c->st));
    launches += defer ? 2 : 1;
  }
  PWA_CUDA(launch_finalize(c->d_parts, c->total_parts, sum_w_mc, sum_w_data, nll_shift, c->d_res, c->st));
  ++launches;
  PWA_CUDA(cudaEventRecord(c->e1, c->st));
  PWA_CUDA(cudaMemcpyAsync(c->h_res, c->d_res, sizeof(EvalResult), cudaMemcpyDeviceToHost, c->st));
  if (h_fx && c->n) PWA_CUDA(cudaMemcpyAsync(h_fx, c->d_fx, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  PWA_CUDA(cudaStreamSynchronize(c->st));
  if (h_fx) to_caller_order(c, h_fx);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->e0, c->e1);
  c->last_ms = ms;
  if (c->timing) {
    c->seg_ms.assign(c->segs.size(), 0.0);
    std::memset(c->h_defer_cnt, 0, sizeof(c->h_defer_cnt));
    if (c->h_table->tab.enabled)
      PWA_CUDA(cudaMemcpy(c->h_defer_cnt, c->d_defer_cnt, sizeof(c->h_defer_cnt), cudaMemcpyDeviceToHost));
    cudaEvent_t prev = c->e0;
    for (size_t i = 0; i < c->segs.size(); ++i) {
      float m = 0;
      cudaEventElapsedTime(&m, prev, c->seg_ev[i]);
      c->seg_ms[i] = m;
      prev = c->seg_ev[i];
    }
  }
  c->last_launches = launches;
  out->nll = c->h_res->nll;
  out->sumint = c->h_res->sumint;
  out->sum_noint = c->h_res->sum_noint;
  out->data_term = c->h_res->data_term;
  out->n_nonpos = (int64_t)c->h_res->n_nonpos;
  return PWA_OK;
}

// Lineshape tables for at most this many points of a batch that move a Pc lineshape; further such
// points are evaluated one by one.
constexpr int BATCH_MAX_TABLES = 128;

int pwa_ctx_eval_nll_batch(pwa_ctx* c, const float* pls, int npoints, int block_stride, int para_size,
                           int vamp_size, int spline_size, int NR, int NZ, int NX, float FFR, float FFB,
                           double sum_w_mc, double sum_w_data, double nll_shift, pwa_result* out,
                           int* n_structured) {
  if (!c || !pls || !out || npoints < 1 || block_stride < para_size + vamp_size + spline_size) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  PWA_CUDA(cudaSetDevice(c->device));
  std::vector<PointTable> H(npoints);
  for (int p = 0; p < npoints; ++p) {
    const int rc = build_point_table(pls + (size_t)p * block_stride, para_size, vamp_size, spline_size, NR, NZ, NX,
                                     FFR, FFB, &H[p], c->build_flags);
    if (rc) return rc;
  }
  // structured points (relative to point 0) and points for the single-point path
  std::vector<BatchPoint> bp(npoints);
  std::vector<cplx> dch((size_t)npoints * 8 * 24);
  std::vector<int> sidx, fidx;
  int ntab = 0;
  for (int p = 0; p < npoints; ++p) {
    bool ok = classify_point(H[0], H[p], &bp[p], dch.data() + (size_t)p * 8 * 24);
    if (ok && bp[p].kind == BP_PCG && c->use_tables) ok = ntab++ < BATCH_MAX_TABLES;
    (ok ? sidx : fidx).push_back(p);
  }
  if (n_structured) *n_structured = (int)sidx.size();
  // lanes of a warp take consecutive points: order them by kind (and group / entry count) so that a
  // warp's 32 points follow one code path; the costliest kind (lineshape points, a pass over the
  // offset rows each) first, so that its points fill whole warps and the partly filled last warp
  // holds cheap points
  auto rank = [](int kind) { return kind == BP_PCG ? 0 : kind == BP_PCC ? 1 : kind == BP_LSTAR ? 2 : 3; };
  std::stable_sort(sidx.begin(), sidx.end(), [&](int a, int b) {
    const BatchPoint &x = bp[a], &y = bp[b];
    if (x.kind != y.kind) return rank(x.kind) < rank(y.kind);
    if (x.kind == BP_PCG) return x.group < y.group;
    if (x.kind == BP_PCC) return x.nq < y.nq;
    return false;
  });
  {
    // a warp whose points differ in kind runs each kind's code: fill the last warp of lineshape points
    // with Lambda* points (the cheapest kind) rather than with coupling points
    const auto is_kind = [&](int k) { return [&, k](int p) { return bp[p].kind == k; }; };
    const auto pcg_end = std::find_if_not(sidx.begin(), sidx.end(), is_kind(BP_PCG));
    const int fill = (32 - (int)((pcg_end - sidx.begin()) % 32)) % 32;
    const auto lst = std::find_if(pcg_end, sidx.end(), is_kind(BP_LSTAR));
    const int nl = (int)std::min<std::ptrdiff_t>(fill, std::count_if(lst, sidx.end(), is_kind(BP_LSTAR)));
    if (fill > 0 && nl > 0) std::rotate(pcg_end, lst, lst + nl);
  }
  const bool tables = c->use_tables != 0 && H[0].NZ > 0;
  const int chunk_cap = BATCH_MAX_POINTS;
  if (!c->d_btables) {
    PWA_CUDA(cudaMalloc(&c->d_btables, (size_t)chunk_cap * sizeof(PointTable)));
    PWA_CUDA(cudaMalloc(&c->d_bpts, (size_t)chunk_cap * sizeof(BatchPoint)));
    PWA_CUDA(cudaMalloc(&c->d_bdc, (size_t)chunk_cap * 8 * 24 * sizeof(cplx)));
    PWA_CUDA(cudaMalloc(&c->d_bres, (size_t)chunk_cap * sizeof(EvalResult)));
    PWA_CUDA(cudaMallocHost(&c->h_bres, (size_t)chunk_cap * sizeof(EvalResult)));
  }
  while (tables && (int)c->bt_tabs.size() < std::min(ntab, BATCH_MAX_TABLES)) {
    void* t = nullptr;
    PWA_CUDA(cudaMalloc(&t, TAB_BYTES_GROUP));
    c->bt_tabs.push_back(t);
  }
  int launches = 0, rc = 0;
  EventSet ev;
  if ((rc = event_set(c, NX, H[0], &ev))) return rc;
  PWA_CUDA(cudaEventRecord(c->e0, c->st));
  // centre: the context's table and lineshape tables
  *c->h_table = H[0];
  if ((rc = upload_point(c, &launches))) return rc;
  const PointTable& T0 = *c->h_table;
  const BatchGroupMap gm = batch_group_map(T0);
  int tab_slot = 0;
  if (c->timing) {
    while (c->bseg_ev.size() < 2 * c->segs.size()) {
      cudaEvent_t e;
      PWA_CUDA(cudaEventCreate(&e));
      c->bseg_ev.push_back(e);
    }
  }
  c->bseg_ms.assign(c->segs.size(), 0.0);
  for (size_t c0 = 0; c0 < sidx.size(); c0 += chunk_cap) {
    const int nc = (int)std::min<size_t>(chunk_cap, sidx.size() - c0);
    std::vector<PointTable> dt(nc);
    std::vector<BatchPoint> dp(nc);
    for (int j = 0; j < nc; ++j) {
      const int p = sidx[c0 + j];
      dt[j] = H[p];  // keeps the point's own guard intervals; tables stay off unless attached here
      if (bp[p].kind == BP_PCG && tables) attach_group_table(&dt[j], bp[p].group, c->bt_tabs[tab_slot++]);
      dp[j] = bp[p];
      dp[j].T = c->d_btables + j;
      dp[j].dc = c->d_bdc + (size_t)j * 8 * 24;
    }
    // neighbouring points that move the same couplings (Minuit's +h and -h of one coupling) are paired
    auto same_couplings = [](const BatchPoint& x, const BatchPoint& y) {
      if (x.kind != y.kind) return false;
      if (x.kind == BP_LSTAR)
        return x.lsmask == 0 && y.lsmask == 0 && x.ldc && y.ldc && x.lmask == y.lmask && x.lcmask == x.lmask &&
               y.lcmask == y.lmask;
      if (x.kind == BP_PCC)
        return x.nq == y.nq && std::memcmp(x.qpos, y.qpos, sizeof(int) * x.nq) == 0 &&
               std::memcmp(x.qsidx, y.qsidx, sizeof(int) * x.nq) == 0;
      return false;
    };
    for (int j = 0; j < nc;) {
      const bool pr = j + 1 < nc && same_couplings(dp[j], dp[j + 1]);
      dp[j].pair = pr ? 1 : 0;
      if (pr) dp[j + 1].pair = 0;
      j += pr ? 2 : 1;
    }
    PWA_CUDA(cudaMemcpyAsync(c->d_btables, dt.data(), nc * sizeof(PointTable), cudaMemcpyHostToDevice, c->st));
    PWA_CUDA(cudaMemcpyAsync(c->d_bpts, dp.data(), nc * sizeof(BatchPoint), cudaMemcpyHostToDevice, c->st));
    std::vector<cplx> dcc((size_t)nc * 8 * 24);
    for (int j = 0; j < nc; ++j)
      std::memcpy(dcc.data() + (size_t)j * 8 * 24, dch.data() + (size_t)sidx[c0 + j] * 8 * 24, 8 * 24 * sizeof(cplx));
    PWA_CUDA(cudaMemcpyAsync(c->d_bdc, dcc.data(), dcc.size() * sizeof(cplx), cudaMemcpyHostToDevice, c->st));
    for (int j = 0; j < nc; ++j)
      if (dt[j].tab.enabled) {
        PWA_CUDA(launch_build_tables(c->d_btables + j, dt[j].tab.n_nodes, c->sm_count, c->st));
        launches += 4;
      }
    // partial rows of all segments
    std::vector<size_t> row_off;
    size_t rows = 0;
    for (auto& sg : c->segs) {
      row_off.push_back(rows);
      rows += batch_segment_rows(sg, T0, gm, nc, c->sm_count, tables, c->batch_waves[sg.kind]);
    }
    if (rows * nc > c->bparts_cap) {
      cudaFree(c->d_bparts);
      c->d_bparts = nullptr;
      PWA_CUDA(cudaMalloc(&c->d_bparts, rows * nc * sizeof(Partial)));
      c->bparts_cap = rows * nc;
    }
    PWA_CUDA(cudaMemsetAsync(c->d_bparts, 0, rows * nc * sizeof(Partial), c->st));
    PWA_CUDA(cudaMemsetAsync(c->d_defer_cnt, 0, 8 * sizeof(int), c->st));
    for (size_t i = 0; i < c->segs.size(); ++i) {
      int32_t* dq = tables ? c->d_defer + c->seg_defer_off[i] : nullptr;
      int* dcnt = tables ? c->d_defer_cnt + i : nullptr;
      if (c->timing) PWA_CUDA(cudaEventRecord(c->bseg_ev[2 * i], c->st));
      PWA_CUDA(launch_batch_segment(ev, c->segs[i], c->d_table, T0, gm, c->d_bpts, nc,
                                    c->d_bparts + row_off[i] * nc, dq, dcnt, c->sm_count, c->st,
                                    c->batch_waves[c->segs[i].kind]));
      if (c->timing) PWA_CUDA(cudaEventRecord(c->bseg_ev[2 * i + 1], c->st));
      launches += tables ? 2 : 1;
    }
    PWA_CUDA(launch_finalize_points(c->d_bparts, (int)std::max<size_t>(rows, 1), nc, sum_w_mc, sum_w_data, nll_shift,
                                    c->d_bres, c->st));
    ++launches;
    PWA_CUDA(cudaMemcpyAsync(c->h_bres, c->d_bres, nc * sizeof(EvalResult), cudaMemcpyDeviceToHost, c->st));
    PWA_CUDA(cudaStreamSynchronize(c->st));
    if (c->timing)
      for (size_t i = 0; i < c->segs.size(); ++i) {
        float m = 0;
        cudaEventElapsedTime(&m, c->bseg_ev[2 * i], c->bseg_ev[2 * i + 1]);
        c->bseg_ms[i] += m;
      }
    for (int j = 0; j < nc; ++j) {
      const EvalResult& r = c->h_bres[j];
      pwa_result& o = out[sidx[c0 + j]];
      o.nll = r.nll;
      o.sumint = r.sumint;
      o.sum_noint = r.sum_noint;
      o.data_term = r.data_term;
      o.n_nonpos = (int64_t)r.n_nonpos;
    }
  }
  PWA_CUDA(cudaEventRecord(c->e1, c->st));
  PWA_CUDA(cudaEventSynchronize(c->e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->e0, c->e1);
  c->last_batch_ms = ms;
  for (int p : fidx) {
    if ((rc = pwa_ctx_eval_nll(c, pls + (size_t)p * block_stride, para_size, vamp_size, spline_size, NR, NZ, NX,
                               FFR, FFB, sum_w_mc, sum_w_data, nll_shift, &out[p], nullptr)))
      return rc;
    c->last_batch_ms += c->last_ms;
    launches += c->last_launches;
  }
  c->last_launches = launches;
  return PWA_OK;
}

double pwa_ctx_last_batch_ms(pwa_ctx* c) { return c ? c->last_batch_ms : 0.0; }

int pwa_ctx_batch_segment_ms(pwa_ctx* c, int i, double* ms) {
  if (!c || !ms || i < 0 || i >= (int)c->segs.size()) return PWA_E_ARG;
  *ms = i < (int)c->bseg_ms.size() ? c->bseg_ms[i] : 0.0;
  return PWA_OK;
}

int pwa_ctx_amp2(pwa_ctx* c, const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                 float FFR, float FFB, double* h_amp2) {
  if (!c || !pl || !h_amp2) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  int rc = build_point_table(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, c->h_table, c->build_flags);
  if (rc) return rc;
  PWA_CUDA(cudaSetDevice(c->device));
  if (c->fx_cap < c->n) {
    cudaFree(c->d_fx);
    c->d_fx = nullptr;
    PWA_CUDA(cudaMalloc(&c->d_fx, std::max<int64_t>(c->n, 1) * sizeof(double)));
    c->fx_cap = c->n;
  }
  EventSet ev;
  if ((rc = event_set(c, NX, *c->h_table, &ev))) return rc;
  int launches = 0;
  if ((rc = upload_point(c, &launches))) return rc;
  const bool defer = c->h_table->tab.enabled != 0;
  if (defer) PWA_CUDA(cudaMemsetAsync(c->d_defer_cnt + 7, 0, sizeof(int), c->st));
  PWA_CUDA(launch_amp2(ev, c->d_table, c->d_fx, defer ? c->d_defer : nullptr, defer ? c->d_defer_cnt + 7 : nullptr,
                       c->sm_count, c->st));
  if (c->n) PWA_CUDA(cudaMemcpyAsync(h_amp2, c->d_fx, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  PWA_CUDA(cudaStreamSynchronize(c->st));
  to_caller_order(c, h_amp2);
  return PWA_OK;
}

int pwa_ctx_mc_integral(pwa_ctx* c, const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                        int NX, float FFR, float FFB, double* integral) {
  if (!c || !pl || !integral) return PWA_E_ARG;
  if (!c->pp) return PWA_E_STATE;
  int rc = build_point_table(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, c->h_table, c->build_flags);
  if (rc) return rc;
  PWA_CUDA(cudaSetDevice(c->device));
  if (c->fx_cap < c->n) {
    cudaFree(c->d_fx);
    c->d_fx = nullptr;
    PWA_CUDA(cudaMalloc(&c->d_fx, std::max<int64_t>(c->n, 1) * sizeof(double)));
    c->fx_cap = c->n;
  }
  EventSet ev;
  if ((rc = event_set(c, NX, *c->h_table, &ev))) return rc;
  int launches = 0;
  if ((rc = upload_point(c, &launches))) return rc;
  const bool defer = c->h_table->tab.enabled != 0;
  if (defer) PWA_CUDA(cudaMemsetAsync(c->d_defer_cnt + 7, 0, sizeof(int), c->st));
  PWA_CUDA(launch_amp2(ev, c->d_table, c->d_fx, defer ? c->d_defer : nullptr, defer ? c->d_defer_cnt + 7 : nullptr,
                       c->sm_count, c->st));
  const int nb = std::max(1, std::min(c->total_parts, 2 * c->sm_count));
  PWA_CUDA(launch_mc_integral(ev, c->d_fx, c->d_parts, nb, c->d_res, c->st));
  PWA_CUDA(cudaMemcpyAsync(c->h_res, c->d_res, sizeof(EvalResult), cudaMemcpyDeviceToHost, c->st));
  PWA_CUDA(cudaStreamSynchronize(c->st));
  *integral = c->h_res->sumint;
  return PWA_OK;
}

int pwa_host_lineshapes(const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                        float FFR, float FFB, double mkp, double mz, double* lstar, double* pc) {
  return pwa_host_lineshapes_km(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, PWA_KMATRIX_DEFAULT, mkp,
                                mz, lstar, pc);
}

int pwa_host_lineshapes_km(const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                           float FFR, float FFB, int kmatrix, double mkp, double mz, double* lstar, double* pc) {
  if (!pl || !lstar || !pc) return PWA_E_ARG;
  if (kmatrix != PWA_KMATRIX_DEFAULT && kmatrix != PWA_KMATRIX_ISOSPIN) return PWA_E_ARG;
  PointTable* T = new PointTable();
  int rc = build_point_table(pl, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, T,
                             kmatrix == PWA_KMATRIX_ISOSPIN ? BUILD_KM_ISOSPIN : 0);
  if (!rc) host_lineshapes(*T, mkp, mz, reinterpret_cast<cplx*>(lstar), reinterpret_cast<cplx*>(pc));
  delete T;
  return rc;
}

double pwa_ctx_last_kernel_ms(pwa_ctx* c) { return c ? c->last_ms : 0.0; }
void* pwa_ctx_stream(pwa_ctx* c) { return c ? (void*)c->st : nullptr; }

int pwa_ctx_set_timing(pwa_ctx* c, int on) {
  if (!c) return PWA_E_ARG;
  c->timing = on ? 1 : 0;
  return PWA_OK;
}

int pwa_ctx_set_lineshape_tables(pwa_ctx* c, int on) {
  if (!c) return PWA_E_ARG;
  c->use_tables = on ? 1 : 0;
  return PWA_OK;
}

int pwa_ctx_segment_count(pwa_ctx* c) { return c ? (int)c->segs.size() : 0; }

int pwa_ctx_segment_info(pwa_ctx* c, int i, int* kind, int64_t* events, double* last_ms) {
  if (!c || i < 0 || i >= (int)c->segs.size()) return PWA_E_ARG;
  if (kind) *kind = c->segs[i].kind;
  if (events) *events = c->segs[i].end - c->segs[i].begin;
  if (last_ms) *last_ms = (i < (int)c->seg_ms.size()) ? c->seg_ms[i] : 0.0;
  return PWA_OK;
}

int pwa_ctx_segment_deferred(pwa_ctx* c, int i, int64_t* deferred) {
  if (!c || !deferred || i < 0 || i >= (int)c->segs.size() || i >= 8) return PWA_E_ARG;
  *deferred = c->timing ? c->h_defer_cnt[i] : 0;
  return PWA_OK;
}

int64_t pwa_point_table_bytes(void) { return (int64_t)sizeof(PointTable); }
int pwa_ctx_last_launches(pwa_ctx* c) { return c ? c->last_launches : 0; }

}  // extern "C"
