// Learned proposal density for toy generation and importance-sampled normalisation integrals.
//
// An autoregressive network (MADE masks) over unit coordinates x in [0,1]^7 of the Lambda_b ->
// J/psi(-> mu mu) p K- phase space (pwa_events_from_unit maps x to an event): q(x) =
// prod_d 64 softmax(logits_d(x_<d))[floor(64 x_d)].  Trained on the GPU by weighted maximum
// likelihood on flat phase-space events weighted by the amplitude (loss -sum_i w_i log q(x_i) /
// sum_i w_i), with the project's own forward and backward kernels: every matrix product is a tcgen05
// BF16 GEMM with FP32 accumulation in TMEM (pwa_flow_gemm.cuh), the epilogues fuse bias, SiLU, the
// softmax loss and its gradient (pwa_flow_epi.cuh); Adam on FP32 master weights.
// No counterpart in the reference, whose toys come from flat hit-or-miss
// (gen_toys/create_efficiency/hit_and_reject.py:40-50).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "../../include/pwa_b200.h"
#include "pwa_flow_epi.cuh"
#include "pwa_flow_gemm.cuh"
#include "pwa_kernels.cuh"

namespace pwa {
namespace flow {

// ------------------------------------------------------------------ element-wise kernels
// Network input of n events: u = F(x) through the pre-maps, 2 u - 1 in columns 0..6 (row-major and
// feature-major), the target bins of u, the weights normalised by their sum (*wsum), and (lq0) the
// pre-maps' log Jacobian sum_d log F_d'(x_d), the part of log q(x) outside the network.
__global__ void k_pack(const double* __restrict__ x, int64_t ldx, const double* __restrict__ pm,
                       const double* __restrict__ w, const double* wsum, int n, int ldT, bf16* xin, bf16* xinT,
                       uint8_t* bins, float* wn, float* lq0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  alignas(16) bf16 row[FLOW_IN];
#pragma unroll
  for (int c = 0; c < FLOW_IN; ++c) row[c] = __float2bfloat16(0.0f);
  double lpm = 0;
  for (int d = 0; d < FLOW_D; ++d) {
    double logf;
    const double ud = pm_forward(pm + d * PM_NODES, x[(size_t)d * ldx + i], &logf);
    lpm += logf;
    row[d] = __float2bfloat16((float)(2.0 * ud - 1.0));
    bins[(size_t)i * 8 + d] = (uint8_t)min(FLOW_BINS - 1, max(0, (int)floor(ud * FLOW_BINS)));
  }
  bins[(size_t)i * 8 + 7] = 0;
  for (int c = 0; c < FLOW_IN; ++c) xinT[(size_t)c * ldT + i] = row[c];
  const uint4* s = reinterpret_cast<const uint4*>(row);
  uint4* d = reinterpret_cast<uint4*>(xin + (size_t)i * FLOW_IN);
#pragma unroll
  for (int q = 0; q < FLOW_IN / 8; ++q) d[q] = s[q];
  if (wn) wn[i] = (float)(w[i] / *wsum);
  if (lq0) lq0[i] = (float)lpm;
}

// Weighted histograms of the n events' coordinates on the pre-map cells (hist [D][PM_BINS], added
// to): per block in shared memory, then once into global memory.
__global__ void k_hist(const double* __restrict__ x, int64_t ldx, const double* __restrict__ w, int64_t n,
                       double* hist) {
  extern __shared__ double sh[];  // [D][PM_BINS]
  for (int j = threadIdx.x; j < FLOW_D * PM_BINS; j += blockDim.x) sh[j] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double wi = w[i];
    for (int d = 0; d < FLOW_D; ++d) {
      const int k = min(PM_BINS - 1, max(0, (int)floor(x[(size_t)d * ldx + i] * PM_BINS)));
      atomicAdd(&sh[d * PM_BINS + k], wi);
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < FLOW_D * PM_BINS; j += blockDim.x)
    if (sh[j] != 0) atomicAdd(&hist[j], sh[j]);
}

__global__ void k_sum(const double* __restrict__ a, int n, double* out) {
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// loss = -sum_i wn_i logq_i
__global__ void k_loss(const float* __restrict__ wn, const float* __restrict__ logq, int n, double* out) {
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s -= (double)wn[i] * (double)logq[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// Bias gradient: out[r] = sum over the n columns of row r of a feature-major matrix.
__global__ void k_rowsum(const bf16* __restrict__ t, int ld, int n, float* out) {
  const bf16* row = t + (size_t)blockIdx.x * ld;
  float s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += __bfloat162float(row[i]);
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
  }
}

// Adam on FP32 master parameters with the autoregressive mask (masked entries stay zero).
__global__ void k_adam(float* p, float* m, float* v, const float* __restrict__ g, const float* __restrict__ mask,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] * mask[i];
  const float mi = b1 * m[i] + (1 - b1) * gi;
  const float vi = b2 * v[i] + (1 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] = (p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps)) * mask[i];
}

// BF16 copies of a weight matrix [rows x cols]: row-major (forward B operand) and transposed
// (backward B operand).
__global__ void k_pack_weight(const float* __restrict__ W, int rows, int cols, bf16* Wb, bf16* WTb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const bf16 b = __float2bfloat16(W[i]);
  Wb[i] = b;
  if (WTb) WTb[(size_t)c * rows + r] = b;
}

// ------------------------------------------------------------------ host side
using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeFn encoder() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  });
  return fn;
}

// Tensor map of a row-major BF16 matrix [rows x cols] (leading dimension ld elements) read in
// boxes of box_rows x 64 columns with 128-byte swizzling.
bool make_map(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows) {
  EncodeFn enc = encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {ld * sizeof(bf16)};
  const cuuint32_t box[2] = {GEMM_BK, box_rows};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct Layer {
  int out = 0, in = 0;
  float *W = nullptr, *mW = nullptr, *vW = nullptr, *gW = nullptr, *maskW = nullptr;
  float *b = nullptr, *mb = nullptr, *vb = nullptr, *gb = nullptr, *maskb = nullptr;
  bf16 *Wb = nullptr, *WTb = nullptr;
  CUtensorMap mapW, mapWT;  // B operands: W [out x in] (forward), W^T [in x out] (backward)
};

// MADE degrees: hidden unit k has degree 1 + k mod (D - 1); input column c < D is dimension c + 1.
inline int degree(int k) { return 1 + k % (FLOW_D - 1); }

}  // namespace flow
}  // namespace pwa

using namespace pwa;
using namespace pwa::flow;

struct pwa_flow {
  int device = 0, max_batch = 0;
  cudaStream_t st = nullptr;
  Layer L[FLOW_LAYERS];
  // activations of up to max_batch rows
  bf16 *xin = nullptr, *xinT = nullptr, *z[4] = {}, *h[4] = {}, *hT[4] = {}, *dlog = nullptr, *dlogT = nullptr,
       *dz[2] = {}, *dzT = nullptr;
  uint8_t* bins = nullptr;
  float *wn = nullptr, *logq = nullptr;
  double *acc = nullptr, *xs = nullptr;  // acc[0] weight sum, acc[1] loss
  double* pm = nullptr;                  // pre-maps [D][PM_NODES]
  int* err = nullptr;
  CUtensorMap mxin, mxinT, mh[4], mhT[4], mdlog, mdlogT, mdz[2], mdzT;
  int64_t step = 0;
  std::vector<void*> owned;
};

namespace {

constexpr int LAYER_OUT[FLOW_LAYERS] = {FLOW_H, FLOW_H, FLOW_H, FLOW_H, FLOW_OUT};
constexpr int LAYER_IN[FLOW_LAYERS] = {FLOW_IN, FLOW_H, FLOW_H, FLOW_H, FLOW_H};

template <class T>
cudaError_t dalloc(pwa_flow* f, T** p, size_t count) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
  if (e == cudaSuccess) {
    f->owned.push_back(*p);
    e = cudaMemsetAsync(*p, 0, count * sizeof(T), f->st);
  }
  return e;
}

template <int BN, class Epi>
cudaError_t gemm(pwa_flow* f, const CUtensorMap& A, const CUtensorMap& B, int M, int n_tiles, int K, int splits,
                 const Epi& epi, int n_tile0 = 0) {
  using S = GemmShape<BN>;
  static bool configured = false;
  cudaError_t e;
  if (!configured) {
    if ((e = cudaFuncSetAttribute(k_gemm<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM)))
      return e;
    configured = true;
  }
  const int kb_total = K / GEMM_BK;
  const int kb_per = (kb_total + splits - 1) / splits;
  splits = (kb_total + kb_per - 1) / kb_per;  // no empty split
  const dim3 grid((M + GEMM_BM - 1) / GEMM_BM, n_tiles, splits);
  k_gemm<BN, Epi><<<grid, 128, S::SMEM, f->st>>>(A, B, kb_per, kb_total, n_tile0, epi, f->err);
  return cudaGetLastError();
}

// Forward through the hidden layers of n rows (xin filled); keep = store z and h^T for a backward pass.
cudaError_t forward_hidden(pwa_flow* f, int n, bool keep) {
  cudaError_t e;
  for (int l = 0; l < 4; ++l) {
    EpiHidden epi{f->L[l].b, f->h[l], keep ? f->hT[l] : nullptr, keep ? f->z[l] : nullptr, n, f->max_batch};
    const CUtensorMap& A = (l == 0) ? f->mxin : f->mh[l - 1];
    if ((e = gemm<256>(f, A, f->L[l].mapW, n, 1, LAYER_IN[l], 1, epi))) return e;
  }
  return cudaSuccess;
}

int check_err(pwa_flow* f) {
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, f->err, sizeof(int), cudaMemcpyDeviceToHost, f->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->st);
  if (e != cudaSuccess) return cuda_fail(e);
  return h ? PWA_E_STATE : PWA_OK;
}

// Loss and all gradients of the weighted maximum-likelihood objective on n rows (n a multiple of 128).
cudaError_t loss_and_grads(pwa_flow* f, const double* d_x, int64_t ldx, const double* d_w, int n) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(f->acc, 0, 2 * sizeof(double), f->st))) return e;
  k_sum<<<64, 256, 0, f->st>>>(d_w, n, f->acc);
  k_pack<<<(n + 255) / 256, 256, 0, f->st>>>(d_x, ldx, f->pm, d_w, f->acc, n, f->max_batch, f->xin, f->xinT,
                                              f->bins, f->wn, f->logq);
  if ((e = forward_hidden(f, n, true))) return e;
  EpiOutput out{f->L[4].b, f->bins, f->wn, f->dlog, f->dlogT, f->logq, n, f->max_batch, 1};
  if ((e = gemm<256>(f, f->mh[3], f->L[4].mapW, n, 2, FLOW_H, 1, out))) return e;
  k_loss<<<64, 256, 0, f->st>>>(f->wn, f->logq, n, f->acc + 1);
  for (int l = 0; l < FLOW_LAYERS; ++l) {
    if ((e = cudaMemsetAsync(f->L[l].gW, 0, (size_t)LAYER_OUT[l] * LAYER_IN[l] * sizeof(float), f->st))) return e;
  }
  const int splits = std::max(1, n / (16 * GEMM_BK));  // 16 K blocks (1024 rows) per split
  // output layer: dh4 = dlog Wo -> dz4; dWo = dlog^T h4; dbo = column sums of dlog
  {
    EpiBackward bw{f->z[3], f->dz[0], f->dzT, n, f->max_batch};
    if ((e = gemm<256>(f, f->mdlog, f->L[4].mapWT, n, 1, FLOW_OUT, 1, bw))) return e;
    EpiWgrad wg{f->L[4].gW, FLOW_OUT, FLOW_H};
    if ((e = gemm<256>(f, f->mdlogT, f->mhT[3], FLOW_OUT, 1, n, splits, wg))) return e;
    k_rowsum<<<FLOW_OUT, 256, 0, f->st>>>(f->dlogT, f->max_batch, n, f->L[4].gb);
  }
  // hidden layers 4, 3, 2: dW_l = dz_l^T h_{l-1}; dz_{l-1} = (dz_l W_l) silu'(z_{l-1})
  int cur = 0;
  for (int l = 3; l >= 1; --l) {
    EpiWgrad wg{f->L[l].gW, FLOW_H, FLOW_H};
    if ((e = gemm<256>(f, f->mdzT, f->mhT[l - 1], FLOW_H, 1, n, splits, wg))) return e;
    k_rowsum<<<FLOW_H, 256, 0, f->st>>>(f->dzT, f->max_batch, n, f->L[l].gb);
    EpiBackward bw{f->z[l - 1], f->dz[1 - cur], f->dzT, n, f->max_batch};
    if ((e = gemm<256>(f, f->mdz[cur], f->L[l].mapWT, n, 1, FLOW_H, 1, bw))) return e;
    cur = 1 - cur;
  }
  // input layer: dW1 = dz1^T xin
  EpiWgrad wg{f->L[0].gW, FLOW_H, FLOW_IN};
  if ((e = gemm<64>(f, f->mdzT, f->mxinT, FLOW_H, 1, n, splits, wg))) return e;
  k_rowsum<<<FLOW_H, 256, 0, f->st>>>(f->dzT, f->max_batch, n, f->L[0].gb);
  return cudaSuccess;
}

cudaError_t repack(pwa_flow* f) {
  for (int l = 0; l < FLOW_LAYERS; ++l) {
    const int n = LAYER_OUT[l] * LAYER_IN[l];
    k_pack_weight<<<(n + 255) / 256, 256, 0, f->st>>>(f->L[l].W, LAYER_OUT[l], LAYER_IN[l], f->L[l].Wb,
                                                        l > 0 ? f->L[l].WTb : nullptr);
  }
  return cudaGetLastError();
}

}  // namespace

extern "C" int64_t pwa_flow_param_count(void) {
  int64_t n = 0;
  for (int l = 0; l < FLOW_LAYERS; ++l) n += (int64_t)LAYER_OUT[l] * LAYER_IN[l] + LAYER_OUT[l];
  return n;
}

extern "C" int pwa_flow_destroy(pwa_flow* f) {
  if (!f) return PWA_OK;
  cudaSetDevice(f->device);
  if (f->st) cudaStreamSynchronize(f->st);
  for (void* p : f->owned) cudaFree(p);
  if (f->st) cudaStreamDestroy(f->st);
  delete f;
  return PWA_OK;
}

extern "C" int pwa_flow_create(int device, int max_batch, uint64_t seed, pwa_flow** out) {
  if (!out || max_batch < 128 || max_batch % 128) return PWA_E_ARG;
  *out = nullptr;
  if (!encoder()) return PWA_E_UNSUPPORTED;
  pwa_flow* f = new pwa_flow();
  f->device = device;
  f->max_batch = max_batch;
  cudaError_t e = cudaSetDevice(device);
  // a blocking stream: ordered with the legacy default stream, on which callers (torch by default)
  // write the events and weights a call reads and free its inputs afterwards
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&f->st, cudaStreamDefault);
  const size_t B = (size_t)max_batch;
  auto fail = [&](cudaError_t err) {
    pwa_flow_destroy(f);
    return cuda_fail(err);
  };
  if (e) return fail(e);
  // parameters: W ~ N(0, 1 / (unmasked fan-in)), biases 0, autoregressive masks
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  for (int l = 0; l < FLOW_LAYERS; ++l) {
    Layer& L = f->L[l];
    L.out = LAYER_OUT[l];
    L.in = LAYER_IN[l];
    const size_t nw = (size_t)L.out * L.in;
    float** bufs[] = {&L.W, &L.mW, &L.vW, &L.gW, &L.maskW};
    for (float** b : bufs)
      if ((e = dalloc(f, b, nw))) return fail(e);
    float** bbufs[] = {&L.b, &L.mb, &L.vb, &L.gb, &L.maskb};
    for (float** b : bbufs)
      if ((e = dalloc(f, b, (size_t)L.out))) return fail(e);
    if ((e = dalloc(f, &L.Wb, nw))) return fail(e);
    if (l > 0 && (e = dalloc(f, &L.WTb, nw))) return fail(e);
    std::vector<float> W(nw), M(nw), Mb(L.out, 1.0f);
    for (int r = 0; r < L.out; ++r) {
      int fan = 0;
      for (int c = 0; c < L.in; ++c) {
        bool keep;
        if (l == 0)
          keep = c < FLOW_D && degree(r) >= c + 1;
        else if (l < 4)
          keep = degree(r) >= degree(c);
        else
          keep = (r / FLOW_BINS) < FLOW_D && (r / FLOW_BINS) + 1 > degree(c);
        M[(size_t)r * L.in + c] = keep ? 1.0f : 0.0f;
        fan += keep;
      }
      if (l == 4 && r / FLOW_BINS >= FLOW_D) Mb[r] = 0.0f;
      const float sd = fan ? 1.0f / std::sqrt((float)fan) : 0.0f;
      for (int c = 0; c < L.in; ++c) W[(size_t)r * L.in + c] = M[(size_t)r * L.in + c] * sd * nd(rng);
    }
    if ((e = cudaMemcpyAsync(L.W, W.data(), nw * 4, cudaMemcpyHostToDevice, f->st)) ||
        (e = cudaMemcpyAsync(L.maskW, M.data(), nw * 4, cudaMemcpyHostToDevice, f->st)) ||
        (e = cudaMemcpyAsync(L.maskb, Mb.data(), L.out * 4, cudaMemcpyHostToDevice, f->st)) ||
        (e = cudaStreamSynchronize(f->st)))
      return fail(e);
    if (!make_map(&L.mapW, L.Wb, L.out, L.in, L.in, L.out > 256 ? 256 : L.out)) return fail(cudaErrorInvalidValue);
    if (l > 0 && !make_map(&L.mapWT, L.WTb, L.in, L.out, L.out, 256)) return fail(cudaErrorInvalidValue);
  }
  // activations
  if ((e = dalloc(f, &f->xin, B * FLOW_IN)) || (e = dalloc(f, &f->xinT, (size_t)FLOW_IN * B)) ||
      (e = dalloc(f, &f->dlog, B * FLOW_OUT)) || (e = dalloc(f, &f->dlogT, (size_t)FLOW_OUT * B)) ||
      (e = dalloc(f, &f->dzT, (size_t)FLOW_H * B)) || (e = dalloc(f, &f->bins, B * 8)) ||
      (e = dalloc(f, &f->wn, B)) || (e = dalloc(f, &f->logq, B)) || (e = dalloc(f, &f->acc, 2)) ||
      (e = dalloc(f, &f->err, 1)) || (e = dalloc(f, &f->pm, (size_t)FLOW_D * PM_NODES)))
    return fail(e);
  {  // identity pre-maps
    std::vector<double> id((size_t)FLOW_D * PM_NODES);
    for (int d = 0; d < FLOW_D; ++d)
      for (int k = 0; k < PM_NODES; ++k) id[(size_t)d * PM_NODES + k] = (double)k / PM_BINS;
    if ((e = cudaMemcpyAsync(f->pm, id.data(), id.size() * sizeof(double), cudaMemcpyHostToDevice, f->st)) ||
        (e = cudaStreamSynchronize(f->st)))
      return fail(e);
  }
  for (int l = 0; l < 4; ++l)
    if ((e = dalloc(f, &f->z[l], B * FLOW_H)) || (e = dalloc(f, &f->h[l], B * FLOW_H)) ||
        (e = dalloc(f, &f->hT[l], (size_t)FLOW_H * B)))
      return fail(e);
  for (int k = 0; k < 2; ++k)
    if ((e = dalloc(f, &f->dz[k], B * FLOW_H))) return fail(e);
  bool ok = make_map(&f->mxin, f->xin, B, FLOW_IN, FLOW_IN, GEMM_BM) &&
            make_map(&f->mxinT, f->xinT, FLOW_IN, B, B, 64) &&
            make_map(&f->mdlog, f->dlog, B, FLOW_OUT, FLOW_OUT, GEMM_BM) &&
            make_map(&f->mdlogT, f->dlogT, FLOW_OUT, B, B, GEMM_BM) &&
            make_map(&f->mdzT, f->dzT, FLOW_H, B, B, GEMM_BM);
  for (int l = 0; l < 4 && ok; ++l)
    ok = make_map(&f->mh[l], f->h[l], B, FLOW_H, FLOW_H, GEMM_BM) && make_map(&f->mhT[l], f->hT[l], FLOW_H, B, B, 256);
  for (int k = 0; k < 2 && ok; ++k) ok = make_map(&f->mdz[k], f->dz[k], B, FLOW_H, FLOW_H, GEMM_BM);
  if (!ok) return fail(cudaErrorInvalidValue);
  if ((e = repack(f)) || (e = cudaStreamSynchronize(f->st))) return fail(e);
  *out = f;
  return PWA_OK;
}

// One Adam step on the weighted maximum-likelihood loss of n events (x: device doubles [7][ldx] in
// [0,1), w: device doubles [n]); *loss receives the batch loss before the step.
extern "C" int pwa_flow_train_step(pwa_flow* f, const double* d_x, int64_t ldx, const double* d_w, int n, float lr,
                                   double* loss) {
  if (!f || !d_x || !d_w || n < 128 || n > f->max_batch || n % 128 || ldx < n) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  if (e || (e = loss_and_grads(f, d_x, ldx, d_w, n))) return cuda_fail(e);
  ++f->step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)f->step), c2 = 1.0f - std::pow(b2, (float)f->step);
  for (int l = 0; l < FLOW_LAYERS; ++l) {
    Layer& L = f->L[l];
    const int nw = L.out * L.in;
    k_adam<<<(nw + 255) / 256, 256, 0, f->st>>>(L.W, L.mW, L.vW, L.gW, L.maskW, nw, lr, b1, b2, 1e-8f, c1, c2);
    k_adam<<<(L.out + 255) / 256, 256, 0, f->st>>>(L.b, L.mb, L.vb, L.gb, L.maskb, L.out, lr, b1, b2, 1e-8f, c1, c2);
  }
  if ((e = repack(f))) return cuda_fail(e);
  if (loss && (e = cudaMemcpyAsync(loss, f->acc + 1, sizeof(double), cudaMemcpyDeviceToHost, f->st))) return cuda_fail(e);
  return check_err(f);
}

// Loss and gradients without an update; h_grad (optional, pwa_flow_param_count floats) receives
// them layer by layer (weights [out x in] row-major, then biases).
extern "C" int pwa_flow_gradients(pwa_flow* f, const double* d_x, int64_t ldx, const double* d_w, int n, double* loss,
                                  float* h_grad) {
  if (!f || !d_x || !d_w || n < 128 || n > f->max_batch || n % 128 || ldx < n) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  if (e || (e = loss_and_grads(f, d_x, ldx, d_w, n))) return cuda_fail(e);
  if (loss && (e = cudaMemcpyAsync(loss, f->acc + 1, sizeof(double), cudaMemcpyDeviceToHost, f->st))) return cuda_fail(e);
  size_t o = 0;
  for (int l = 0; l < FLOW_LAYERS && h_grad; ++l) {
    const size_t nw = (size_t)LAYER_OUT[l] * LAYER_IN[l];
    if ((e = cudaMemcpyAsync(h_grad + o, f->L[l].gW, nw * 4, cudaMemcpyDeviceToHost, f->st)) ||
        (e = cudaMemcpyAsync(h_grad + o + nw, f->L[l].gb, LAYER_OUT[l] * 4, cudaMemcpyDeviceToHost, f->st)))
      return cuda_fail(e);
    o += nw + LAYER_OUT[l];
  }
  return check_err(f);
}

// log q(x) of n events (any n; processed in chunks of max_batch) into d_logq (device floats).
extern "C" int pwa_flow_log_density(pwa_flow* f, const double* d_x, int64_t ldx, int64_t n, float* d_logq) {
  if (!f || !d_x || !d_logq || n < 0 || ldx < n) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  if (e) return cuda_fail(e);
  for (int64_t c0 = 0; c0 < n; c0 += f->max_batch) {
    const int m = (int)std::min<int64_t>(f->max_batch, n - c0);
    const int mp = (m + 127) / 128 * 128;
    k_pack<<<(m + 255) / 256, 256, 0, f->st>>>(d_x + c0, ldx, f->pm, nullptr, nullptr, m, f->max_batch, f->xin,
                                                f->xinT, f->bins, nullptr, d_logq + c0);
    if ((e = forward_hidden(f, mp, false))) return cuda_fail(e);
    EpiOutput out{f->L[4].b, f->bins, nullptr, nullptr, nullptr, d_logq + c0, m, f->max_batch, 0};
    if ((e = gemm<256>(f, f->mh[3], f->L[4].mapW, mp, 2, FLOW_H, 1, out))) return cuda_fail(e);
  }
  return check_err(f);
}

// n events drawn from q: x into device doubles [7][ldx], log q(x) into d_logq.  Seeded, counter-based:
// event i of a call is a function of (seed, i).
extern "C" int pwa_flow_sample(pwa_flow* f, int64_t n, uint64_t seed, double* d_x, int64_t ldx, float* d_logq) {
  if (!f || !d_x || !d_logq || n < 0 || ldx < n) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  if (e) return cuda_fail(e);
  for (int64_t c0 = 0; c0 < n; c0 += f->max_batch) {
    const int m = (int)std::min<int64_t>(f->max_batch, n - c0);
    const int mp = (m + 127) / 128 * 128;
    if ((e = cudaMemsetAsync(f->xin, 0, (size_t)mp * FLOW_IN * sizeof(bf16), f->st)) ||
        (e = cudaMemsetAsync(d_logq + c0, 0, m * sizeof(float), f->st)))
      return cuda_fail(e);
    for (int d = 0; d < FLOW_D; ++d) {
      if ((e = forward_hidden(f, mp, false))) return cuda_fail(e);
      EpiSample smp{f->L[4].b, d_x + c0, f->xin, f->bins, d_logq + c0, f->pm, seed, c0, m, (int)ldx, d};
      if ((e = gemm<256>(f, f->mh[3], f->L[4].mapW, mp, 1, FLOW_H, 1, smp, d / 4))) return cuda_fail(e);
    }
  }
  return check_err(f);
}

extern "C" int pwa_flow_get_params(pwa_flow* f, float* h_params) {
  if (!f || !h_params) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  size_t o = 0;
  for (int l = 0; l < FLOW_LAYERS && e == cudaSuccess; ++l) {
    const size_t nw = (size_t)LAYER_OUT[l] * LAYER_IN[l];
    e = cudaMemcpyAsync(h_params + o, f->L[l].W, nw * 4, cudaMemcpyDeviceToHost, f->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_params + o + nw, f->L[l].b, LAYER_OUT[l] * 4, cudaMemcpyDeviceToHost, f->st);
    o += nw + LAYER_OUT[l];
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->st);
  return e == cudaSuccess ? PWA_OK : cuda_fail(e);
}

// Sets the FP32 parameters (same layout); masked entries are zeroed.
extern "C" int pwa_flow_set_params(pwa_flow* f, const float* h_params) {
  if (!f || !h_params) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  size_t o = 0;
  for (int l = 0; l < FLOW_LAYERS && e == cudaSuccess; ++l) {
    const size_t nw = (size_t)LAYER_OUT[l] * LAYER_IN[l];
    e = cudaMemcpyAsync(f->L[l].W, h_params + o, nw * 4, cudaMemcpyHostToDevice, f->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f->L[l].b, h_params + o + nw, LAYER_OUT[l] * 4, cudaMemcpyHostToDevice, f->st);
    // a zero-learning-rate Adam step applies the masks without moving the parameters
    k_adam<<<((int)nw + 255) / 256, 256, 0, f->st>>>(f->L[l].W, f->L[l].mW, f->L[l].vW, f->L[l].gW, f->L[l].maskW,
                                                     (int)nw, 0.0f, 1.0f, 1.0f, 1.0f, 1.0f, 1.0f);
    o += nw + LAYER_OUT[l];
  }
  if (e == cudaSuccess) e = repack(f);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->st);
  return e == cudaSuccess ? PWA_OK : cuda_fail(e);
}

// Fits the pre-maps to the weighted marginals of n events (x: device doubles [7][ldx], w: device
// doubles [n], w >= 0): F_d' = (1 - mix) x (the weighted histogram of x_d on PM_BINS cells, normalised)
// + mix (a uniform floor that keeps F strictly increasing).  The network's input changes with the
// pre-maps: fit them before training.
extern "C" int pwa_flow_fit_premap(pwa_flow* f, const double* d_x, int64_t ldx, const double* d_w, int64_t n,
                                   double mix) {
  if (!f || !d_x || !d_w || n < 1 || ldx < n || !(mix > 0.0 && mix <= 1.0)) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  if (e) return cuda_fail(e);
  const size_t cells = (size_t)FLOW_D * PM_BINS;
  double* d_hist = nullptr;
  if ((e = cudaMalloc(&d_hist, cells * sizeof(double)))) return cuda_fail(e);
  std::vector<double> hist(cells), cdf((size_t)FLOW_D * PM_NODES);
  const int smem = (int)(cells * sizeof(double));
  e = cudaFuncSetAttribute(k_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_hist, 0, cells * sizeof(double), f->st);
  if (e == cudaSuccess) {
    k_hist<<<296, 512, smem, f->st>>>(d_x, ldx, d_w, n, d_hist);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(hist.data(), d_hist, cells * sizeof(double), cudaMemcpyDeviceToHost, f->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->st);
  cudaFree(d_hist);
  if (e) return cuda_fail(e);
  for (int d = 0; d < FLOW_D; ++d) {
    const double* h = hist.data() + (size_t)d * PM_BINS;
    double tot = 0;
    for (int k = 0; k < PM_BINS; ++k) tot += h[k];
    if (!(tot > 0) || !std::isfinite(tot)) return PWA_E_ARG;
    double* c = cdf.data() + (size_t)d * PM_NODES;
    c[0] = 0;
    for (int k = 0; k < PM_BINS; ++k) c[k + 1] = c[k] + (1.0 - mix) * h[k] / tot + mix / PM_BINS;
    for (int k = 1; k < PM_BINS; ++k) c[k] /= c[PM_BINS];
    c[PM_BINS] = 1.0;
  }
  if ((e = cudaMemcpyAsync(f->pm, cdf.data(), cdf.size() * sizeof(double), cudaMemcpyHostToDevice, f->st)) ||
      (e = cudaStreamSynchronize(f->st)))
    return cuda_fail(e);
  return PWA_OK;
}

// The pre-maps' nodes (host doubles [7][PWA_FLOW_PREMAP_NODES]).
extern "C" int pwa_flow_get_premap(pwa_flow* f, double* h_cdf) {
  if (!f || !h_cdf) return PWA_E_ARG;
  cudaError_t e = cudaSetDevice(f->device);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h_cdf, f->pm, (size_t)FLOW_D * PM_NODES * sizeof(double), cudaMemcpyDeviceToHost, f->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->st);
  return e == cudaSuccess ? PWA_OK : cuda_fail(e);
}

// Sets them (each row: 0 first, 1 last, strictly increasing; anything else is refused).
extern "C" int pwa_flow_set_premap(pwa_flow* f, const double* h_cdf) {
  if (!f || !h_cdf) return PWA_E_ARG;
  for (int d = 0; d < FLOW_D; ++d) {
    const double* c = h_cdf + (size_t)d * PM_NODES;
    if (c[0] != 0.0 || c[PM_BINS] != 1.0) return PWA_E_ARG;
    for (int k = 0; k < PM_BINS; ++k)
      if (!(c[k + 1] > c[k])) return PWA_E_ARG;
  }
  cudaError_t e = cudaSetDevice(f->device);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(f->pm, h_cdf, (size_t)FLOW_D * PM_NODES * sizeof(double), cudaMemcpyHostToDevice, f->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->st);
  return e == cudaSuccess ? PWA_OK : cuda_fail(e);
}
