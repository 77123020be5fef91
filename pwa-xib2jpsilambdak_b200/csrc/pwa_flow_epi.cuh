// Epilogues of the proposal network's GEMMs and the network's element-wise kernels.
//
// The network is an autoregressive density over u in [0,1]^7 (MADE masks): input 2u - 1 padded to 64
// columns, four hidden layers of 256 SiLU units, and 8 x 64 output logits (dimension d's 64 logits
// give the bin probabilities of u_d given u_<d; the eighth block is padding).  q_u(u) =
// prod_d 64 softmax(logits_d)[floor(64 u_d)], a piecewise-constant conditional per dimension.
// Each coordinate first passes a fixed monotone pre-map u_d = F_d(x_d), a piecewise-linear CDF on
// PM_BINS equal cells fitted to the target's marginal (identity until fitted), so that the 64 bins
// are narrow where the marginal is peaked; q(x) = q_u(F(x)) prod_d F_d'(x_d).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace pwa {
namespace flow {

constexpr int FLOW_D = 7;       // dimensions
constexpr int FLOW_BINS = 64;   // bins per dimension
constexpr int FLOW_IN = 64;     // padded input width (one 64-element K block)
constexpr int FLOW_H = 256;     // hidden width
constexpr int FLOW_OUT = 512;   // 8 blocks of 64 logits (the last is padding)
constexpr int FLOW_LAYERS = 5;  // 4 hidden + output
constexpr float LOG_BINS = 4.1588830833596715f;  // log(64)
constexpr int PM_BINS = 1024;   // cells of each coordinate's pre-map
constexpr int PM_NODES = PM_BINS + 1;

using bf16 = __nv_bfloat16;

__device__ __forceinline__ float silu(float t) { return t / (1.0f + __expf(-t)); }
__device__ __forceinline__ float silu_grad(float t) {
  const float s = 1.0f / (1.0f + __expf(-t));
  return s * (1.0f + t * (1.0f - s));
}

__device__ __forceinline__ void store_row32(bf16* dst, const float (&v)[32]) {
  alignas(16) bf16 b[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) b[j] = __float2bfloat16(v[j]);
  const uint4* s = reinterpret_cast<const uint4*>(b);
  uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
  for (int q = 0; q < 4; ++q) d[q] = s[q];
}

// Counter-based uniforms in (0, 1) (splitmix64 finaliser of the key and counter).
__device__ __forceinline__ double hash_uniform(uint64_t key, uint64_t ctr) {
  uint64_t z = key + 0x9E3779B97F4A7C15ull * (ctr + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// Pre-map of one coordinate: u = F(x) with F piecewise linear through cdf[k] at x = k / PM_BINS
// (cdf[0] = 0, cdf[PM_BINS] = 1, strictly increasing); *logf = log F'(x).
__device__ __forceinline__ double pm_forward(const double* __restrict__ cdf, double x, double* logf) {
  double t = x * PM_BINS;
  const int k = min(PM_BINS - 1, max(0, (int)floor(t)));
  t -= k;
  const double a = cdf[k], b = cdf[k + 1];
  *logf = log((b - a) * PM_BINS);
  return a + t * (b - a);
}

// Its inverse: x = F^-1(u) by bisection over the nodes; *logf = log F'(x).
__device__ __forceinline__ double pm_inverse(const double* __restrict__ cdf, double u, double* logf) {
  int lo = 0, hi = PM_BINS;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (cdf[mid] <= u)
      lo = mid;
    else
      hi = mid;
  }
  const double a = cdf[lo], b = cdf[lo + 1];
  *logf = log((b - a) * PM_BINS);
  return (lo + (u - a) / (b - a)) * (1.0 / PM_BINS);
}

struct NoState {};

// Hidden layer forward: z = acc + b; h = silu(z); h row-major (next layer's A operand), h^T
// feature-major (the weight gradient's B operand), z row-major (the backward pass's SiLU derivative).
struct EpiHidden {
  static constexpr int CHUNK = 32;
  using State = NoState;
  const float* bias;
  bf16 *h, *hT, *z;
  int M, ldT;
  __device__ void apply(State&, int row, int col, float (&v)[32]) const {
    if (row >= M) return;
    float zz[32], hh[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      zz[j] = v[j] + bias[col + j];
      hh[j] = silu(zz[j]);
      if (hT) hT[(size_t)(col + j) * ldT + row] = __float2bfloat16(hh[j]);
    }
    store_row32(h + (size_t)row * FLOW_H + col, hh);
    if (z) store_row32(z + (size_t)row * FLOW_H + col, zz);
  }
  __device__ void finish(State&, int) const {}
};

// Output layer.  Per row and dimension d (one 64-column chunk): log of the density factor
// log(64 p_bin) with bin = the row's target bin; mode TRAIN also writes the loss gradient w.r.t. the
// logits, w (softmax - onehot(bin)) (row-major and feature-major), for the weighted maximum-likelihood
// loss -sum w log q with weights w normalised to sum 1; every mode adds the row's log q into logq.
struct EpiOutput {
  static constexpr int CHUNK = 64;
  struct State {
    float lq;
  };
  const float* bias;
  const uint8_t* bins;  // [M][8]
  const float* w;       // [M] (TRAIN)
  bf16 *dlog, *dlogT;   // TRAIN
  float* logq;          // [M], added to (two column tiles contribute)
  int M, ldT, train;
  __device__ void apply(State& st, int row, int col, float (&v)[64]) const {
    const int d = col / FLOW_BINS;
    if (row >= M) return;
    if (d >= FLOW_D) {  // padding block: zero gradient
      if (train) {
        float zero[32] = {};
        store_row32(dlog + (size_t)row * FLOW_OUT + col, zero);
        store_row32(dlog + (size_t)row * FLOW_OUT + col + 32, zero);
        for (int j = 0; j < 64; ++j) dlogT[(size_t)(col + j) * ldT + row] = __float2bfloat16(0.0f);
      }
      return;
    }
    float mx = -3.0e38f;
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      v[j] += bias[col + j];
      mx = fmaxf(mx, v[j]);
    }
    float s = 0;
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      v[j] = __expf(v[j] - mx);
      s += v[j];
    }
    const int b = bins[(size_t)row * 8 + d];
    float pb = 0;
#pragma unroll
    for (int j = 0; j < 64; ++j) pb = (j == b) ? v[j] : pb;
    st.lq += LOG_BINS + __logf(pb / s);
    if (train) {
      const float wr = w[row], inv = 1.0f / s;
      float g[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        g[j] = wr * (v[j] * inv - (j == b ? 1.0f : 0.0f));
        dlogT[(size_t)(col + j) * ldT + row] = __float2bfloat16(g[j]);
      }
      store_row32(dlog + (size_t)row * FLOW_OUT + col, *reinterpret_cast<float(*)[32]>(g));
      store_row32(dlog + (size_t)row * FLOW_OUT + col + 32, *reinterpret_cast<float(*)[32]>(g + 32));
    }
  }
  __device__ void finish(State& st, int row) const {
    if (row < M) atomicAdd(logq + row, st.lq);
  }
};

// Sampling pass of dimension d: bin from the conditional (inverse CDF on a counter-based uniform),
// u_d uniform inside the bin and x_d = F_d^-1(u_d); writes x_d (double [D][ldx]), the network input
// 2 u_d - 1 of later passes, the bin, and adds log(64 p_bin) + log F_d'(x_d) to logq.
struct EpiSample {
  static constexpr int CHUNK = 64;
  using State = NoState;
  const float* bias;
  double* x;      // [D][ldx]
  bf16* xin;      // [M][FLOW_IN]
  uint8_t* bins;  // [M][8]
  float* logq;
  const double* pm;  // pre-maps [D][PM_NODES]
  uint64_t key;
  int64_t row0;   // global index of row 0 (counter base)
  int M, ldx, d;
  __device__ void apply(State&, int row, int col, float (&v)[64]) const {
    if (row >= M || col / FLOW_BINS != d) return;
    float mx = -3.0e38f;
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      v[j] += bias[col + j];
      mx = fmaxf(mx, v[j]);
    }
    float s = 0;
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      v[j] = __expf(v[j] - mx);
      s += v[j];
    }
    const uint64_t ctr = (uint64_t)(row0 + row) * 16 + 2 * d;
    const float u = (float)hash_uniform(key, ctr) * s;
    int b = FLOW_BINS - 1;
    float acc = 0;
#pragma unroll 1
    for (int j = 0; j < FLOW_BINS; ++j) {
      acc += v[j];
      if (u < acc) {
        b = j;
        break;
      }
    }
    const double ud = (b + hash_uniform(key, ctr + 1)) / FLOW_BINS;
    double logf;
    x[(size_t)d * ldx + row] = pm_inverse(pm + d * PM_NODES, ud, &logf);
    xin[(size_t)row * FLOW_IN + d] = __float2bfloat16((float)(2.0 * ud - 1.0));
    bins[(size_t)row * 8 + d] = (uint8_t)b;
    logq[row] += LOG_BINS + __logf(v[b] / s) + (float)logf;
  }
  __device__ void finish(State&, int) const {}
};

// Backward through a hidden layer's activation: dz = acc * silu'(z); dz row-major (the next backward
// GEMM's A operand) and feature-major (the weight gradient's A operand).
struct EpiBackward {
  static constexpr int CHUNK = 32;
  using State = NoState;
  const bf16* z;
  bf16 *dz, *dzT;
  int M, ldT;
  __device__ void apply(State&, int row, int col, float (&v)[32]) const {
    if (row >= M) return;
    const bf16* zr = z + (size_t)row * FLOW_H + col;
    float g[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      g[j] = v[j] * silu_grad(__bfloat162float(zr[j]));
      dzT[(size_t)(col + j) * ldT + row] = __float2bfloat16(g[j]);
    }
    store_row32(dz + (size_t)row * FLOW_H + col, g);
  }
  __device__ void finish(State&, int) const {}
};

// Weight gradient (split over K = the batch): atomically added into dW [rows x ldw] (FP32).
struct EpiWgrad {
  static constexpr int CHUNK = 32;
  using State = NoState;
  float* dW;
  int M, ldw;
  __device__ void apply(State&, int row, int col, float (&v)[32]) const {
    if (row >= M) return;
    float* d = dW + (size_t)row * ldw + col;
#pragma unroll
    for (int j = 0; j < 32; ++j) atomicAdd(d + j, v[j]);
  }
  __device__ void finish(State&, int) const {}
};

}  // namespace flow
}  // namespace pwa
