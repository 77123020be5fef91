// Tensor-core GEMM for the proposal-density network: C[M x N] = A[M x K] B[N x K]^T with BF16
// operands (both K-major) staged by TMA, tcgen05 MMAs accumulating in FP32 in TMEM, and a fused
// epilogue that reads the accumulator tile out of TMEM row by row (thread = row).
//
// One CTA computes a 128 x BN tile over the K blocks of its split (gridDim.z splits K): thread 0
// issues the TMA loads of a 4-stage ring (A block 128 x 64, B block BN x 64), thread 32 issues the
// MMAs (four K = 16 steps per block) and frees each stage with tcgen05.commit, and all four warps run
// the epilogue once the last MMA has completed.  Every wait is bounded (2 s of global time): on
// expiry the CTA records an error code in *err and finishes without touching its output.
#pragma once
#include <cuda_bf16.h>

#include "pwa_tc.cuh"

namespace pwa {
namespace flow {

constexpr int GEMM_BM = 128, GEMM_BK = 64, GEMM_STAGES = 4;
constexpr uint64_t GEMM_WAIT_NS = 2000000000ull;
enum GemmError : int { GEMM_OK = 0, GEMM_TIMEOUT_LOAD = 1, GEMM_TIMEOUT_MMA = 2, GEMM_TIMEOUT_EPILOGUE = 3 };

template <int BN>
struct GemmShape {
  static_assert(BN == 64 || BN == 128 || BN == 256, "tile width");
  static constexpr uint32_t A_BYTES = GEMM_BM * GEMM_BK * 2;
  static constexpr uint32_t B_BYTES = BN * GEMM_BK * 2;
  static constexpr size_t SMEM = 1024 + GEMM_STAGES * (size_t)(A_BYTES + B_BYTES) + 128;
  static constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
};

// Epilogue interface: Epi::CHUNK (32 or 64) accumulator columns per call of
//   apply(State&, int row, int col, float (&v)[CHUNK])   (row, col: global indices)
// and finish(State&, int row) once per thread; rows past the matrix are passed too (row >= M).
template <int BN, class Epi>
__global__ void __launch_bounds__(128, 1)
    k_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int kb_per_split,
           int kb_total, int n_tile0, Epi epi, int* err) {
  using S = GemmShape<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + GEMM_STAGES * S::A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + GEMM_STAGES * S::B_BYTES);
  uint64_t* empty = full + GEMM_STAGES;
  uint64_t* done = empty + GEMM_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int failed;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * GEMM_BM, n0 = (blockIdx.y + n_tile0) * BN;
  const int kb0 = blockIdx.z * kb_per_split;
  const int nkb = min(kb_per_split, kb_total - kb0);
  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < GEMM_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    tc::fence_barrier_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, S::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {  // TMA producer
    for (int i = 0; i < nkb; ++i) {
      const int s = i % GEMM_STAGES;
      if (i >= GEMM_STAGES && !tc::mbar_wait(&empty[s], ((i / GEMM_STAGES) - 1) & 1, GEMM_WAIT_NS)) {
        atomicExch(&failed, GEMM_TIMEOUT_LOAD);
        break;
      }
      tc::mbar_arrive_expect_tx(&full[s], S::A_BYTES + S::B_BYTES);
      tc::tma_load_2d(sA + s * S::A_BYTES, &ta, &full[s], (kb0 + i) * GEMM_BK, m0);
      tc::tma_load_2d(sB + s * S::B_BYTES, &tb, &full[s], (kb0 + i) * GEMM_BK, n0);
    }
  } else if (threadIdx.x == 32) {  // MMA issuer
    constexpr uint32_t idesc = tc::idesc_bf16_f32(GEMM_BM, BN);
    int i = 0;
    for (; i < nkb; ++i) {
      const int s = i % GEMM_STAGES;
      if (!tc::mbar_wait(&full[s], (i / GEMM_STAGES) & 1, GEMM_WAIT_NS)) {
        atomicExch(&failed, GEMM_TIMEOUT_MMA);
        break;
      }
      tc::tc_fence_after();
      const uint64_t ad = tc::desc_kmajor_sw128(tc::smem_u32(sA + s * S::A_BYTES));
      const uint64_t bd = tc::desc_kmajor_sw128(tc::smem_u32(sB + s * S::B_BYTES));
#pragma unroll
      for (int k = 0; k < GEMM_BK / 16; ++k)  // +32 bytes of start address per K step of 16
        tc::mma_bf16(tmem, ad + 2 * k, bd + 2 * k, idesc, (i > 0 || k > 0) ? 1u : 0u);
      tc::mma_commit(&empty[s]);
    }
    tc::mma_commit(done);  // completes when every MMA issued above has completed
  }
  __syncwarp();
  // epilogue: warp w owns TMEM lanes 32w .. 32w + 31, i.e. tile rows m0 + 32w + lane
  const bool ok = tc::mbar_wait(done, 0, GEMM_WAIT_NS);
  if (!ok && lane == 0) atomicExch(&failed, GEMM_TIMEOUT_EPILOGUE);
  tc::tc_fence_after();
  __syncthreads();
  if (!failed) {
    typename Epi::State st{};
    const int row = m0 + warp * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c = 0; c < BN; c += Epi::CHUNK) {
      float v[Epi::CHUNK];
#pragma unroll
      for (int h = 0; h < Epi::CHUNK / 32; ++h) tc::tmem_ld32(tl + c + 32 * h, *reinterpret_cast<float(*)[32]>(v + 32 * h));
      epi.apply(st, row, n0 + c, v);
    }
    epi.finish(st, row);
  } else if (threadIdx.x == 0) {
    atomicExch(err, failed);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::TMEM_COLS);
}

}  // namespace flow
}  // namespace pwa
