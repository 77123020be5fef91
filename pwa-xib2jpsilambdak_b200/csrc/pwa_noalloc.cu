// Allocation-free NLL evaluation (pwa_eval_nll_noalloc).
//
// For callers that must not allocate device memory while they evaluate the likelihood: a fit whose
// process already hands all GPU memory to another framework's caching allocator (a further
// cudaMalloc there fails or fragments that pool), or an analysis job that has a fixed device-memory
// budget on a shared node and must not grow it after start-up.  Such a caller provides the event
// planes and receives the result; every scratch buffer of the evaluation (decoded parameter table,
// per-block partial sums, tail index lists, result slot) lives in one file-scope device array of
// fixed size, so this entry point calls no cudaMalloc, cudaFree or other allocating routine.
//
// The array is PWA_NOALLOC_SCRATCH_BYTES (4.5 MiB) on every GPU that loads the library and is
// held until the process exits.  Samples are limited to PWA_NOALLOC_MAX_EVENTS events.  All calls
// share the array and it keeps the last call's contents: a call rewrites everything it reads
// before reading it.  Calls that overlap on the GPU race on the array; calls from threads of one
// process are serialised by a lock here, overlapping use from elsewhere must be avoided by the
// caller.  The first call on a device looks up the array's device address (cudaGetSymbolAddress, with
// that device current) and caches it; make that first call before any stream capture.  Under CUDA's
// default lazy module loading that lookup is also what loads this library's device code onto the
// device, and with it the array: the first call on each device takes the array's memory (and the
// code's), later calls take none.  A caller that hands the device's free memory to another
// allocator should therefore make its first call before doing so, or run with
// CUDA_MODULE_LOADING=EAGER, which loads the module (and the array) when the CUDA context is created.
// Every call waits on the host for its result (it synchronises `stream`).
//
// The event-class kernels and the final reduction are the ones of pwa_ctx_eval_nll, launched with
// the same segments, grid sizes and partial-slot layout, so both entry points give the same result.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "../../include/pwa_b200.h"
#include "pwa_kernels.cuh"

namespace pwa {
cudaError_t configure_kernels();
}

namespace {

using namespace pwa;

constexpr int64_t kMaxEvents = PWA_NOALLOC_MAX_EVENTS;
constexpr int kMaxParts = 4096;
constexpr int kChunk = 1024;  // events per classification block
constexpr int kMaxChunks = (int)(kMaxEvents / kChunk);
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffTable = 0;
constexpr size_t kOffResult = align256(kOffTable + sizeof(PointTable));
constexpr size_t kOffParts = align256(kOffResult + sizeof(EvalResult));
constexpr size_t kOffCounts = align256(kOffParts + kMaxParts * sizeof(Partial));
constexpr size_t kOffOffsets = align256(kOffCounts + (kMaxChunks + 1) * sizeof(int));
constexpr size_t kOffLists = align256(kOffOffsets + (kMaxChunks + 1) * sizeof(int));
constexpr size_t kScratchBytes = PWA_NOALLOC_SCRATCH_BYTES;
static_assert(align256(kOffLists + kMaxEvents * sizeof(int32_t)) <= kScratchBytes,
              "scratch layout exceeds PWA_NOALLOC_SCRATCH_BYTES");

// The scratch.  In host code this name is a host-side stand-in, not a device address: kernels get the
// address looked up with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};

__device__ __forceinline__ bool in_window(float mz) { return (mz > 4.4 && mz < 4.48) || (mz > 4.27 && mz < 4.34); }

// counts[c] = window events in chunk c of the tail region [r0, n)
__global__ void k_count(const float* pp, int64_t ns, int64_t r0, int64_t n, int* counts) {
  const int64_t base = r0 + (int64_t)blockIdx.x * kChunk;
  int c = 0;
  for (int i = threadIdx.x; i < kChunk; i += 32) {
    const int64_t e = base + i;
    c += (e < n && in_window(pp[e + ns])) ? 1 : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// exclusive prefix over chunks; offsets[nchunks] = total window events
__global__ void k_scan(const int* counts, int nchunks, int* offsets) {
  int acc = 0;
  for (int c = 0; c < nchunks; ++c) {
    offsets[c] = acc;
    acc += counts[c];
  }
  offsets[nchunks] = acc;
}

// ordered scatter: window events to lw, the others to lu (event order preserved in both)
__global__ void k_scatter(const float* pp, int64_t ns, int64_t r0, int64_t n, const int* offsets, int32_t* lw,
                          int32_t* lu) {
  const int64_t base = r0 + (int64_t)blockIdx.x * kChunk;
  int nw = offsets[blockIdx.x];
  int nu = (int)(blockIdx.x * (int64_t)kChunk) - nw;
  const int lane = threadIdx.x;
  for (int i = 0; i < kChunk; i += 32) {
    const int64_t e = base + i + lane;
    const bool valid = e < n;
    const bool w = valid && in_window(pp[e + ns]);
    const unsigned mw = __ballot_sync(0xffffffffu, w);
    const unsigned mu = __ballot_sync(0xffffffffu, valid && !w);
    const unsigned below = (1u << lane) - 1u;
    if (w) lw[nw + __popc(mw & below)] = (int32_t)e;
    if (valid && !w) lu[nu + __popc(mu & below)] = (int32_t)e;
    nw += __popc(mw);
    nu += __popc(mu);
  }
}

int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return PWA_E_ARG;
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e);
    if (!p) return PWA_E_CUDA;
    if ((e = configure_kernels()) != cudaSuccess) return cuda_fail(e);
    g_addr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[device];
  return PWA_OK;
}

}  // namespace

extern "C" int pwa_eval_nll_noalloc(int device, const float* d_pp, const float* d_pp1, const float* d_pp2,
                                    const float* d_sw, int64_t n, int64_t n_size, int64_t nda, int64_t nda_smr,
                                    int64_t nda_fine, const float* h_paraList, int para_size, int vamp_size,
                                    int spline_size, int NR, int NZ, int NX, float FFR, float FFB,
                                    double sum_w_mc, double sum_w_data, double nll_shift, void* stream,
                                    pwa_result* out) {
  if (!d_pp || !d_pp1 || !d_pp2 || (nda > 0 && !d_sw) || !h_paraList || !out) return PWA_E_ARG;
  if (n < 0 || nda < 0 || nda > n || n_size < n) return PWA_E_ARG;
  if (n > kMaxEvents) return PWA_E_SIZE;  // PWA_NOALLOC_MAX_EVENTS
  if (spline_size != 0) return PWA_E_UNSUPPORTED;
  if (NX != 0) return PWA_E_UNSUPPORTED;  // no Zcs planes among this entry point's arguments
  std::lock_guard<std::mutex> lock(g_mu);
  thread_local PointTable table;
  int rc = build_point_table(h_paraList, para_size, vamp_size, spline_size, NR, NZ, NX, FFR, FFB, &table);
  if (rc) return rc;
  int prev = 0;
  cudaError_t e = cudaGetDevice(&prev);
  if (e == cudaSuccess) e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e);
  auto finish = [&](int code) {
    cudaSetDevice(prev);
    return code;
  };
  // every CUDA failure below is recorded for pwa_last_cuda_error
  auto fail = [&](cudaError_t err) { return finish(cuda_fail(err)); };
  unsigned char* base = nullptr;
  if ((rc = scratch_address(device, &base))) return finish(rc);
  int sm_count = 0;
  if ((e = cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return fail(e);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PointTable* d_table = reinterpret_cast<PointTable*>(base + kOffTable);
  EvalResult* d_res = reinterpret_cast<EvalResult*>(base + kOffResult);
  Partial* d_parts = reinterpret_cast<Partial*>(base + kOffParts);
  int* d_counts = reinterpret_cast<int*>(base + kOffCounts);
  int* d_offsets = reinterpret_cast<int*>(base + kOffOffsets);
  int32_t* d_lists = reinterpret_cast<int32_t*>(base + kOffLists);

  // same ranges as the context path (fake_kernel_store_fx, kernel_calEva.cu:920-961, begin = 0)
  const int64_t b1e = std::max<int64_t>(0, std::min(n, nda_smr));
  const int64_t b2s = std::max<int64_t>(0, nda_smr);
  const int64_t b2e = std::max<int64_t>(b2s, std::min(n, nda_smr + nda_fine));
  const int64_t r0 = std::min(n, std::max<int64_t>(0, nda_smr + nda_fine));
  const int64_t tail = n - r0;
  int nw = 0;
  if ((e = cudaMemcpyAsync(d_table, &table, sizeof(PointTable), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e);
  if (tail > 0) {
    const int nchunks = (int)((tail + kChunk - 1) / kChunk);
    k_count<<<nchunks, 32, 0, st>>>(d_pp, n_size, r0, n, d_counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    k_scan<<<1, 1, 0, st>>>(d_counts, nchunks, d_offsets);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    // the window list takes the front of the list region and the other tail events follow it, so the
    // window total is needed before the scatter
    if ((e = cudaMemcpyAsync(&nw, d_offsets + nchunks, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return fail(e);
    k_scatter<<<nchunks, 32, 0, st>>>(d_pp, n_size, r0, n, d_offsets, d_lists, d_lists + nw);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  }
  Segment segs[4];
  int nseg = 0;
  if (b2e > b2s) segs[nseg++] = Segment{SMEAR_150, b2s, b2e, nullptr};
  if (b1e > 0) segs[nseg++] = Segment{SMEAR_30, 0, b1e, nullptr};
  if (nw > 0) segs[nseg++] = Segment{SMEAR_20, 0, (int64_t)nw, d_lists};
  if (tail - nw > 0) segs[nseg++] = Segment{SMEAR_NONE, 0, tail - nw, d_lists + nw};
  int tot = 0;
  int offs[4];
  for (int i = 0; i < nseg; ++i) {
    offs[i] = tot;
    tot += segment_blocks(segs[i], sm_count);
  }
  if (tot > kMaxParts) return finish(PWA_E_SIZE);
  EventSet ev{d_pp, d_pp1, d_pp2, d_sw, n_size, n, nda};
  ev.lgen = lstar_has_general(table);
  for (int i = 0; i < nseg; ++i)
    if ((e = launch_segment(ev, segs[i], d_table, d_parts + offs[i], nullptr, nullptr, nullptr, sm_count, st)) !=
        cudaSuccess)
      return fail(e);
  // An empty sample launches no segment: the one slot finalize reads is cleared here, since the
  // array still holds the previous call's partials (a memset allocates nothing).
  if (tot == 0 && (e = cudaMemsetAsync(d_parts, 0, sizeof(Partial), st)) != cudaSuccess) return fail(e);
  if ((e = launch_finalize(d_parts, std::max(tot, 1), sum_w_mc, sum_w_data, nll_shift, d_res, st)) != cudaSuccess)
    return fail(e);
  EvalResult r;
  if ((e = cudaMemcpyAsync(&r, d_res, sizeof(EvalResult), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return fail(e);
  out->nll = r.nll;
  out->sumint = r.sumint;
  out->sum_noint = r.sum_noint;
  out->data_term = r.data_term;
  out->n_nonpos = (int64_t)r.n_nonpos;
  return finish(PWA_OK);
}
