// Host-visible declarations of the likelihood kernels (pwa_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "pwa_point.cuh"

struct pwa_ctx;

namespace pwa {

// Per-block partial sums written by the event kernels and reduced by finalize.
struct Partial {
  double data;      // sum of sw * ln(fx) over data events (fx <= 0 contributes -1e12)
  double mc;        // sum of w * fx over MC events
  double mc_noint;  // sum of w * fx without Pc/Lambda* interference over MC events
  double n_nonpos;  // events with fx <= 0 or non-finite fx
};

// Evaluation result copied back to the host.
struct EvalResult {
  double nll;        // NLL_SHIFT + sumW_data * ln(I / sumW_mc) - sum sw ln fx (+1000 guard)
  double sumint;     // sum over MC of w * fx
  double sum_noint;  // same without interference
  double data_term;  // sum over data of sw * ln fx
  double n_nonpos;
  double status;
};

// Event ranges of one evaluation.  Smeared classes are given as index lists or contiguous ranges.
struct EventSet {
  const float* pp;
  const float* pp1;
  const float* pp2;
  const float* sw;  // data sWeights, index = event index (may be null when there is no data)
  int64_t n_size;   // plane stride
  int64_t n;        // events
  int64_t nda;      // events [0, nda) are data (NLL term), the rest MC (normalisation)
  // Zcs chain planes (needed when the model has Zcs entries): pp3 97 planes (m(J/psi K), AX Re/Im),
  // pp4 96 planes (DX)
  const float* pp3 = nullptr;
  const float* pp4 = nullptr;
  // the model has spline or revised K-matrix Lambda* entries: selects the unsmeared-event kernel that
  // evaluates those lineshapes (the Breit-Wigner-only variant keeps its register allocation)
  int lgen = 0;
};

inline int lstar_has_general(const PointTable& T) {
  for (int r = 0; r < T.NR; ++r)
    if (T.L[r].type == LT_SPLINE || T.L[r].type == LT_RKM) return 1;
  return 0;
}

// Event classes: unsmeared, the reference's three quantile schemes (offsets in units of the mass
// resolution, equal weights), and a weighted grid of absolute offsets (fixed-width Gaussian).
enum Smear : int { SMEAR_NONE = 0, SMEAR_20 = 1, SMEAR_30 = 2, SMEAR_150 = 3, SMEAR_GRID = 4 };
constexpr int SMEAR_KINDS = 5;
constexpr int GRID_MAX_NB = 127;

struct Segment {
  int kind;             // Smear
  int64_t begin, end;   // contiguous event range when list == nullptr
  const int32_t* list;  // event indices, [begin, end) positions in the list otherwise
  const double* grid = nullptr;  // SMEAR_GRID: (offset in GeV, weight) pairs on the device
  int grid_nb = 0;               // SMEAR_GRID: number of offsets
};

// Blocks of the pass over a segment (and partial slots of that pass).
int segment_blocks(const Segment& s, int sm_count);

// Partial slots a segment uses: its pass, plus the pass over deferred events when deferred is true.
int segment_parts(const Segment& s, int sm_count, bool deferred);

// Records a failed CUDA call's message (pwa_last_cuda_error) and returns PWA_E_CUDA, or PWA_E_NOMEM
// for a failed allocation.
int cuda_fail(cudaError_t e);

// What other parts of the library read of a context: its device, events and resolution model.
struct CtxView {
  int device, sm_count;
  cudaStream_t st;
  const float *pp, *pp1, *pp2, *sw, *pp3, *pp4;
  int64_t n, n_size, nda;
  int gauss;            // 1: Gaussian resolution on a weighted grid (d_grid, grid_nb)
  const double* grid;
  int grid_nb;
  int use_tables;
  int build_flags;  // build_point_table flags (K-matrix variant)
};
int ctx_view(const pwa_ctx* c, CtxView* v);

// Builds the point table from a float parameter block; returns 0 or a PWA_E_* code.  flags:
// BUILD_KM_ISOSPIN selects the 7-channel isospin-split K-matrix (the reference's ISOSPIN_SIGMACD).
constexpr int BUILD_KM_ISOSPIN = 1;
int build_point_table(const float* pl, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                      float ffr, float ffb, PointTable* out, int flags = 0);

// Launches one segment; partials written at out[0 .. segment_parts).  fx_out (optional) receives
// per-event fx (weighted by w for MC, like the reference's d_fx).  With the lineshape tables on, defer
// (room for the segment's events) and defer_count (zeroed before the launch) receive the events the
// tables cannot serve, which a second pass evaluates exactly; with tables off both are null.
cudaError_t launch_segment(const EventSet& ev, const Segment& seg, const PointTable* d_table, Partial* out,
                           double* fx_out, int32_t* defer, int* defer_count, int sm_count, cudaStream_t st);

// Fills the per-point Pc entry tables from the device copy of the point table, verifies every
// interval, refines and verifies the failing ones (four launches).
cudaError_t launch_build_tables(const PointTable* d_table, int n_nodes, int sm_count, cudaStream_t st);

// Attaches TAB_BYTES of device memory (256-byte aligned) for the two-level tables to a host point
// table: enables interpolation of the Pc lineshapes.
void attach_tables(PointTable* T, void* d_mem);

// Attaches TAB_BYTES_GROUP of device memory to a host point table for a table of Pc group g alone
// (the grid of attach_tables, stride = the group's entry count): the table of a batch point that
// moves only that group's lineshape.
void attach_group_table(PointTable* T, int g, void* d_mem);

// Reduces nparts partials and assembles the NLL.
cudaError_t launch_finalize(const Partial* parts, int nparts, double sum_w_mc, double sum_w_data,
                            double nll_shift, EvalResult* res, cudaStream_t st);

// Host evaluation of the decoded lineshapes (see pwa_kernels.cu).
void host_lineshapes(const PointTable& T, double mkp, double mz, cplx* lstar, cplx* pc);

// ------------------------------------------------------------------ batched evaluation
// A parameter point of a batch that differs from the batch centre (point 0) in one part of the
// amplitude only (pwa_batch.cu).
enum BatchKind : int { BP_SAME = 0, BP_LSTAR = 1, BP_PCC = 2, BP_PCG = 3 };
struct BatchPoint {
  int kind;
  unsigned lmask;          // BP_LSTAR: changed Lambda* (bit r)
  unsigned lsmask;         // BP_LSTAR: ... whose lineshape constants changed
  unsigned lcmask;         // BP_LSTAR: ... whose couplings changed
  int ldc;                 // BP_LSTAR: 1 when dc holds the coupling differences of the lcmask resonances
                           // (in r order, 12 used of each 24), 0 when more than 8 changed
  int group;               // BP_PCG: Pc group whose lineshapes changed
  int nq;                  // BP_PCC: Pc entries whose couplings changed (at most BATCH_MAXQ_PC = 4)
  int qpos[8], qsidx[8];   // their order positions and d-function spin indices
  const cplx* dc;          // BP_PCC: coupling differences point - centre, [nq][24] (device)
  const PointTable* T;     // device copy of the point's table (BP_LSTAR, BP_PCG)
  int pair;                // 1: the next point moves the same couplings (Lambda* couplings only, or the
                           // same Pc entries); the unsmeared kernel forms both from one pass over the planes
};

// Per Pc group of the batch centre: entries with identical couplings (the non-resonant K-matrix
// entries of a J^P group share theirs) share one slot of the per-event angular amplitudes.
struct BatchGroupMap {
  int slot[MAX_PC];             // order position -> slot within its group
  int nslot[MAX_GROUPS];        // slots per group
  int rep[MAX_GROUPS * 8];      // [g * 8 + s] -> order position of the entry representing slot s
  int max_slots;
};
BatchGroupMap batch_group_map(const PointTable& T0);

// Classifies point Tp against the batch centre T0: fills bp (kind, masks; bp->dc and bp->T are left
// for the caller) and, for BP_PCC, the coupling differences dc_host[nq][24].  Returns false when the
// point differs in more than one part of the amplitude (evaluate it with the single-point path).
bool classify_point(const PointTable& T0, const PointTable& Tp, BatchPoint* bp, cplx* dc_host);

// Largest number of points one batched launch takes (shared memory holds per-point sums).
constexpr int BATCH_MAX_POINTS = 512;

// Partial rows a segment of a batched evaluation writes (its pass, plus the deferred pass when
// deferred is true); each row holds npts partials.
int batch_segment_rows(const Segment& s, const PointTable& T0, const BatchGroupMap& gm, int npts, int sm_count,
                       bool deferred, int waves = 1);

// Launches the batched passes over one segment: partial rows out[0 .. batch_segment_rows) x npts.
// The points with kind BP_PCG must come first in d_pts.
cudaError_t launch_batch_segment(const EventSet& ev, const Segment& seg, const PointTable* d_T0, const PointTable& T0,
                                 const BatchGroupMap& gm, const BatchPoint* d_pts, int npts, Partial* out,
                                 int32_t* defer, int* defer_count, int sm_count, cudaStream_t st,
                                 int waves = 1);

// Reduces rows x npts partials (row-major) into npts results.
cudaError_t launch_finalize_points(const Partial* parts, int rows, int npts, double sum_w_mc, double sum_w_data,
                                   double nll_shift, EvalResult* res, cudaStream_t st);

cudaError_t configure_batch_kernels();

// Sum over the MC events of w * fx (fx: per-event values on the device) into res->sumint, through
// nblocks partial slots.
cudaError_t launch_mc_integral(const EventSet& ev, const double* fx, Partial* parts, int nblocks, EvalResult* res,
                               cudaStream_t st);

// Per-event unsmeared |A|^2 without weights (host_store_amp2s semantics) for n events.
cudaError_t launch_amp2(const EventSet& ev, const PointTable* d_table, double* out, int32_t* defer, int* defer_count,
                        int sm_count, cudaStream_t st);

}  // namespace pwa
