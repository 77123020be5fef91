/* pwa_b200.h -- C ABI of the B200 likelihood library (libpwa_b200.so).
 *
 * The hot path replaced here is the reference's GPU likelihood boundary
 * (RooTDalitz/kernel_calEva.h:20-27, implemented in src/kernel_calEva.cu and
 * src/cu_DPFPropogator.cu).  The reference exposes it with C++ linkage, std::vector arguments,
 * file-scope device buffers and abort-on-error; this ABI carries the same data (the reference's SoA
 * planes and float parameter block, unchanged) through plain pointers, an explicit context and int
 * status codes.  The C++ functions with the reference's exact signatures are declared in
 * kernel_calEva_compat.h and implemented on top of this ABI.
 *
 * Data layout (identical to the reference, src/RooDalitzAmplitude.cxx:548-770):
 *   events are columns, planes are rows, plane stride n_size = (n / 32 + 1) * 32 floats.
 *   pp  : 111 planes  0 mKp, 1 m(J/psi p), 2 weight (<= -1000 marks data), 3..50 Lambda* angular
 *         factors (Re/Im interleaved), 51..110 Lambda* d-functions
 *   pp1 :  96 planes  Pc angular factors (Re/Im interleaved)
 *   pp2 :  96 planes  Pc d-functions
 *   sw  :  n_size floats, data sWeights for events [0, nda)
 *   pp3 :  97 planes  (models with Zcs entries) 0 m(J/psi K), 1..96 Zcs angular factors AX
 *         (Re/Im interleaved, plane 1 + 2 (i*24 + j*12 + m))
 *   pp4 :  96 planes  Zcs d-functions DX (plane s*24 + k*12 + m)
 * Events [0, nda) are data, sorted into m(J/psi p) bands; [nda, n) are MC.
 *
 * Parameter block ("h_paraList"): the reference's float layout (cu_init_data,
 * src/RooDalitzAmplitude.cxx:3141-3210): 6 floats per resonance, then (Re, Im) helicity couplings,
 * spline coefficients, and 4 x 32 K-matrix floats.
 *
 * Threading: a context is used by one host thread at a time; distinct contexts are independent
 * (no global device state besides read-only constant tables).
 */
#ifndef PWA_B200_H
#define PWA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PWA_OK = 0,
  PWA_E_CUDA = 1,        /* a CUDA runtime call failed (see pwa_last_cuda_error) */
  PWA_E_ARG = 2,         /* null pointer or negative size */
  PWA_E_LAYOUT = 3,      /* parameter block sizes inconsistent with the resonance table */
  PWA_E_SIZE = 4,        /* a model size exceeds the compiled maximum */
  PWA_E_UNSUPPORTED = 5, /* lineshape type or entry point option not supported */
  PWA_E_PARAM = 6,       /* invalid resonance parameters (spin, K-matrix channel) */
  PWA_E_STATE = 7,       /* no events uploaded (or no Zcs planes for a model with Zcs entries) */
  PWA_E_NOMEM = 8        /* device allocation failed */
};

typedef struct pwa_ctx pwa_ctx;

typedef struct {
  double nll;       /* NLL_SHIFT + sumW_data ln(sumint / sumW_mc) - sum sw ln fx (+1000 guard) */
  double sumint;    /* sum over MC of w |A|^2 (host_store_fx's return value) */
  double sum_noint; /* same without Pc / Lambda* interference */
  double data_term; /* sum over data of sw ln |A|^2 */
  int64_t n_nonpos; /* events whose |A|^2 was <= 0 or not finite */
} pwa_result;

/* Context on CUDA device `device` (its own stream and buffers).  Replaces the file-scope state of
 * kernel_calEva.cu:76-80. */
/* A context owns a blocking CUDA stream (pwa_ctx_stream): its work is ordered with the legacy default
 * stream, so device inputs written there before a call are complete when the call reads them; inputs
 * written on other streams must be complete before the call. */
int pwa_ctx_create(int device, pwa_ctx** out);
int pwa_ctx_destroy(pwa_ctx* ctx);

/* Copies events from host planes (reference layout) to the device (cu_malloc_h_pp,
 * kernel_calEva.cu:1447-1457, for all planes at once).  nda_smr / nda_fine are the band arguments
 * host_store_fx receives (IntegralMethod2 passes its first band count minus one). */
int pwa_ctx_upload_events(pwa_ctx* ctx, const float* pp, const float* pp1, const float* pp2, const float* sw,
                          int64_t n, int64_t n_size, int64_t nda, int64_t nda_smr, int64_t nda_fine);

/* Uses caller-owned device planes instead (the reference's d_float_pp* vectors); the context does
 * not free them. */
int pwa_ctx_set_device_events(pwa_ctx* ctx, const float* d_pp, const float* d_pp1, const float* d_pp2,
                              const float* d_sw, int64_t n, int64_t n_size, int64_t nda, int64_t nda_smr,
                              int64_t nda_fine);

/* Evaluate only the data events [first, first + n_data) (with all MC events): one toy of an ensemble
 * whose toys' data were uploaded one after another, each sorted into its own m(J/psi p) bands, with
 * the MC shared.  nda_smr / nda_fine are that toy's band arguments (as host_store_fx receives them),
 * counted from `first`; the caller passes the toy's sum of data weights to pwa_ctx_eval_nll.
 * n_data < 0 selects all data again (first ignored).  Per-event outputs hold values of the selected
 * events only.  No counterpart in the reference, where each toy is a separate PDF object with its own
 * upload of the same MC (gen_toys workflow). */
int pwa_ctx_select_data(pwa_ctx* ctx, int64_t first, int64_t n_data, int64_t nda_smr, int64_t nda_fine);

/* Zcs chain planes of the uploaded events (the reference's d_float_pp3 / d_float_pp4, filled from
 * cu_Jpsihh_dlz's mjpsik, AXRe/AXIm and DX members, src/RooDalitzAmplitude.cxx:564-717), needed by
 * models with Zcs entries (NX > 0).  Call after the event upload; the same n_size and event order
 * (including the band order of an unsorted upload, applied here too).  A new event upload drops
 * them. */
#define PWA_PP3_PLANES 97
#define PWA_PP4_PLANES 96
int pwa_ctx_upload_zcs_events(pwa_ctx* ctx, const float* h_pp3, const float* h_pp4);
/* Caller-owned device planes instead (not freed by the context); in the context's event order. */
int pwa_ctx_set_device_zcs_events(pwa_ctx* ctx, const float* d_pp3, const float* d_pp4);

/* Resolution model of m(J/psi p).  PWA_SMEAR_REFERENCE (default): the reference's event classes
 * (kernel_calEva.cu:819-961): the two data bands smeared with 30 / 150 quantile offsets times
 * mres(m), MC in the two windows with 20, the rest unsmeared.  PWA_SMEAR_GAUSS: every event smeared
 * with a Gaussian of width sigma (GeV) sampled on offsets (b - half_bins) * step, b = 0 .. 2 half_bins
 * (at most 127 offsets), weights exp(-offset^2 / 2 sigma^2) normalised to 1: |A|^2 =
 * sum_b w_b |A(m + offset_b)|^2; the band arguments are then unused.  Applies to the uploaded
 * events and later uploads, and to the single-point and the batch call alike. */
#define PWA_SMEAR_REFERENCE 0
#define PWA_SMEAR_GAUSS 1
int pwa_ctx_set_smearing(pwa_ctx* ctx, int mode, double sigma, double step, int half_bins);

/* Data in any order (gen_toys/rearrange_mJpsip/reOrder.C made the reference's inputs legal by sorting
 * them): the data columns [0, nda) are put into the three m(J/psi p) bands (30-offset, 150-offset,
 * unsmeared; order kept inside each band) before the upload, and the band counts are derived as
 * RooDalitzAmplitude does (src/RooDalitzAmplitude.cxx:391-396, passing the band-1 count minus one as
 * IntegralMethod2 does).  Per-event outputs (h_fx, amp2) come back in the caller's order. */
int pwa_ctx_upload_events_unsorted(pwa_ctx* ctx, const float* h_pp, const float* h_pp1, const float* h_pp2,
                                   const float* h_sw, int64_t n, int64_t n_size, int64_t nda);

/* The reOrder.C permutation of nda data masses (float m(J/psi p)): order[i] = index of the i-th
 * event in band order; band counts of the 30- and 150-offset bands.  Host only. */
int pwa_band_order(const float* mz, int64_t nda, int32_t* order, int64_t* n_band1, int64_t* n_band2);

/* One likelihood evaluation (host_store_fx, kernel_calEva.cu:1186-1363): parameter block from host
 * memory in, result out; h_fx (optional, n doubles) receives per-event fx like the reference's
 * store_h_fx copy.  Blocks until the result is on the host. */
int pwa_ctx_eval_nll(pwa_ctx* ctx, const float* h_paraList, int para_size, int vamp_size, int spline_size,
                     int NR, int NZ, int NX, float FFR, float FFB, double sum_w_mc, double sum_w_data,
                     double nll_shift, pwa_result* out, double* h_fx);

/* Likelihood at npoints parameter points in one call; point p's float block starts at
 * h_paraLists + p * block_stride (same sizes and model for all points).  Made for the 2N+1 points of
 * Minuit's numerical gradient (RooMinuit/Minuit2 calling host_store_fx once per point,
 * kernel_calEva.cu:1186-1363): points that differ from point 0 in the couplings or lineshape of one
 * Lambda*, in the couplings of up to 8 Pc entries, or in the lineshapes of one Pc group are evaluated
 * together in one pass over the events from the centre's per-event terms (exact FP64); other points
 * go through pwa_ctx_eval_nll one by one.  n_structured (optional) receives the number of points of
 * the first kind.  out: npoints results. */
int pwa_ctx_eval_nll_batch(pwa_ctx* ctx, const float* h_paraLists, int npoints, int block_stride, int para_size,
                           int vamp_size, int spline_size, int NR, int NZ, int NX, float FFR, float FFB,
                           double sum_w_mc, double sum_w_data, double nll_shift, pwa_result* out,
                           int* n_structured);

/* Device time of the last pwa_ctx_eval_nll_batch in milliseconds (CUDA events; includes the points
 * evaluated one by one). */
double pwa_ctx_last_batch_ms(pwa_ctx* ctx);

/* Device time (ms, CUDA events) of segment i's batched passes in the last pwa_ctx_eval_nll_batch with
 * timing on (pwa_ctx_set_timing); segments as pwa_ctx_segment_info numbers them.  Diagnostic, no
 * counterpart in the reference. */
int pwa_ctx_batch_segment_ms(pwa_ctx* ctx, int i, double* ms);

/* Sum over the MC events of w * |A|^2 (unsmeared |A|^2 as host_store_amp2s gives it, w the event weight):
 * the normalisation integral of one parameter block that the reference's fit and interference
 * fractions divide (RooDalitzAmplitude::getIFandFF, src/RooDalitzAmplitude.cxx:5250-5435, evaluated
 * with subset couplings as in storeResonanceWeights :985-1292). */
int pwa_ctx_mc_integral(pwa_ctx* ctx, const float* h_paraList, int para_size, int vamp_size, int spline_size,
                        int NR, int NZ, int NX, float FFR, float FFB, double* integral);

/* Per-event unsmeared |A|^2 for toy weights (host_store_amp2s, kernel_calEva.cu:1376-1419). */
int pwa_ctx_amp2(pwa_ctx* ctx, const float* h_paraList, int para_size, int vamp_size, int spline_size, int NR,
                 int NZ, int NX, float FFR, float FFB, double* h_amp2);

/* Device time of the last pwa_ctx_eval_nll kernels in milliseconds (CUDA events). */
double pwa_ctx_last_kernel_ms(pwa_ctx* ctx);

/* The context's CUDA stream (cudaStream_t), for callers that bracket calls with their own events. */
void* pwa_ctx_stream(pwa_ctx* ctx);

/* Per-kernel timing: when on, pwa_ctx_eval_nll records a CUDA event after each event-class kernel.
 * Classes (segments): 0 unsmeared, 1 20-offset smearing, 2 30-offset, 3 150-offset. */
int pwa_ctx_set_timing(pwa_ctx* ctx, int on);
int pwa_ctx_segment_count(pwa_ctx* ctx);
int pwa_ctx_segment_info(pwa_ctx* ctx, int i, int* kind, int64_t* events, double* last_ms);
/* With timing on: events of segment i that the last evaluation deferred from the table-only pass to
 * the exact pass (lineshape masses the interpolation tables cannot serve).  No reference counterpart. */
int pwa_ctx_segment_deferred(pwa_ctx* ctx, int i, int64_t* deferred);

/* Launch shape of the batched evaluation's passes over one event class (the kind pwa_ctx_segment_info
 * reports: 0 unsmeared, 1/2/3 the 20/30/150-offset classes, 4 the weighted grid): grid = min(blocks
 * for its events, waves x SMs x resident blocks per SM), waves 1..64 (default 1).  More waves than
 * one balance uneven per-event work at the cost of more block starts; the batch autotuner
 * (pwa_b200.autotune.tune_batch) picks them per class by timing and caches the choice.  No reference
 * counterpart (the reference launches one fixed shape). */
int pwa_ctx_set_batch_waves(pwa_ctx* ctx, int kind, int waves);

/* Coupled-channel K-matrix of the context's evaluations.  PWA_KMATRIX_DEFAULT: 4 channels (J/psi p,
 * Sigma_c D*, Sigma_c* D*, Sigma_c D; Default_KMatrix, cu_DPFPropogator.cu:588-813).
 * PWA_KMATRIX_ISOSPIN: the 7-channel isospin split of the reference's ISOSPIN_SIGMACD build
 * (Isospin_KMatrix, :384-586): charged and neutral partners of each Sigma_c(*) D(*) channel with their
 * own masses and Sigma_c(*) widths, couplings and scattering terms spread with the isospin factors
 * sqrt(2/3) and -sqrt(1/3), and poles of channels 1 and 3 shifted by Re(i g^2 (2 rho_charged +
 * rho_neutral) / 3).  The reference selects it at compile time; here it is a run-time switch of the
 * context (the allocation-free entry point and the reference-signature functions use the default). */
#define PWA_KMATRIX_DEFAULT 0
#define PWA_KMATRIX_ISOSPIN 1
int pwa_ctx_set_kmatrix(pwa_ctx* ctx, int kmatrix);

/* Order in which the kernels walk the MC events of each class under the reference's resolution model
 * (the 20-offset windows and the unsmeared rest): 0 (default) by event index, so that neighbouring
 * warps share the 32-byte sectors of the event planes; 1 by m(J/psi p), so that they read neighbouring
 * nodes of the per-point lineshape tables (the batched gradient's points that move a K-matrix group
 * each read their own table).  Results differ only by the order of the FP64 sums.  Re-splits the
 * uploaded events.  No counterpart in the reference. */
int pwa_ctx_set_event_order(pwa_ctx* ctx, int by_mass);
/* K-matrix lineshape tables (default on): each evaluation first tabulates the exact FP64 K-matrix
 * outputs on a 10 keV m(J/psi p) grid and interpolates them (6-point Lagrange), evaluating exactly
 * near thresholds, branch switches and pole clamps.  Off: every lookup solves the K-matrix. */
int pwa_ctx_set_lineshape_tables(pwa_ctx* ctx, int on);

/* Bytes copied host to device per evaluation (the decoded parameter table). */
int64_t pwa_point_table_bytes(void);

/* Number of kernels launched by the last pwa_ctx_eval_nll. */
int pwa_ctx_last_launches(pwa_ctx* ctx);

/* Host-side diagnostic, no GPU needed: decodes the parameter block as the kernels do and evaluates
 * each Lambda* lineshape times its Lambda_b barrier at mkp (lstar: 2*NR doubles, Re/Im) and each Pc
 * lineshape times its barrier at mz (pc: 2*NZ doubles).  Plays the role of the reference's
 * host_store_lineshapeLsKM diagnostic (kernel_calEva.cu:1545-1584) for the Breit-Wigner and
 * K-matrix lineshapes. */
int pwa_host_lineshapes(const float* h_paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                        int NX, float FFR, float FFB, double mkp, double mz, double* lstar, double* pc);
/* The same with a K-matrix variant (PWA_KMATRIX_DEFAULT or PWA_KMATRIX_ISOSPIN). */
int pwa_host_lineshapes_km(const float* h_paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                           int NX, float FFR, float FFB, int kmatrix, double mkp, double mz, double* lstar,
                           double* pc);

/* Lambda* lineshape diagnostic on the device (replaces host_store_lineshapeLsKM,
 * RooTDalitz/kernel_calEva.h:27, src/kernel_calEva.cu:1490-1584): for every Lambda* entry r < NR of the
 * parameter block and every mass h_mkp[i], the revised K-matrix lineshape in its refactored form
 * (Revised_KMAMP_refactor, src/cu_DPFPropogator.cu:998-1063) and the Breit-Wigner (BW_AMP), each times
 * the Lambda_b barrier BTerm with radius FFR, whatever the entry's type, as the reference computes
 * them.  FP64 on the float parameters; outputs km_re/km_im/bw_re/bw_im[r * n_points + i] (host
 * memory, NR * n_points doubles each).  Only the resonance table (the first 6 NR floats) is read.
 * Allocates and frees its own device buffers; blocks until the outputs are on the host. */
int pwa_lineshapes_lstar_km(int device, const float* h_mkp, int n_points, int NR, float FFR,
                            const float* h_paraList, int para_size, double* km_re, double* km_im, double* bw_re,
                            double* bw_im);

/* Synthetic events on the device (flat phase space, the reference ntuple maker's helicity angles,
 * the filldlz basis), written into columns [col0, col0 + n) of device planes with stride n_size.
 * Event t uses the counter-based random stream (seed, first_id + t).  data != 0 writes the data
 * weight sentinel -1001, else a weight uniform in [w_lo, w_hi].  stream: cudaStream_t or NULL. */
int pwa_generate_events(float* d_pp, float* d_pp1, float* d_pp2, int64_t n_size, int64_t col0, int64_t n,
                        uint64_t seed, uint64_t first_id, float w_lo, float w_hi, int data, void* stream);

/* Basis from given angles (device arrays [16][n]: mLk, mjpsiL, cosTheta_Lb, cosTheta_L, cosTheta_Jpsi,
 * phiK, phiMu, Z_cosTheta_Lb, Z_cosTheta_Z, Z_cosTheta_Jpsi, Z_phiZ, Z_phiJpsi, Z_phiMu,
 * cosTheta_Lambda, alpha_Mu, weight) into columns [0, n). */
int pwa_basis_from_angles(const double* d_angles, int64_t n, float* d_pp, float* d_pp1, float* d_pp2,
                          int64_t n_size, void* stream);

/* Helicity angles from four-vectors in the Lambda_b rest frame (device [16][n]: p, K, mu+, mu-, each
 * px py pz E) into device [15][n] (the first 15 rows of the layout above). */
int pwa_angles_from_vectors(const double* d_vectors, int64_t n, double* d_angles, void* stream);

/* ---- Learned proposal density (no counterpart in the reference, whose toys are flat hit-or-miss,
 * gen_toys/create_efficiency/hit_and_reject.py:40-50; the exact amplitude reweights every event).
 *
 * Unit coordinates x in [0,1]^7 of the phase space: x0, x1 the Dalitz point (m^2(J/psi p) linear in x0
 * over its range, then m^2(Kp) linear in x1 across the Dalitz row: Pc bands at fixed x0, the region's
 * boundary at x1 = 0 and 1), x2..x4 the decay's orientation in the Lambda_b rest frame (cos of the
 * J/psi angle to the flight axis, its azimuth, the roll of the decay plane), x5, x6 the mu+ direction in
 * the J/psi frame.  Arrays of x are device doubles [7][ldx] (coordinate-major). */

/* Events at unit coordinates into columns [col0, col0 + n) of device planes (reference layout, as
 * pwa_generate_events writes them; data != 0 writes the data weight sentinel, else weight w), and
 * (d_flat, optional) the flat phase-space density of each x. */
int pwa_events_from_unit(const double* d_x, int64_t ldx, int64_t n, float* d_pp, float* d_pp1, float* d_pp2,
                         int64_t n_size, int64_t col0, float w, int data, double* d_flat, void* stream);
/* n flat phase-space events in unit coordinates (counter-based: event i is a function of (seed, first_id + i)). */
int pwa_unit_flat(int64_t n, uint64_t seed, uint64_t first_id, double* d_x, int64_t ldx, void* stream);

/* The proposal network: autoregressive 4 x 256 SiLU MLP over x (masked), 64 bins per coordinate,
 * q(x) = prod_d 64 p_d(bin(x_d) | x_<d).  Kernels: BF16 tcgen05 GEMMs with FP32 accumulation in TMEM,
 * fused epilogues; Adam on FP32 master weights.  max_batch: a multiple of 128 (rows per step / chunk). */
typedef struct pwa_flow pwa_flow;
/* Calls run on the handle's own blocking stream (ordered with the legacy default stream, as for a
 * context) and return when their work is done. */
int pwa_flow_create(int device, int max_batch, uint64_t seed, pwa_flow** out);
int pwa_flow_destroy(pwa_flow* flow);
/* Parameters (FP32, layer by layer: weights [out x in] row-major then biases; layers 256 x 64,
 * 3 x 256 x 256, 512 x 256). */
int64_t pwa_flow_param_count(void);
int pwa_flow_get_params(pwa_flow* flow, float* h_params);
int pwa_flow_set_params(pwa_flow* flow, const float* h_params);
/* One Adam step (learning rate lr) on the loss -sum_i w_i log q(x_i) / sum_i w_i of n events (n a multiple
 * of 128, at most max_batch; d_w device doubles); *loss: the loss before the step. */
int pwa_flow_train_step(pwa_flow* flow, const double* d_x, int64_t ldx, const double* d_w, int n, float lr,
                        double* loss);
/* The same loss and its gradients (h_grad: pwa_flow_param_count floats, parameter layout) without an update. */
int pwa_flow_gradients(pwa_flow* flow, const double* d_x, int64_t ldx, const double* d_w, int n, double* loss,
                       float* h_grad);
/* log q(x) of n events into device floats. */
int pwa_flow_log_density(pwa_flow* flow, const double* d_x, int64_t ldx, int64_t n, float* d_logq);
/* n events drawn from q (counter-based on seed): x into device doubles [7][ldx], log q(x) into d_logq. */
int pwa_flow_sample(pwa_flow* flow, int64_t n, uint64_t seed, double* d_x, int64_t ldx, float* d_logq);
/* Pre-maps: before the network, each coordinate passes a fixed monotone map u = F(x), piecewise linear
 * through PWA_FLOW_PREMAP_NODES nodes at x = k / (nodes - 1), and q(x) = q_net(F(x)) prod_d F_d'(x_d).
 * Identity at creation.  fit: F_d' = (1 - mix) (weighted histogram of x_d, normalised) + mix, from n
 * events with weights w >= 0 (device doubles), 0 < mix <= 1; fit before training, as the network's
 * input changes with them.  get/set: host doubles [7][PWA_FLOW_PREMAP_NODES] (set refuses rows that do
 * not run strictly upward from 0 to 1). */
#define PWA_FLOW_PREMAP_NODES 1025
int pwa_flow_fit_premap(pwa_flow* flow, const double* d_x, int64_t ldx, const double* d_w, int64_t n, double mix);
int pwa_flow_get_premap(pwa_flow* flow, double* h_cdf);
int pwa_flow_set_premap(pwa_flow* flow, const double* h_cdf);

/* ---- Toy ensembles fitted together (no counterpart in the reference, which builds one PDF per toy and
 * integrates the MC anew at every call: src/RooDalitzAmplitude.cxx:1293-1628, gen_toys/).
 *
 * For fits that float the helicity couplings with the lineshape parameters held where the ensemble is
 * set up.  |A|^2 of an event is then a Hermitian form in the coupling "slots": c_{r,k,m} of Lambda* r
 * (slot k NS + 6 r + m) and c_{q,k,m} of the Pc entry at group-order position q (slot k NS + 6 NR +
 * 12 q + m), NS = 6 NR + 12 NZ, proton helicity k, helicity index m as in the parameter block.  The MC
 * normalisation of any toy is c^H M c (M: FP64 Gram matrix over the shared MC, built at creation), and
 * one call evaluates every toy's data term over its own window with its gradient.
 *
 * create: over the context's events (borrowed: keep them uploaded, unchanged), the lineshape part of the
 * model from the block (its couplings are not used), toy t = data events [first[t], first[t] + count[t])
 * with the band arguments nda_smr[t], nda_fine[t] that pwa_ctx_select_data takes for it, sum_w_data[t]
 * its data weight sum and sum_w_mc that of the MC; active (optional, one byte per slot): slots that can
 * be non-zero in the fit (the Gram matrix is accumulated for those only; null: all).  Models with Zcs
 * entries: PWA_E_UNSUPPORTED.  Memory: (2 NR + 2 NZ + NZ (NZ + 1)) doubles per data event. */
typedef struct pwa_ens pwa_ens;
int pwa_ens_create(pwa_ctx* ctx, const float* h_paraList, int para_size, int vamp_size, int spline_size, int NR,
                   int NZ, int NX, float FFR, float FFB, int n_toys, const int64_t* first, const int64_t* count,
                   const int64_t* nda_smr, const int64_t* nda_fine, const double* sum_w_data, double sum_w_mc,
                   const uint8_t* active, pwa_ens** out);
int pwa_ens_destroy(pwa_ens* ens);
/* Number of slots (2 NS). */
int pwa_ens_slot_count(const pwa_ens* ens);
/* The slot values (Re, Im doubles, 2 (6 NR + 12 NZ) slots) of a parameter block. */
int pwa_ens_slots(const float* h_paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ, int NX,
                  float FFR, float FFB, double* h_slots);
/* The Gram matrices M and Mn (non-interference sum), row-major slot x slot complex (Re, Im doubles). */
int pwa_ens_gram(const pwa_ens* ens, double* h_M, double* h_Mn);
/* Launch shape of the per-call kernel: warps per block (4, 8, 12 or 16) and events per work item; the
 * project's autotuner (pwa_b200.ensemble.autotune) picks them by timing.  A shape whose shared memory
 * exceeds one block's (large models at 16 warps) returns PWA_E_SIZE and the current shape stays. */
int pwa_ens_set_launch(pwa_ens* ens, int warps, int tile_events);
/* One evaluation of every toy t with on[t] != 0 (on null: all) at its slot vector h_slots[t] ([n_toys]
 * [slots] x (Re, Im)), as one CUDA-graph launch (captured at the first call and after a launch-shape or
 * nll_shift change): h_out[4 t ..] = NLL (nll_shift + W_t ln(I / W_mc) - D_t, +1000 under the reference's
 * non-interference guard), D_t = sum sw ln|A|^2 over its data, I = c^H M c, In = c^H Mn c;
 * h_grad[t] (optional) = dNLL / d conj(c), slot-wise (Re, Im); h_bad[t] (optional): data events with
 * |A|^2 <= 0 or not finite.  Rows of toys that are off are left as they were. */
int pwa_ens_eval(pwa_ens* ens, const double* h_slots, const int* h_on, double nll_shift, double* h_out,
                 double* h_grad, int64_t* h_bad);
/* Device time of the last pwa_ens_eval (ms) and of the set-up passes (factor rows, Gram matrices). */
double pwa_ens_last_ms(const pwa_ens* ens);
int pwa_ens_setup_ms(const pwa_ens* ens, double* factors_ms, double* gram_ms);

/* Allocation-free likelihood evaluation.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory while they evaluate the likelihood -- for
 * example a fit running in a process whose GPU memory is already handed to another framework's
 * caching allocator, where a further cudaMalloc fails or fragments that pool, or a job with a fixed
 * device-memory budget on a shared node.  Inputs (the event planes, same layout and band arguments
 * as pwa_ctx_set_device_events, and the host parameter block) and the output are the caller's; all
 * scratch of the evaluation lives in a fixed device array of PWA_NOALLOC_SCRATCH_BYTES inside the
 * library, present on every GPU that loads the library until the process exits.  The call makes no
 * cudaMalloc, cudaFree or other allocating call.
 *
 * Limits: at most PWA_NOALLOC_MAX_EVENTS events (larger samples return PWA_E_SIZE).  All calls share
 * the array, which keeps the last call's contents; calls that overlap on the GPU race on it (calls
 * from threads of one process are serialised inside the library).  The first call on a device
 * resolves the array's device address for that device; make that first call before any stream
 * capture.  Under CUDA's default lazy module loading, that first call is also when the library's
 * device code and the array are loaded onto the device, i.e. when their memory is taken: make the
 * first call before handing the device's free memory to another allocator, or run the process with
 * CUDA_MODULE_LOADING=EAGER (module and array loaded with the CUDA context).  Later calls take no
 * device memory.  Work is queued on `stream` (cudaStream_t, NULL for the default stream) and the
 * call waits on the host until the result is there.
 *
 * Lineshapes: with no room for the interpolation tables of pwa_ctx_eval_nll (about 49 MB per point),
 * this entry point evaluates every Pc lineshape exactly (one K-matrix solve per event and offset),
 * which costs about twice the time of the context entry point on the K-matrix model; results agree
 * with it to FP64 rounding.  Spline blocks (spline_size > 0) and Zcs models (NX > 0) return
 * PWA_E_UNSUPPORTED.  An empty sample (n = 0) gives sumint = data_term = 0. */
#define PWA_NOALLOC_MAX_EVENTS (1 << 20)
#define PWA_NOALLOC_SCRATCH_BYTES 4718592 /* 4.5 MiB */
int pwa_eval_nll_noalloc(int device, const float* d_pp, const float* d_pp1, const float* d_pp2, const float* d_sw,
                         int64_t n, int64_t n_size, int64_t nda, int64_t nda_smr, int64_t nda_fine,
                         const float* h_paraList, int para_size, int vamp_size, int spline_size, int NR, int NZ,
                         int NX, float FFR, float FFB, double sum_w_mc, double sum_w_data, double nll_shift,
                         void* stream, pwa_result* out);

const char* pwa_error_string(int code);
const char* pwa_last_cuda_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PWA_B200_H */
