// TEST INFRASTRUCTURE ONLY -- C entry points around the reference's own likelihood code built for
// host cores (see oracle/build_ref.py).  The reference functions are called unmodified; this file
// only adapts raw pointers to the reference's std::vector interface
// (RooTDalitz/kernel_calEva.h:20-27) and silences its per-call stdout line.
#include <cuda_runtime.h>
#include <iostream>
#include <sstream>
#include <vector>

thread_local dim3 blockIdx;
thread_local dim3 threadIdx;
thread_local dim3 blockDim;

// Reference declarations (RooTDalitz/kernel_calEva.h:20-27).
void cu_Free_pp(std::vector<float*>, std::vector<float*>, std::vector<float*>, std::vector<float*>,
                std::vector<float*>);
double host_store_fx(std::vector<float*>, std::vector<float*>, std::vector<float*>, std::vector<float*>,
                     std::vector<float*>, std::vector<float*>, float*, int, int, int, double*, int, int, int,
                     int, int, int, int, int, double&, double, double, float, float, bool);
void cuda_configure_Pc_KMatrix(const float*);
void cuda_configure_ampcount(const float*, const int);
void cuda_configure_smear();
void host_store_amp2s(std::vector<float*>, std::vector<float*>, std::vector<float*>, std::vector<float*>,
                      std::vector<float*>, float*, int, int, int, double*, int, int, int, int, int, float, float);
void host_store_lineshapeLsKM(const float*, float*, float*, float*, float*, const int, const int, const int,
                              const float, float*, const int, const int, const int);

extern "C" {

// The three one-time configuration calls of the RooDalitzAmplitude constructor
// (RooDalitzAmplitude.cxx:519-521).  para_size = 6 * (NR + NZ + NX).
void ref_configure(const float* paraList, int para_size) {
  cuda_configure_Pc_KMatrix(paraList);
  cuda_configure_ampcount(paraList, para_size);
  cuda_configure_smear();
}

// Drops the reference's lazily allocated per-event buffers so the next call re-sizes them.
void ref_reset() {
  std::vector<float*> none(1, nullptr);
  cu_Free_pp(none, none, none, none, none);
}

// One host_store_fx call (kernel_calEva.cu:1186-1363).  Returns the MC normalisation sum and
// writes the NLL.  Buffers are host memory in the reference SoA layout.
double ref_host_store_fx(float* pp, float* pp1, float* pp2, float* pp3, float* pp4, float* sw,
                         float* h_paraList, int para_size, int vamp_size, int spline_size, double* h_fx,
                         int end, int begin, int nda, int nda_smr, int nda_fine, int NR, int NZ, int NX,
                         double* mynll, double sum_w, double sum_w_data, float ffr, float ffb,
                         int store_h_fx, int quiet) {
  std::stringstream sink;
  std::streambuf* saved = nullptr;
  if (quiet) saved = std::cout.rdbuf(sink.rdbuf());
  double nll = 0;
  const double r = host_store_fx({pp}, {pp1}, {pp2}, {pp3}, {pp4}, {sw}, h_paraList, para_size, vamp_size,
                                 spline_size, h_fx, end, begin, nda, nda_smr, nda_fine, NR, NZ, NX, nll, sum_w,
                                 sum_w_data, ffr, ffb, store_h_fx != 0);
  if (quiet) std::cout.rdbuf(saved);
  *mynll = nll;
  return r;
}

// Per-event unsmeared |A|^2 (host_store_amp2s, kernel_calEva.cu:1376-1419).
void ref_host_store_amp2s(float* pp, float* pp1, float* pp2, float* pp3, float* pp4, float* h_paraList,
                          int para_size, int vamp_size, int spline_size, double* out, int n, int NR, int NZ,
                          int NX, float ffr, float ffb) {
  host_store_amp2s({pp}, {pp1}, {pp2}, {pp3}, {pp4}, h_paraList, para_size, vamp_size, spline_size, out, n, 0,
                   NR, NZ, NX, ffr, ffb);
}

// Lambda* lineshape diagnostic (host_store_lineshapeLsKM, kernel_calEva.cu:1545-1584).  Its kernel
// has no bounds check: n_points must be a multiple of its 32-thread blocks.
void ref_host_store_lineshapeLsKM(const float* mkp, float* km_re, float* km_im, float* bw_re, float* bw_im,
                                  int n_points, int NR, int nLz, float ffr, float* h_paraList, int para_size,
                                  int vamp_size, int spline_size) {
  host_store_lineshapeLsKM(mkp, km_re, km_im, bw_re, bw_im, n_points, NR, nLz, ffr, h_paraList, para_size,
                           vamp_size, spline_size);
}
}
