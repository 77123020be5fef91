/* kernel_calEva_compat.h -- the reference's GPU boundary with its exact C++ signatures
 * (RooTDalitz/kernel_calEva.h:20-27), implemented by libpwa_b200.so on top of pwa_b200.h.
 *
 * An unmodified src/RooDalitzAmplitude.cxx links against these symbols.  Semantics follow
 * src/kernel_calEva.cu, with the differences listed per function.  Errors are reported on stderr
 * and turned into a NaN NLL / NaN return value instead of cudaDeviceReset() + assert(0).
 */
#ifndef PWA_KERNEL_CALEVA_COMPAT_H
#define PWA_KERNEL_CALEVA_COMPAT_H

#include <vector>

/* Allocates mem_length bytes on device `device` and copies the host plane there
 * (kernel_calEva.cu:1447-1457). */
void cu_malloc_h_pp(float* h_float_pp, float*& d_float_pp, int mem_length, int device);

/* Frees the five plane vectors and the per-event buffers (kernel_calEva.cu:1459-1493). */
void cu_Free_pp(std::vector<float*> d_float_pp, std::vector<float*> d_float_pp1, std::vector<float*> d_float_pp2,
                std::vector<float*> d_float_pp3, std::vector<float*> d_float_pp4);

/* One likelihood evaluation (kernel_calEva.cu:1186-1363).  Returns the MC normalisation sum and
 * writes the NLL to mynll.  NUMLz/NUMPc/NUMZcs are the model sizes (compile-time constants in the
 * reference, run-time here); the Zcs planes d_float_pp3 / d_float_pp4 are read when NUMZcs > 0.
 * h_fx receives all per-event values when store_h_fx is true. */
double host_store_fx(std::vector<float*> d_float_pp, std::vector<float*> d_float_pp1,
                     std::vector<float*> d_float_pp2, std::vector<float*> d_float_pp3,
                     std::vector<float*> d_float_pp4, std::vector<float*> d_float_sw, float* h_paraList,
                     int para_size, int vamp_size, int paraSpline_size, double* h_fx, int end, int begin, int Nda,
                     int Nda_SMR, int Nda_SMR_finebinning, int NUMLz, int NUMPc, int NUMZcs, double& mynll,
                     double SumW, double sumW_data, float _FFR, float _FFB, bool store_h_fx);

/* Resonance-table driven one-time configuration (kernel_calEva.cu:978-1152).  The tables they
 * filled are derived from the parameter block on every call here, so these validate and record the
 * model sizes only. */
void cuda_configure_Pc_KMatrix(const float* paraList);
void cuda_configure_ampcount(const float* paraList, const int paraSize);
void cuda_configure_smear();

/* Per-event unsmeared |A|^2 (kernel_calEva.cu:1376-1419). */
void host_store_amp2s(std::vector<float*> d_float_pp, std::vector<float*> d_float_pp1,
                      std::vector<float*> d_float_pp2, std::vector<float*> d_float_pp3,
                      std::vector<float*> d_float_pp4, float* h_paraList, int para_size, int vamp_size,
                      int paraSpline_size, double* h_amp2s, int end, int begin, int NUMLz, int NUMPc, int NUMZcs,
                      float _FFR, float _FFB);

/* Lambda* lineshape diagnostic (kernel_calEva.cu:1545-1584): revised K-matrix and Breit-Wigner
 * lineshapes of every Lambda* entry (times the Lambda_b barrier with radius _FFR) at n_points masses,
 * written as floats to [iLz * n_points + i] for iLz < NR (nLz >= NR rows must fit).  Computed in FP64 by
 * pwa_lineshapes_lstar_km and rounded to float. */
void host_store_lineshapeLsKM(const float* h_mkp, float* h_KM_real, float* h_KM_imag, float* h_BW_real,
                              float* h_BW_imag, const int n_points, const int NR, const int nLz, const float _FFR,
                              float* h_paraList, const int para_size, const int vamp_size,
                              const int paraSpline_size);

#endif
