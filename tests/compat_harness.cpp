// ROOT-free replay of RooDalitzAmplitude's calls into the GPU boundary (src/RooDalitzAmplitude.cxx:
// 519-521 configuration, :708-746 plane upload via cu_malloc_h_pp, :1931-1955 host_store_fx with
// the _Nda_SMR1 - 1 band argument and store_h_fx = true, destructor cu_Free_pp), linked only
// against libpwa_b200.so through include/kernel_calEva_compat.h.
//
// usage: compat_harness <dir>   reads meta.txt, pp.bin, pp1.bin, pp2.bin, sw.bin, para.bin from dir,
// writes out.txt (nll sumint) and fx.bin.
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "kernel_calEva_compat.h"

static std::vector<float> read_f(const std::string& p) {
  std::ifstream f(p, std::ios::binary | std::ios::ate);
  const size_t n = f.tellg();
  std::vector<float> v(n / sizeof(float));
  f.seekg(0);
  f.read(reinterpret_cast<char*>(v.data()), n);
  return v;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string d = argv[1];
  int n, n_size, nda, nda_smr1, nda_fine, para_size, vamp_size, NR, NZ, reps;
  double sumw, sumw_data;
  float ffr, ffb;
  FILE* m = std::fopen((d + "/meta.txt").c_str(), "r");
  if (!m || std::fscanf(m, "%d %d %d %d %d %d %d %d %d %lf %lf %f %f %d", &n, &n_size, &nda, &nda_smr1, &nda_fine,
                        &para_size, &vamp_size, &NR, &NZ, &sumw, &sumw_data, &ffr, &ffb, &reps) != 14)
    return 3;
  std::fclose(m);
  auto pp = read_f(d + "/pp.bin"), pp1 = read_f(d + "/pp1.bin"), pp2 = read_f(d + "/pp2.bin");
  auto sw = read_f(d + "/sw.bin"), para = read_f(d + "/para.bin");
  cuda_configure_Pc_KMatrix(para.data());
  cuda_configure_ampcount(para.data(), para_size);
  cuda_configure_smear();
  float *dpp, *dpp1, *dpp2, *dsw, *dpp3 = nullptr, *dpp4 = nullptr;
  cu_malloc_h_pp(pp.data(), dpp, 111 * n_size * sizeof(float), 0);
  cu_malloc_h_pp(pp1.data(), dpp1, 96 * n_size * sizeof(float), 0);
  cu_malloc_h_pp(pp2.data(), dpp2, 96 * n_size * sizeof(float), 0);
  cu_malloc_h_pp(sw.data(), dsw, n_size * sizeof(float), 0);
  std::vector<double> fx(n);
  double nll = 0, sumint = 0;
  for (int r = 0; r < reps; ++r)
    sumint = host_store_fx({dpp}, {dpp1}, {dpp2}, {dpp3}, {dpp4}, {dsw}, para.data(), para_size, vamp_size, 0,
                           fx.data(), n, 0, nda, nda_smr1 - 1, nda_fine, NR, NZ, 0, nll, sumw, sumw_data, ffr, ffb,
                           true);
  std::vector<double> amp(n);
  host_store_amp2s({dpp}, {dpp1}, {dpp2}, {dpp3}, {dpp4}, para.data(), para_size, vamp_size, 0, amp.data(), n, 0, NR,
                   NZ, 0, ffr, ffb);
  cu_Free_pp({dpp}, {dpp1}, {dpp2}, {dpp3}, {dpp4});
  FILE* o = std::fopen((d + "/out.txt").c_str(), "w");
  std::fprintf(o, "%.17g %.17g\n", nll, sumint);
  std::fclose(o);
  std::ofstream(d + "/fx.bin", std::ios::binary).write(reinterpret_cast<char*>(fx.data()), n * sizeof(double));
  std::ofstream(d + "/amp2.bin", std::ios::binary).write(reinterpret_cast<char*>(amp.data()), n * sizeof(double));
  return 0;
}
