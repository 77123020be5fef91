// TEST INFRASTRUCTURE ONLY -- C entry points for the reference's ROOT-free helpers built for host
// cores by oracle/build_ref.py: the Clebsch-Gordan tables (src/EvtCGCoefSingle.cpp) and the Wigner
// d-functions dfunhalf / dfunone / dfun (src/RooDalitzAmplitude.cxx:2443-2590).
#include "RooTDalitz/EvtCGCoefSingle.hh"

double ref_dfunhalf_impl(double beta, int am, int an);
double ref_dfunone_impl(double beta, int am, int an);
double ref_dfun_impl(double beta, double aj, double am, double an);

extern "C" {
// <j1/2 m1/2; j2/2 m2/2 | J/2 M/2>, all doubled, from EvtCGCoefSingle(j1, j2).coef(J, M, j1, j2, m1, m2).
double ref_cg(int j1, int j2, int J, int M, int m1, int m2) {
  EvtCGCoefSingle c(j1, j2);
  return c.coef(J, M, j1, j2, m1, m2);
}
double ref_dfunhalf(double beta, int am, int an) { return ref_dfunhalf_impl(beta, am, an); }
double ref_dfunone(double beta, int am, int an) { return ref_dfunone_impl(beta, am, an); }
double ref_dfun(double beta, double aj, double am, double an) { return ref_dfun_impl(beta, aj, am, an); }
}
