// Per-parameter-point table: the float parameter block (the reference's h_paraList, layout of
// RooDalitzAmplitude::cu_init_data, src/RooDalitzAmplitude.cxx:3141-3210) decoded once per point into
// FP64 coefficients and every constant that does not depend on the event.  Built on the host
// (build_point_table) and copied to the device; kernels read it from shared memory.
#pragma once
#include <cstdint>

#include "pwa_physics.cuh"

namespace pwa {

constexpr int MAX_LSTAR = 24;
constexpr int MAX_PC = 16;
constexpr int MAX_GROUPS = MAX_PC + 4;  // K-matrix J^P groups + one group per non-K-matrix Pc entry
constexpr int NSET = 6;

enum LineType : int { LT_BW = 1, LT_NR = 2, LT_KM = 3 };
// Lineshape type codes of the parameter block (Resonances.h:97-108).
constexpr int REF_BREITWIGNER = 1;
constexpr int REF_KMATRIX = 240;
constexpr int REF_NONRESONANT = 361;

struct LstarEntry {
  int type;   // LT_BW or LT_NR
  int sidx;   // d-function spin index (2J-1)/2
  int LR, LB;
  int branch;  // 0: m_r above pK threshold, 1: below threshold (Sigma pi channel), 2: m_r < 0
  int ncm;     // helicity couplings per proton helicity: 4 (J=1/2) or 6
  double m_r, g_r, pR0, polyR0, norm, pR0_sp;  // Breit-Wigner constants
  double pB0, polyB0, lb_scale;                // Lambda_b barrier: F ratio * (pB/mLb)^LB * lb_scale
  double inv_pR0, sqrt_polyR0, inv_pR0_sp, sqrt_polyB0;  // the same constants in the form the kernels use
  cplx c[12];                                  // c[k*6+m]; |c| < 1e-10 stored as 0
};

struct PcEntry {
  int type;  // LT_BW, LT_NR, LT_KM
  int sidx, LR, LB;
  int group, slot;  // K-matrix J^P group and P-vector output slot
  int bw_above;     // Breit-Wigner mass above J/psi p threshold
  int pB0_event;    // Lambda_b barrier momentum at the resonance equals the event's (m0 in [0,1e-10])
  double m_r, g_r, pR0, polyR0, norm;
  double pB0, polyB0;
  double inv_pR0, sqrt_polyR0, sqrt_polyB0;
  cplx c[24];  // c[k*12+m], 12 helicity slots per proton helicity (disallowed slots are 0)
};

struct KmGroup {
  int J2, P, Lna, npole;
  double m0sq[NPMAX];     // pole mass^2 after the near-threshold shift
  double g[NPMAX][NKMC];  // pole couplings
  double f[NKMC][NKMC];   // scattering matrix
};

// Pc entries are evaluated group by group: a K-matrix J^P group shares one solve; every other
// entry is a group of its own.  Entries of a group share the d-function spin index.
struct PcGroup {
  int km;       // K-matrix group index (0..3) or -1
  int sidx;     // common spin index
  int first, count;  // range in PointTable::order
};

// Per-point tables of the K-matrix P-vector outputs on a uniform m(J/psi p) grid, interpolated with
// 6-point Lagrange polynomials.  Guard intervals surround every mass where the reference's lineshape
// is not smooth (real-mass thresholds, the branch switches of its complex square root, the pole
// clamp |m0^2 - s| < 1e-3, the upper kinematic edge).  In addition every grid interval is verified
// after the table is built: its interpolant is compared with exact solves at interior points, and
// intervals off by more than TAB_CHECK_TOL (parameter-dependent narrow states, e.g. a K-matrix pole
// just below a real-mass threshold) are flagged.  Lookups in a guard interval, a flagged interval or
// near the grid ends evaluate the K-matrix exactly.
constexpr int MAX_GUARDS = 48;
struct LineTables {
  int enabled;
  int n_nodes;
  double m_lo, h, inv_h;
  int nguard;
  double guard_lo[MAX_GUARDS], guard_hi[MAX_GUARDS];
  const cplx* data[4];          // per K-matrix J^P group: [node][output], NPMAX + NKMC outputs per node
  const unsigned char* bad[4];  // per group and interval: 1 when the interpolant failed the check
};
constexpr double TAB_CHECK_TOL = 1e-11;
constexpr double TAB_M_LO = 4.030, TAB_M_HI = 5.130, TAB_H = 1e-5;  // GeV
constexpr int TAB_NODES = 110001;
constexpr int TAB_SLOTS = NPMAX + NKMC;

struct PointTable {
  int NR, NZ, ngroups;
  int status;  // 0 ok, else a PWA_E_* code
  // Blatt-Weisskopf orders L in use (bit L set): decay barriers of the Lambda* Breit-Wigners, their
  // production barriers, production barriers of the Pc entries, decay barriers of Pc Breit-Wigners;
  // needs_sigma_pi: a Lambda* below the pK threshold uses the Sigma pi channel momentum.
  int lmask_lstar_R, lmask_lstar_B, lmask_pc_B, lmask_pc_R, needs_sigma_pi;
  double ffr, ffb;
  LstarEntry L[MAX_LSTAR];
  PcEntry Z[MAX_PC];
  KmGroup G[4];
  PcGroup grp[MAX_GROUPS];
  int order[MAX_PC];  // Pc entries in group order
  LineTables tab;
};

}  // namespace pwa
