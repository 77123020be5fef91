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
constexpr int MAX_ZCS = 4;
constexpr int MAX_GROUPS = MAX_PC + 4;  // K-matrix J^P groups + one group per non-K-matrix Pc entry
constexpr int NSET = 6;

// Lineshapes: Breit-Wigner, constant (non-resonant), coupled-channel K-matrix, spline
// (model-independent wave), revised K-matrix, triangle cusp.
enum LineType : int { LT_BW = 1, LT_NR = 2, LT_KM = 3, LT_SPLINE = 4, LT_RKM = 5, LT_CUSP = 6 };
// Lineshape type codes of the parameter block (Resonances.h:108-120).
constexpr int REF_BREITWIGNER = 1;
constexpr int REF_MODELINDEPENDENT = 3;
constexpr int REF_TRIANGLE = 7;
constexpr int REF_KMATRIX = 240;
constexpr int REF_REVISEDKMATRIX = 360;
constexpr int REF_NONRESONANT = 361;
// Spline knots of the Lambda* and Pc model-independent waves (Resonances.h:5-6); a spline block holds
// the knots, (y, b, c, d) per knot of the real part, then of the imaginary part: 9 floats per knot.
constexpr int SPL_KNOTS_L = 24, SPL_KNOTS_Z = 11;
constexpr int SPL_FLOATS = 2 * 9 * SPL_KNOTS_L + 2 * 9 * SPL_KNOTS_Z;  // two waves of each chain
// Entries of revised K-matrices per chain (all spin-parity sets together).
constexpr int MAX_RKM = 6;

// Revised K-matrix entry (Revised_KMAMP, cu_DPFPropogator.cu:825-926): the constants of its own term
// (chain two-body system) and of the term it adds to the other entries of its set (KMatrixTerm,
// :928-972, always in the p K system).  Entries with equal spin and parity form one set.
struct RkmEntry {
  int set;     // 2J * 2 + (P > 0): entries with equal set are coupled
  int LR;
  int branch;  // own term: 0 mass above the chain threshold, 1 below it (Sigma pi channel),
               // 2 at it, 3 non-resonant (mass <= 0)
  int pad;
  double m, g;
  double inv_pR0c, polyR0c;  // own term: 1 / reference momentum, Blatt-Weisskopf polynomial there
  double inv_pR0sp;          // branch 1: 1 / Sigma pi momentum at the mass
  double factor;             // 0.948850 m sqrt(g kr / sqrt(m (m + kr))) for m > 0, else 1
  double inv_pR0k, polyR0k;  // KMatrixTerm: p K reference momentum and polynomial
};

struct LstarEntry {
  int type;   // LT_BW, LT_NR, LT_SPLINE, LT_RKM
  int sidx;   // d-function spin index (2J-1)/2
  int LR, LB;
  int branch;  // 0: m_r above pK threshold, 1: below threshold (Sigma pi channel), 2: m_r < 0
  int ncm;     // helicity couplings per proton helicity: 4 (J=1/2) or 6
  double m_r, g_r, pR0, polyR0, norm, pR0_sp;  // Breit-Wigner constants
  double pB0, polyB0, lb_scale;                // Lambda_b barrier: F ratio * (pB/mLb)^LB * lb_scale
  double inv_pR0, sqrt_polyR0, inv_pR0_sp, sqrt_polyB0;  // the same constants in the form the kernels use
  cplx c[12];                                  // c[k*6+m]; |c| < 1e-10 stored as 0
  int aux;  // LT_SPLINE: first float of its block in PointTable::spl; LT_RKM: index in PointTable::rkm[0]
};

struct PcEntry {
  int type;  // LT_BW, LT_NR, LT_KM, LT_SPLINE, LT_RKM, LT_CUSP
  int sidx, LR, LB;
  int group, slot;  // K-matrix J^P group and P-vector output slot
  int bw_above;     // Breit-Wigner mass above J/psi p threshold
  int pB0_event;    // Lambda_b barrier momentum at the resonance equals the event's (m0 in [0,1e-10])
  double m_r, g_r, pR0, polyR0, norm;
  double pB0, polyB0;
  double inv_pR0, sqrt_polyR0, sqrt_polyB0;
  cplx c[24];  // c[k*12+m], 12 helicity slots per proton helicity (disallowed slots are 0)
  int aux;     // LT_SPLINE: first float of its block in PointTable::spl; LT_RKM: index in PointTable::rkm[1]
};

// Zcs -> J/psi K entry (Breit-Wigner BW_AMPX with production barrier BTermX,
// cu_DPFPropogator.cu:205-246).  Couplings in the order GetAmpZcs (kernel_calEva.cu:192-286) reads
// them: per proton helicity k, N(J) consecutive (Re, Im) pairs from the resonance's coupling offset
// (N = 0, 9, 12, 12 for 2J = 0, 2, 4, 6), slot m of c[k*12+m] selecting the AX / DX planes.
struct XEntry {
  int sidx;      // DX spin index 2J / 2
  int LR, LB;
  int bw_above;  // Breit-Wigner mass above the J/psi K threshold
  int lb_mode;   // production barrier: 0 F ratio with pB0(m_r), 1 ratio 1 (pB0 = event's), 2 no ratio
  int pad;
  double m_r, g_r, norm, inv_pR0, sqrt_polyR0, sqrt_polyB0;
  cplx c[24];
};

struct KmGroup {
  int J2, P, Lna, npole;
  int iso, pad;           // 1: the 7-channel isospin-split K-matrix (the reference's ISOSPIN_SIGMACD build)
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
  int mmask[2];      // helicity slots with a non-zero coupling in any entry, per proton helicity
};

// Per-point tables of every Pc entry's lineshape (production barrier included; all of them depend on
// m(J/psi p) only) on a uniform grid, interpolated with 6-point Lagrange polynomials.  Guard
// intervals surround every mass where the reference's lineshapes are not smooth (real-mass
// thresholds, the branch switches of its complex square root, the K-matrix pole clamp
// |m0^2 - s| < 1e-3, the upper kinematic edge).  In addition every grid interval is verified after
// the table is built: its interpolant is compared with exact evaluations at interior points, group by
// group, and intervals off by more than TAB_CHECK_TOL relative to the group's largest entry
// (parameter-dependent narrow states, e.g. a K-matrix pole just below a real-mass threshold) are
// flagged and refined.  Lookups that neither level can serve, and those near the grid ends, evaluate
// the lineshapes exactly.
constexpr int MAX_GUARDS = 48;
// Entries of one Pc group (a K-matrix J^P group shares one solve).
constexpr int MAX_GROUP_ENTRIES = 8;
// Intervals that fail the check are refined: each gets a block of TAB_SUB sub-intervals (step
// h / TAB_SUB) with TAB_SUB + 5 nodes (the 6-point stencils of all sub-intervals), verified the same
// way.  Up to TAB_MAX_BLOCKS intervals are refined per point; the others and sub-intervals that fail
// again are evaluated exactly.
constexpr int TAB_SUB = 16;
constexpr int TAB_SUB_NODES = TAB_SUB + 5;
constexpr int TAB_MAX_BLOCKS = 4096;
struct LineTables {
  int enabled;
  int n_nodes, stride;  // stride: complex values per node (entries in group order)
  // The table holds groups [g_lo, g_hi), whose entries start at order position pos0: every group
  // for a context's table (stride NZ), one group for a batch point that moves only that group's
  // lineshape (stride = its entry count, on the coarser group grid below).
  int g_lo, g_hi, pos0;
  double m_lo, h, inv_h;
  int nguard;
  double guard_lo[MAX_GUARDS], guard_hi[MAX_GUARDS];
  const cplx* data;   // [node][order position]
  const int* cell;    // per interval [j, j+1]: 0 interpolate, -1 exact, b + 1 refined in block b
  const cplx* sub;    // [block][TAB_SUB_NODES][order position]
  const unsigned char* sub_bad;  // [block][TAB_SUB]: 1 when lookups must evaluate exactly
  int* nblocks;       // refined-block counter (reset by the build kernel)
  int* block_interval;  // [block] -> interval j
};
constexpr double TAB_CHECK_TOL = 1e-11;
constexpr double TAB_M_LO = 4.030, TAB_M_HI = 5.130, TAB_H = 1e-5;  // GeV
constexpr int TAB_NODES = 110001;
// Device memory a context attaches for the tables (bytes, 256-aligned parts).
constexpr size_t tab_align(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t TAB_BYTES_DATA = tab_align((size_t)TAB_NODES * MAX_PC * 16);
constexpr size_t TAB_BYTES_CELL = tab_align((size_t)TAB_NODES * 4);
constexpr size_t TAB_BYTES_SUB = tab_align((size_t)TAB_MAX_BLOCKS * TAB_SUB_NODES * MAX_PC * 16);
constexpr size_t TAB_BYTES_SUB_BAD = tab_align((size_t)TAB_MAX_BLOCKS * TAB_SUB);
constexpr size_t TAB_BYTES_BLOCKS = tab_align((size_t)(TAB_MAX_BLOCKS + 1) * 4);
constexpr size_t TAB_BYTES =
    TAB_BYTES_DATA + TAB_BYTES_CELL + TAB_BYTES_SUB + TAB_BYTES_SUB_BAD + TAB_BYTES_BLOCKS;
// A table of one Pc group (a batch point that moves only that group's lineshape): the same grid,
// stride = the group's entry count.
constexpr size_t TAB_BYTES_GROUP_DATA = tab_align((size_t)TAB_NODES * MAX_GROUP_ENTRIES * 16);
constexpr size_t TAB_BYTES_GROUP_SUB = tab_align((size_t)TAB_MAX_BLOCKS * TAB_SUB_NODES * MAX_GROUP_ENTRIES * 16);
constexpr size_t TAB_BYTES_GROUP = TAB_BYTES_GROUP_DATA + TAB_BYTES_CELL + TAB_BYTES_GROUP_SUB +
                                   TAB_BYTES_SUB_BAD + TAB_BYTES_BLOCKS;

// Plane slots of one event staged in shared memory (as doubles): pp 111, pp1 96, pp2 96, pp3 97, pp4 96.
constexpr int SLOT_PP = 0, SLOT_PP1 = 111, SLOT_PP2 = 207, SLOT_PP3 = 303, SLOT_PP4 = 400, SLOT_ALL = 496;

struct alignas(16) PointTable {
  int NR, NZ, ngroups;
  int status;  // 0 ok, else a PWA_E_* code
  int NX;      // Zcs entries
  int lmask_x_R, lmask_x_B;  // Blatt-Weisskopf orders of the Zcs decay and production barriers
  int x_mmask[2];            // Zcs helicity slots with a non-zero coupling, per proton helicity
  // Blatt-Weisskopf orders L in use (bit L set): decay barriers of the Lambda* Breit-Wigners, their
  // production barriers, production barriers of the Pc entries, decay barriers of Pc Breit-Wigners;
  // needs_sigma_pi: a Lambda* below the pK threshold uses the Sigma pi channel momentum.
  int lmask_lstar_R, lmask_lstar_B, lmask_pc_B, lmask_pc_R, needs_sigma_pi;
  // helicity slots m (bit m) with a non-zero coupling, per proton helicity k
  int lstar_mmask[2], pc_mmask[2];
  double ffr, ffb;
  LstarEntry L[MAX_LSTAR];
  PcEntry Z[MAX_PC];
  XEntry X[MAX_ZCS];
  KmGroup G[4];
  PcGroup grp[MAX_GROUPS];
  int order[MAX_PC];  // Pc entries in group order
  LineTables tab;
  // the plane slots this point's amplitude reads (kernels that stage an event copy only these)
  int nstage;
  short stage[SLOT_ALL];
  // revised K-matrix entries per chain (0 Lambda*, 1 Pc) in resonance order, and spline blocks
  int nrkm[2];
  RkmEntry rkm[2][MAX_RKM];
  float spl[SPL_FLOATS];
};

}  // namespace pwa
