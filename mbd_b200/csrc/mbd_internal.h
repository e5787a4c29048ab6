// Internal declarations shared by the host planner, the kernels and the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mbd_b200.h"

namespace mbd {

constexpr int kNFreq = MBD_N_FREQ;

// Constants of init_constants (UTILS.f90:78-93) and the report (UTILS.f90:288,313).
constexpr double kBohr = 0.52917721;
constexpr double kPi = 3.14159265358979323846;
constexpr double kOtd = 0.33333333333333333333;
constexpr double kC6Prefactor = 0.954929658551372;

// Gauss-Legendre imaginary-frequency grid (UTILS.f90:1188-1211).  The
// reference writes REAL*4 literals, so the values are the float32 roundings.
extern const double kCasimirOmega[kNFreq];
extern const double kCasimirWeight[kNFreq];

struct VdwParam {
  double alpha0, c6, r0;
};
// Free-atom table of get_vdw_param (UTILS.f90:1324-1703), float32-rounded.
bool vdw_param(int z, VdwParam* out);
int element_z(const char* symbol);

// beta of get_beta (UTILS.f90:353-372), float32-rounded literals.
double beta_for_xc(int xc);

// Host-side plan of one geometry: everything derived from the inputs that is
// O(N + images) and needed to size and launch the kernels.
struct GeomPlan {
  int N = 0;                 // atoms
  int n = 0;                 // 3N, relay dimension
  int ld = 0;                // padded leading dimension of relay matrices (elements)
  int nsl = 1;               // supercell cells
  int sl[3] = {1, 1, 1};
  int nH = 0;                // 3 N nsl, CFDM dimension
  int ldH = 0;
  int n_periodic = 0;
  double beta = 0.0;
  double scs_cut = 0.0;      // bohr
  double scs_eval_cut = 0.0; // bohr: min(scs_cut, damping radius), see build_plan
  double cfdm_cut = 0.0;     // bohr
  double lat[9] = {0};       // lattice vectors, lat[3k+c], bohr
  // SCS translations t = -(n1 a1 + n2 a2 + n3 a3) that can reach some pair
  // within scs_eval_cut; xyz triples.  The zero translation is always first.
  std::vector<double> scs_shifts;
  // CFDM translations -(n . A_SL) that can reach some pair within cfdm_cut.
  std::vector<double> cfdm_shifts;
  // Distinct cell differences (rc - cc) of the supercell, as translations
  // (rc - cc) . a, plus for each the list of (row cell, col cell) indices.
  std::vector<double> diff_shift;       // 3 per difference
  std::vector<int> diff_is_zero;        // 1 for the zero difference
  std::vector<int> place_offset;        // CSR offsets into place_rc/place_cc, per difference
  std::vector<int> place_rc, place_cc;  // cell indices (k*SLj*SLi + j*SLi + i)
  int vac[3] = {0, 0, 0};     // vacuum axes (no images along them)
  std::vector<int> species;   // learned warm start: 0 H, 1 C, 2 N, 3 O, 4 other
  // per-atom free-atom data
  std::vector<double> alpha0, c6free, r0, hirsh;
  std::vector<double> coords;           // 3N, xyz per atom (bohr)
  // Per-atom arrays above are in an internal spatial order: internal atom q
  // is the caller's atom perm[q] (results are scattered back on download).
  std::vector<int> perm;
};

// Builds the plan; returns an MBD_* status.
int build_plan(const mbd_geom& g, GeomPlan* p);

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace mbd
