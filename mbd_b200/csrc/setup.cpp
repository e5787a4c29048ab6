// Host-side planning: free-atom table, beta, image ranges, supercell, and
// the translation lists the tensor-build kernels iterate over.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "mbd_internal.h"

namespace mbd {

namespace {
// Fortran REAL*4 literal -> the double the reference computes with.
constexpr double f32(double v) { return static_cast<double>(static_cast<float>(v)); }
}  // namespace

// UTILS.f90:1189-1209 (REAL*4 literals).
const double kCasimirOmega[kNFreq] = {
    f32(0.0000000), f32(0.0392901), f32(0.1183580), f32(0.1989120), f32(0.2820290),
    f32(0.3689190), f32(0.4610060), f32(0.5600270), f32(0.6681790), f32(0.7883360),
    f32(0.9243900), f32(1.0817900), f32(1.2684900), f32(1.4966100), f32(1.7856300),
    f32(2.1691700), f32(2.7106200), f32(3.5457300), f32(5.0273400), f32(8.4489600),
    f32(25.451700)};
const double kCasimirWeight[kNFreq] = {
    f32(0.0000000), f32(0.0786611), f32(0.0796400), f32(0.0816475), f32(0.0847872),
    f32(0.0892294), f32(0.0952317), f32(0.1031720), f32(0.1136050), f32(0.1273500),
    f32(0.1456520), f32(0.1704530), f32(0.2049170), f32(0.2544560), f32(0.3289620),
    f32(0.4480920), f32(0.6556060), f32(1.0659600), f32(2.0635700), f32(5.6851000),
    f32(50.955800)};

namespace {
struct Entry {
  int z;
  const char* sym;
  double alpha0, c6, r0;
};
// Tkatchenko-Scheffler free-atom polarizability alpha0 [bohr^3], C6 [Ha bohr^6]
// and vdW radius R0 [bohr] for H..Rn as listed by get_vdw_param
// (UTILS.f90:1336-1691); La..Lu have no entry there and are rejected.
const Entry kTable[] = {
    {1, "H", 4.5, 6.5, 3.1},           {2, "He", 1.38, 1.46, 2.65},
    {3, "Li", 164.2, 1387.0, 4.16},    {4, "Be", 38.0, 214.0, 4.17},
    {5, "B", 21.0, 99.5, 3.89},        {6, "C", 12.0, 46.6, 3.59},
    {7, "N", 7.4, 24.2, 3.34},         {8, "O", 5.4, 15.6, 3.19},
    {9, "F", 3.8, 9.52, 3.04},         {10, "Ne", 2.67, 6.38, 2.91},
    {11, "Na", 162.7, 1556.0, 3.73},   {12, "Mg", 71.0, 627.0, 4.27},
    {13, "Al", 60.0, 528.0, 4.33},     {14, "Si", 37.0, 305.0, 4.2},
    {15, "P", 25.0, 185.0, 4.01},      {16, "S", 19.6, 134.0, 3.86},
    {17, "Cl", 15.0, 94.6, 3.71},      {18, "Ar", 11.1, 64.3, 3.55},
    {19, "K", 292.9, 3897.0, 3.71},    {20, "Ca", 160.0, 2221.0, 4.65},
    {21, "Sc", 120.0, 1383.0, 4.59},   {22, "Ti", 98.0, 1044.0, 4.51},
    {23, "V", 84.0, 832.0, 4.44},      {24, "Cr", 78.0, 602.0, 3.99},
    {25, "Mn", 63.0, 552.0, 3.97},     {26, "Fe", 56.0, 482.0, 4.23},
    {27, "Co", 50.0, 408.0, 4.18},     {28, "Ni", 48.0, 373.0, 3.82},
    {29, "Cu", 42.0, 253.0, 3.76},     {30, "Zn", 40.0, 284.0, 4.02},
    {31, "Ga", 60.0, 498.0, 4.19},     {32, "Ge", 41.0, 354.0, 4.2},
    {33, "As", 29.0, 246.0, 4.11},     {34, "Se", 25.0, 210.0, 4.04},
    {35, "Br", 20.0, 162.0, 3.93},     {36, "Kr", 16.8, 129.6, 3.82},
    {37, "Rb", 319.2, 4691.0, 3.72},   {38, "Sr", 199.0, 3170.0, 4.54},
    {39, "Y", 126.737, 1968.58, 4.8151}, {40, "Zr", 119.97, 1677.91, 4.53},
    {41, "Nb", 101.603, 1263.61, 4.2365}, {42, "Mo", 88.4225785, 1028.73, 4.099},
    {43, "Tc", 80.083, 1390.87, 4.076}, {44, "Ru", 65.895, 609.754, 3.9953},
    {45, "Rh", 56.1, 469.0, 3.95},     {46, "Pd", 23.68, 157.5, 3.66},
    {47, "Ag", 50.6, 339.0, 3.82},     {48, "Cd", 39.7, 452.0, 3.99},
    {49, "In", 70.22, 707.046, 4.23198}, {50, "Sn", 55.95, 587.417, 4.303},
    {51, "Sb", 43.67197, 459.322, 4.276}, {52, "Te", 37.65, 396.0, 4.22},
    {53, "I", 35.0, 385.0, 4.17},      {54, "Xe", 27.3, 285.9, 4.08},
    {55, "Cs", 427.12, 6582.08, 3.78}, {56, "Ba", 275.0, 5727.0, 4.77},
    {72, "Hf", 99.52, 1274.8, 4.21},   {73, "Ta", 82.53, 1019.92, 4.15},
    {74, "W", 71.041, 847.93, 4.08},   {75, "Re", 63.04, 710.2, 4.02},
    {76, "Os", 55.055, 596.67, 3.84},  {77, "Ir", 42.51, 359.1, 4.0},
    {78, "Pt", 39.68, 347.1, 3.92},    {79, "Au", 36.5, 298.0, 3.86},
    {80, "Hg", 33.9, 392.0, 3.98},     {81, "Tl", 69.92, 717.44, 3.91},
    {82, "Pb", 61.8, 697.0, 4.31},     {83, "Bi", 49.02, 571.0, 4.32},
    {84, "Po", 45.013, 530.92, 4.097}, {85, "At", 38.93, 457.53, 4.07},
    {86, "Rn", 33.54, 390.63, 4.23},
};
constexpr int kTableSize = sizeof(kTable) / sizeof(kTable[0]);

double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Atoms in Morton (Z-curve) order of their coordinates: perm[p] = the
// caller's index of internal atom p.  Consecutive internal atoms are then
// spatial neighbours, so a 64-row diagonal tile of the relay matrix holds the
// strongest couplings of its ~21 atoms (the block-CG preconditioner of the
// MIXED_LEARNED mode inverts those tiles).  Ties keep the input order.
void spatial_order(const double* xyz, int N, std::vector<int>* perm) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::min(lo[c], xyz[3 * i + c]);
      hi[c] = std::max(hi[c], xyz[3 * i + c]);
    }
  const double ext = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), std::max(hi[2] - lo[2], 1e-300));
  std::vector<std::pair<uint32_t, int>> key(N);
  for (int i = 0; i < N; ++i) {
    uint32_t code = 0;
    uint32_t q[3];
    for (int c = 0; c < 3; ++c) q[c] = (uint32_t)std::min(1023.0, std::floor((xyz[3 * i + c] - lo[c]) / ext * 1024.0));
    for (int b = 0; b < 10; ++b)
      for (int c = 0; c < 3; ++c) code |= ((q[c] >> b) & 1u) << (3 * b + c);
    key[i] = {code, i};
  }
  std::stable_sort(key.begin(), key.end(), [](const std::pair<uint32_t, int>& a, const std::pair<uint32_t, int>& b) {
    return a.first < b.first;
  });
  perm->resize(N);
  for (int p = 0; p < N; ++p) (*perm)[p] = key[p].second;
}

// Upper bound of every entry of the short-range tensor at distance r
// (gaussian_dipole_tensor, UTILS.f90:637-696):
//   |(3 dd - r^2 I) zeta_l| <= 2/r^3        since 0 <= erf(x) - 2/sqrt(pi) x e^{-x^2} <= 1,
//   |dd zeta_r|             <= 4/sqrt(pi) e^{-r^2/sgm_hi^2} / sgm_lo^3,
//   1 - fermi               <= exp(-6 (r/(beta R_hi) - 1)).
double sr_tensor_bound(double r, double beta_rhi, double sgm_lo, double sgm_hi) {
  double g = 2.0 / (r * r * r) + 4.0 / std::sqrt(kPi) * std::exp(-(r * r) / (sgm_hi * sgm_hi)) /
                                     (sgm_lo * sgm_lo * sgm_lo);
  return g * std::exp(-6.0 * (r / beta_rhi - 1.0));
}

// Image box of get_scs_image / get_cfdm_image (UTILS.f90:1215-1248,1287-1320):
// +-ceil(cut/|a_k|) on periodic, non-vacuum axes, 0 otherwise.
void image_box(const double* lat, int n_periodic, const int* vacuum, double cut, int rng[3]) {
  for (int k = 0; k < 3; ++k) {
    rng[k] = 0;
    if (n_periodic != 0 && !vacuum[k]) rng[k] = (int)std::ceil(cut / norm3(lat + 3 * k));
  }
}

// Translations -(n . lat) of the box whose length is <= reach, zero first.
void collect_shifts(const double* lat, const int rng[3], double reach, bool include_zero,
                    std::vector<double>* out) {
  out->clear();
  if (include_zero) out->insert(out->end(), {0.0, 0.0, 0.0});
  for (int i = -rng[0]; i <= rng[0]; ++i)
    for (int j = -rng[1]; j <= rng[1]; ++j)
      for (int k = -rng[2]; k <= rng[2]; ++k) {
        if (i == 0 && j == 0 && k == 0) continue;
        double t[3];
        for (int c = 0; c < 3; ++c) t[c] = -(i * lat[c] + j * lat[3 + c] + k * lat[6 + c]);
        if (norm3(t) <= reach) out->insert(out->end(), {t[0], t[1], t[2]});
      }
}
}  // namespace

bool vdw_param(int z, VdwParam* out) {
  for (int i = 0; i < kTableSize; ++i)
    if (kTable[i].z == z) {
      out->alpha0 = f32(kTable[i].alpha0);
      out->c6 = f32(kTable[i].c6);
      out->r0 = f32(kTable[i].r0);
      return true;
    }
  return false;
}

int element_z(const char* symbol) {
  if (!symbol) return 0;
  // CHARACTER*2 semantics: first two characters, trailing blanks ignored, case-sensitive.
  char s[3] = {0, 0, 0};
  for (int i = 0; i < 2 && symbol[i] && symbol[i] != ' '; ++i) s[i] = symbol[i];
  for (int i = 0; i < kTableSize; ++i)
    if (std::strcmp(kTable[i].sym, s) == 0) return kTable[i].z;
  return 0;
}

double beta_for_xc(int xc) {
  switch (xc) {
    case 1: return f32(0.83);
    case 2: return f32(0.85);
    case 3: return f32(0.85);
    default: return 1.0;
  }
}

int build_plan(const mbd_geom& g, GeomPlan* p) {
  if (g.n_atoms < 1 || !g.z || !g.coords_bohr || !g.hirshfeld) return MBD_ERR_ARG;
  if (g.n_periodic != 0 && !g.lattice_bohr) return MBD_ERR_ARG;
  const int N = g.n_atoms;
  p->N = N;
  p->n = 3 * N;
  p->ld = round_up(p->n, 32);
  p->n_periodic = g.n_periodic;
  p->beta = beta_for_xc(g.xc);
  p->scs_cut = g.scs_cut_A / kBohr;
  p->cfdm_cut = g.cfdm_cut_A / kBohr;
  for (int i = 0; i < 9; ++i) p->lat[i] = g.n_periodic ? g.lattice_bohr[i] : 0.0;
  p->alpha0.resize(N);
  p->c6free.resize(N);
  p->r0.resize(N);
  p->hirsh.resize(N);
  p->coords.resize(3 * N);
  for (int k = 0; k < 3; ++k) p->vac[k] = (g.n_periodic != 0 && g.vacuum[k]) ? 1 : 0;
  p->species.resize(N);
  for (int i = 0; i < N; ++i) {
    VdwParam v;
    if (!vdw_param(g.z[i], &v)) return MBD_ERR_UNKNOWN_ELEMENT;
    if (!(g.hirshfeld[i] > 0.0) || !std::isfinite(g.hirshfeld[i])) return MBD_ERR_ARG;
    for (int c = 0; c < 3; ++c)
      if (!std::isfinite(g.coords_bohr[3 * i + c])) return MBD_ERR_ARG;
  }
  // every per-atom array in the internal (spatial) order
  spatial_order(g.coords_bohr, N, &p->perm);
  for (int q = 0; q < N; ++q) {
    const int i = p->perm[q];
    VdwParam v;
    vdw_param(g.z[i], &v);
    p->species[q] = g.z[i] == 1 ? 0 : g.z[i] == 6 ? 1 : g.z[i] == 7 ? 2 : g.z[i] == 8 ? 3 : 4;
    p->alpha0[q] = v.alpha0;
    p->c6free[q] = v.c6;
    p->r0[q] = v.r0;
    p->hirsh[q] = g.hirshfeld[i];
    for (int c = 0; c < 3; ++c) p->coords[3 * q + c] = g.coords_bohr[3 * i + c];
  }

  // Supercell (get_supercell, UTILS.f90:1252-1283).
  p->nsl = 1;
  for (int k = 0; k < 3; ++k) {
    p->sl[k] = 1;
    if (g.n_periodic != 0 && !g.vacuum[k])
      p->sl[k] = (int)std::ceil((g.sc_cut_A / kBohr) / norm3(p->lat + 3 * k));
    if (p->sl[k] < 1) return MBD_ERR_ARG;
    p->nsl *= p->sl[k];
  }
  p->nH = p->n * p->nsl;
  p->ldH = round_up(p->nH, 32);
  double lat_sl[9];
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) lat_sl[3 * k + c] = p->lat[3 * k + c] * p->sl[k];

  // Extent of the atom set (upper bound of any |r_i - r_j|).
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < N; ++i)
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::min(lo[c], p->coords[3 * i + c]);
      hi[c] = std::max(hi[c], p->coords[3 * i + c]);
    }
  double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const double diam = norm3(ext);

  // Short-range damping radius.  Beyond it every SR tensor entry is below
  // 1e-30 of the smallest 1/alpha on the relay diagonal, so skipping the term
  // leaves the FP64 relay matrix unchanged to ~1e-30 relative; the
  // reference's own r <= mbd_scs_dip_cutoff test (UTILS.f90:574,623) still
  // applies inside it.
  // sigma = (alpha / 3 sqrt(2 / pi))^(1/3) rises with alpha: its extremes
  // come from the extremes of alpha over atoms and frequencies
  double rmax_iso = 0.0, amax = 0.0, amin = 1e300;
  for (int i = 0; i < N; ++i) {
    rmax_iso = std::max(rmax_iso, std::pow(p->hirsh[i], kOtd) * p->r0[i]);
    for (int f = 0; f < kNFreq; ++f) {
      double w = kCasimirOmega[f];
      double wp = (4.0 / 3.0) * p->c6free[i] / (p->alpha0[i] * p->alpha0[i]);
      double aw = (p->hirsh[i] * p->alpha0[i]) / (1.0 + (w * w) / (wp * wp));
      amin = std::min(amin, aw);
      amax = std::max(amax, aw);
    }
  }
  const double sgm_lo = std::pow((amin / 3.0) * std::sqrt(2.0 / kPi), kOtd);
  const double sgm_hi = std::pow((amax / 3.0) * std::sqrt(2.0 / kPi), kOtd) * std::sqrt(2.0);
  const double beta_rhi = p->beta * 2.0 * rmax_iso;
  const double tau = 1e-30 / amax;
  double r_lo = beta_rhi, r_hi = beta_rhi * 64.0 + 64.0;
  while (sr_tensor_bound(r_hi, beta_rhi, sgm_lo, sgm_hi) > tau) r_hi *= 2.0;
  for (int it = 0; it < 100; ++it) {
    double mid = 0.5 * (r_lo + r_hi);
    if (sr_tensor_bound(mid, beta_rhi, sgm_lo, sgm_hi) > tau) r_lo = mid; else r_hi = mid;
  }
  p->scs_eval_cut = std::min(p->scs_cut, r_hi);

  int rng[3];
  image_box(p->lat, g.n_periodic, g.vacuum, p->scs_cut, rng);
  collect_shifts(p->lat, rng, p->scs_eval_cut + diam, true, &p->scs_shifts);

  // Cell differences and their placements (supercell_*_block, UTILS.f90:883-994;
  // cell index = k*SL_j*SL_i + j*SL_i + i, UTILS.f90:915,921).
  p->diff_shift.clear();
  p->diff_is_zero.clear();
  p->place_offset.assign(1, 0);
  p->place_rc.clear();
  p->place_cc.clear();
  double max_cell_shift = 0.0;
  const int* sl = p->sl;
  for (int di = -(sl[0] - 1); di <= sl[0] - 1; ++di)
    for (int dj = -(sl[1] - 1); dj <= sl[1] - 1; ++dj)
      for (int dk = -(sl[2] - 1); dk <= sl[2] - 1; ++dk) {
        double t[3];
        for (int c = 0; c < 3; ++c) t[c] = di * p->lat[c] + dj * p->lat[3 + c] + dk * p->lat[6 + c];
        p->diff_shift.insert(p->diff_shift.end(), {t[0], t[1], t[2]});
        p->diff_is_zero.push_back(di == 0 && dj == 0 && dk == 0);
        max_cell_shift = std::max(max_cell_shift, norm3(t));
        for (int rk = 0; rk < sl[2]; ++rk)
          for (int rj = 0; rj < sl[1]; ++rj)
            for (int ri = 0; ri < sl[0]; ++ri) {
              int ci = ri - di, cj = rj - dj, ck = rk - dk;
              if (ci < 0 || cj < 0 || ck < 0 || ci >= sl[0] || cj >= sl[1] || ck >= sl[2]) continue;
              p->place_rc.push_back(rk * sl[1] * sl[0] + rj * sl[0] + ri);
              p->place_cc.push_back(ck * sl[1] * sl[0] + cj * sl[0] + ci);
            }
        p->place_offset.push_back((int)p->place_rc.size());
      }

  image_box(lat_sl, g.n_periodic, g.vacuum, p->cfdm_cut, rng);
  collect_shifts(lat_sl, rng, p->cfdm_cut + diam + max_cell_shift, true, &p->cfdm_shifts);
  return MBD_OK;
}

}  // namespace mbd
