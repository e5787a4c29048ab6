// pmbd_b200: the pmbd.x front end (MBD_rsSCS.f90:1-239) over the C ABI.
//
//   pmbd_b200 geometry.in [setting.in] [--mode plain|mixed|mixed_learned]
//             [--network FILE] [--device N]
//
// Reads the two input files pmbd.x takes (MBD_rsSCS.f90:59-60), converts the
// coordinates and lattice vectors from Angstrom to bohr as MBD_rsSCS.f90:211-212
// does, computes the MBD@rsSCS energy with one mbd_rsscs_energy call on the
// GPU and prints the MBD section of pmbd.x's report (UTILS.f90:223-331).
// --mode mixed_learned without --network starts block-CG from zero (the
// method without the network).  Exit status 0 on success; 1, with the
// engine's message on stderr, when the input cannot be read or the geometry
// fails (unknown element, relay matrix not positive definite, ...); 2 for a
// bad command line.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "mbd_b200.h"
#include "pmbd_io.h"

namespace {

constexpr double kBohr = 0.52917721;   // UTILS.f90:85

const char* kUsage =
    "usage: pmbd_b200 geometry.in [setting.in] [--mode plain|mixed|mixed_learned]\n"
    "                 [--network FILE] [--device N]\n";

std::string slurp(const std::string& path) {
  std::ifstream fh(path, std::ios::binary);
  if (!fh) throw pmbd::InputError(path + ": cannot open");
  std::ostringstream ss;
  ss << fh.rdbuf();
  return ss.str();
}

struct Args {
  std::string geometry, settings, network;
  int mode = MBD_MODE_PLAIN_FP64;
  int device = 0;
};

int usage_error(const std::string& msg) {
  std::fprintf(stderr, "%spmbd_b200: %s\n", kUsage, msg.c_str());
  return 2;
}

// Returns -1 when the arguments parse, else the exit status to return.
int parse_args(int argc, char** argv, Args& a) {
  std::vector<std::string> pos;
  for (int i = 1; i < argc; ++i) {
    const std::string t = argv[i];
    if (t == "-h" || t == "--help") {
      std::fputs(kUsage, stdout);
      return 0;
    }
    if (t != "--mode" && t != "--network" && t != "--device") {
      if (t.size() > 1 && t[0] == '-') return usage_error("unknown option '" + t + "'");
      pos.push_back(t);
      continue;
    }
    if (i + 1 >= argc) return usage_error(t + " needs a value");
    const std::string v = argv[++i];
    if (t == "--mode") {
      if (v == "plain") a.mode = MBD_MODE_PLAIN_FP64;
      else if (v == "mixed") a.mode = MBD_MODE_MIXED;
      else if (v == "mixed_learned") a.mode = MBD_MODE_MIXED_LEARNED;
      else return usage_error("unknown mode '" + v + "'");
    } else if (t == "--network") {
      a.network = v;
    } else {
      char* end = nullptr;
      a.device = (int)std::strtol(v.c_str(), &end, 10);
      if (v.empty() || *end) return usage_error("bad device '" + v + "'");
    }
  }
  if (pos.empty()) return usage_error("the geometry file is required");
  if (pos.size() > 2) return usage_error("at most two input files");
  a.geometry = pos[0];
  if (pos.size() == 2) a.settings = pos[1];
  return -1;
}

int fail(int code) {
  std::fprintf(stderr, "pmbd_b200: %s (status %d)\n", mbd_rsscs_strerror(code), code);
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  const int rc_args = parse_args(argc, argv, a);
  if (rc_args >= 0) return rc_args;
  try {
    const pmbd::Geometry g = pmbd::parse_geometry(slurp(a.geometry));
    const pmbd::Settings s = pmbd::parse_settings(a.settings.empty() ? std::string() : slurp(a.settings));
    std::vector<float> params;
    if (a.mode == MBD_MODE_MIXED_LEARNED && !a.network.empty()) {
      params = pmbd::read_network_file(a.network);
      const int want = mbd_rsscs_learned_param_count();
      if ((long long)params.size() != want)
        throw pmbd::InputError(a.network + ": " + std::to_string(params.size()) + " parameters, the engine's network has " +
                               std::to_string(want));
    }

    const int n = (int)g.names.size();
    std::vector<int> z(n);
    for (int i = 0; i < n; ++i) z[i] = mbd_rsscs_element_z(g.names[i].c_str());
    std::vector<double> coords(3 * (size_t)n), lattice(9);
    for (size_t i = 0; i < coords.size(); ++i) coords[i] = g.coords[i] / kBohr;
    for (int i = 0; i < 9; ++i) lattice[i] = g.lattice[i] / kBohr;

    mbd_geom geom{};
    geom.n_atoms = n;
    geom.z = z.data();
    geom.coords_bohr = coords.data();
    geom.hirshfeld = g.hirshfeld.data();
    geom.n_periodic = g.n_periodic;
    geom.lattice_bohr = lattice.data();
    geom.scs_cut_A = s.mbd_scs_dip_cutoff;
    geom.cfdm_cut_A = s.mbd_cfdm_dip_cutoff;
    geom.sc_cut_A = s.mbd_supercell_cutoff;
    for (int k = 0; k < 3; ++k) geom.vacuum[k] = s.mbd_scs_vacuum_axis[k] ? 1 : 0;
    geom.xc = s.xc;

    pmbd::Report rep;
    rep.c6_eff.assign(n, 0.0);
    rep.alpha_eff.assign(n, 0.0);
    rep.molpol_eig.assign(MBD_N_FREQ * 3, 0.0);
    rep.omega.assign(MBD_N_FREQ, 0.0);
    std::vector<double> alpha_iw((size_t)MBD_N_FREQ * n);
    mbd_result res{};
    res.alpha_eff = rep.alpha_eff.data();
    res.c6_eff = rep.c6_eff.data();
    res.alpha_iw = alpha_iw.data();
    res.molpol_eig = rep.molpol_eig.data();

    int rc = mbd_rsscs_frequency_grid(rep.omega.data(), nullptr, MBD_N_FREQ);
    if (rc != MBD_OK) return fail(rc);
    mbd_ctx* ctx = nullptr;
    rc = mbd_rsscs_create(&ctx, a.device);
    if (rc != MBD_OK) return fail(rc);
    if (a.mode == MBD_MODE_MIXED_LEARNED)
      rc = params.empty() ? mbd_rsscs_learned_use_network(ctx, 0)
                          : mbd_rsscs_learned_set_params(ctx, params.data(), (int)params.size());
    if (rc == MBD_OK) rc = mbd_rsscs_energy(ctx, &geom, a.mode, &res);
    mbd_rsscs_destroy(ctx);
    if (rc != MBD_OK) return fail(rc);

    rep.energy_Ha = res.energy_Ha;
    rep.c6_mol = res.c6_mol;
    rep.nimag = res.nimag;
    for (int k = 0; k < 3; ++k) rep.supercell[k] = res.supercell[k];
    std::printf("%s\n", pmbd::format_report(g, rep).c_str());
    return 0;
  } catch (const pmbd::InputError& e) {
    std::fprintf(stderr, "pmbd_b200: %s\n", e.what());
    return 1;
  }
}
