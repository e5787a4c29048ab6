// pmbd_b200: the pmbd.x front end (MBD_rsSCS.f90:1-239) over the C ABI.
//
//   pmbd_b200 geometry.in [setting.in] [--mode plain|mixed|mixed_learned]
//             [--network FILE] [--device N]
//   pmbd_b200 --batch LIST --out-dir DIR [--mode ...] [--network FILE] [--device N]
//
// Reads the two input files pmbd.x takes (MBD_rsSCS.f90:59-60), converts the
// coordinates and lattice vectors from Angstrom to bohr as MBD_rsSCS.f90:211-212
// does, computes the MBD@rsSCS energy with one mbd_rsscs_energy call on the
// GPU and prints the MBD section of pmbd.x's report (UTILS.f90:223-331).
// --batch: LIST names one geometry per line ("geometry.in [setting.in]",
// relative paths taken from LIST's directory, blank lines and lines starting
// with '#' skipped); all of them go to the GPU in one mbd_rsscs_energy_batch
// call (the reference runs one geometry per process), and each geometry's
// report is written to DIR/<geometry file name without extension>.out.
// --mode mixed_learned without --network starts block-CG from zero (the
// method without the network).  Exit status 0 on success; 1, with the
// engine's message on stderr, when an input cannot be read or a geometry
// fails (unknown element, relay matrix not positive definite, ...; in a
// batch the other geometries' reports are still written, while an input
// that cannot be read stops the batch before the GPU is used); 2 for a bad
// command line.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "mbd_b200.h"
#include "pmbd_io.h"

namespace {

constexpr double kBohr = 0.52917721;   // UTILS.f90:85

const char* kUsage =
    "usage: pmbd_b200 geometry.in [setting.in] [--mode plain|mixed|mixed_learned]\n"
    "                 [--network FILE] [--device N]\n"
    "       pmbd_b200 --batch LIST --out-dir DIR [--mode ...] [--network FILE] [--device N]\n";

std::string slurp(const std::string& path) {
  std::ifstream fh(path, std::ios::binary);
  if (!fh) throw pmbd::InputError(path + ": cannot open");
  std::ostringstream ss;
  ss << fh.rdbuf();
  return ss.str();
}

struct Args {
  std::string geometry, settings, network, batch, out_dir;
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
    if (t != "--mode" && t != "--network" && t != "--device" && t != "--batch" && t != "--out-dir") {
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
    } else if (t == "--batch") {
      a.batch = v;
    } else if (t == "--out-dir") {
      a.out_dir = v;
    } else {
      char* end = nullptr;
      a.device = (int)std::strtol(v.c_str(), &end, 10);
      if (v.empty() || *end) return usage_error("bad device '" + v + "'");
    }
  }
  if (!a.batch.empty()) {
    if (!pos.empty()) return usage_error("--batch takes its input files from LIST");
    if (a.out_dir.empty()) return usage_error("--batch needs --out-dir");
    return -1;
  }
  if (!a.out_dir.empty()) return usage_error("--out-dir goes with --batch");
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

// One geometry: its inputs as read, the C ABI structures pointing into its
// own arrays (so a Job must not move once prepared), and its report.
struct Job {
  std::string path;
  pmbd::Geometry g;
  pmbd::Settings s;
  std::vector<int> z;
  std::vector<double> coords, lattice, alpha_iw;
  pmbd::Report rep;
  mbd_geom geom{};
  mbd_result res{};
};

std::unique_ptr<Job> load_job(const std::string& geometry, const std::string& settings) {
  std::unique_ptr<Job> j(new Job());
  j->path = geometry;
  j->g = pmbd::parse_geometry(slurp(geometry));
  j->s = pmbd::parse_settings(settings.empty() ? std::string() : slurp(settings));
  const pmbd::Geometry& g = j->g;
  const pmbd::Settings& s = j->s;
  const int n = (int)g.names.size();
  j->z.resize(n);
  for (int i = 0; i < n; ++i) j->z[i] = mbd_rsscs_element_z(g.names[i].c_str());
  j->coords.resize(3 * (size_t)n);
  j->lattice.resize(9);
  for (size_t i = 0; i < j->coords.size(); ++i) j->coords[i] = g.coords[i] / kBohr;
  for (int i = 0; i < 9; ++i) j->lattice[i] = g.lattice[i] / kBohr;
  mbd_geom& geom = j->geom;
  geom.n_atoms = n;
  geom.z = j->z.data();
  geom.coords_bohr = j->coords.data();
  geom.hirshfeld = g.hirshfeld.data();
  geom.n_periodic = g.n_periodic;
  geom.lattice_bohr = j->lattice.data();
  geom.scs_cut_A = s.mbd_scs_dip_cutoff;
  geom.cfdm_cut_A = s.mbd_cfdm_dip_cutoff;
  geom.sc_cut_A = s.mbd_supercell_cutoff;
  for (int k = 0; k < 3; ++k) geom.vacuum[k] = s.mbd_scs_vacuum_axis[k] ? 1 : 0;
  geom.xc = s.xc;
  pmbd::Report& rep = j->rep;
  rep.c6_eff.assign(n, 0.0);
  rep.alpha_eff.assign(n, 0.0);
  rep.molpol_eig.assign(MBD_N_FREQ * 3, 0.0);
  j->alpha_iw.assign((size_t)MBD_N_FREQ * n, 0.0);
  j->res.alpha_eff = rep.alpha_eff.data();
  j->res.c6_eff = rep.c6_eff.data();
  j->res.alpha_iw = j->alpha_iw.data();
  j->res.molpol_eig = rep.molpol_eig.data();
  return j;
}

std::string report_of(Job& j, const std::vector<double>& omega) {
  j.rep.omega = omega;
  j.rep.energy_Ha = j.res.energy_Ha;
  j.rep.c6_mol = j.res.c6_mol;
  j.rep.nimag = j.res.nimag;
  for (int k = 0; k < 3; ++k) j.rep.supercell[k] = j.res.supercell[k];
  return pmbd::format_report(j.g, j.rep);
}

std::string dir_of(const std::string& path) {
  const size_t k = path.find_last_of('/');
  return k == std::string::npos ? std::string() : path.substr(0, k + 1);
}

std::string stem_of(const std::string& path) {
  std::string b = path.substr(path.find_last_of('/') == std::string::npos ? 0 : path.find_last_of('/') + 1);
  const size_t dot = b.find_last_of('.');
  return dot == std::string::npos || dot == 0 ? b : b.substr(0, dot);
}

// The (geometry, settings) pairs of a --batch list, paths resolved against
// the list's directory.
std::vector<std::pair<std::string, std::string>> read_list(const std::string& list) {
  const std::string base = dir_of(list);
  auto resolve = [&](const std::string& p) { return p.empty() || p[0] == '/' ? p : base + p; };
  std::vector<std::pair<std::string, std::string>> out;
  for (const std::string& line : pmbd::split_lines(slurp(list))) {
    const std::vector<std::string> tok = pmbd::tokens(line);
    if (tok.empty() || tok[0][0] == '#') continue;
    if (tok.size() > 2) throw pmbd::InputError(list + ": '" + line + "': expected geometry.in [setting.in]");
    out.emplace_back(resolve(tok[0]), tok.size() > 1 ? resolve(tok[1]) : std::string());
  }
  if (out.empty()) throw pmbd::InputError(list + ": no geometries listed");
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  const int rc_args = parse_args(argc, argv, a);
  if (rc_args >= 0) return rc_args;
  try {
    std::vector<std::unique_ptr<Job>> jobs;
    std::vector<std::string> outs;
    if (a.batch.empty()) {
      jobs.push_back(load_job(a.geometry, a.settings));
    } else {
      for (const auto& e : read_list(a.batch)) {
        jobs.push_back(load_job(e.first, e.second));
        const std::string out = a.out_dir + "/" + stem_of(e.first) + ".out";
        for (const std::string& o : outs)
          if (o == out) throw pmbd::InputError(a.batch + ": two geometries would both write " + out);
        outs.push_back(out);
      }
    }
    std::vector<float> params;
    if (a.mode == MBD_MODE_MIXED_LEARNED && !a.network.empty()) {
      params = pmbd::read_network_file(a.network);
      const int want = mbd_rsscs_learned_param_count();
      if ((long long)params.size() != want)
        throw pmbd::InputError(a.network + ": " + std::to_string(params.size()) + " parameters, the engine's network has " +
                               std::to_string(want));
    }
    std::vector<double> omega(MBD_N_FREQ, 0.0);
    int rc = mbd_rsscs_frequency_grid(omega.data(), nullptr, MBD_N_FREQ);
    if (rc != MBD_OK) return fail(rc);

    mbd_ctx* ctx = nullptr;
    rc = mbd_rsscs_create(&ctx, a.device);
    if (rc != MBD_OK) return fail(rc);
    if (a.mode == MBD_MODE_MIXED_LEARNED)
      rc = params.empty() ? mbd_rsscs_learned_use_network(ctx, 0)
                          : mbd_rsscs_learned_set_params(ctx, params.data(), (int)params.size());
    if (rc != MBD_OK) {
      mbd_rsscs_destroy(ctx);
      return fail(rc);
    }
    if (a.batch.empty()) {
      rc = mbd_rsscs_energy(ctx, &jobs[0]->geom, a.mode, &jobs[0]->res);
      mbd_rsscs_destroy(ctx);
      if (rc != MBD_OK) return fail(rc);
      std::printf("%s\n", report_of(*jobs[0], omega).c_str());
      return 0;
    }
    std::vector<mbd_geom> geoms;
    std::vector<mbd_result> results;
    for (const auto& j : jobs) {
      geoms.push_back(j->geom);
      results.push_back(j->res);
    }
    mbd_rsscs_energy_batch(ctx, (int)jobs.size(), geoms.data(), a.mode, results.data());
    mbd_rsscs_destroy(ctx);
    int status = 0;
    for (size_t k = 0; k < jobs.size(); ++k) {
      Job& j = *jobs[k];
      j.res = results[k];
      if (j.res.status != MBD_OK) {
        std::fprintf(stderr, "pmbd_b200: %s: %s (status %d)\n", j.path.c_str(), mbd_rsscs_strerror(j.res.status),
                     j.res.status);
        status = 1;
        continue;
      }
      std::ofstream fh(outs[k], std::ios::binary);
      fh << report_of(j, omega) << "\n";
      if (!fh) {
        std::fprintf(stderr, "pmbd_b200: %s: cannot write\n", outs[k].c_str());
        status = 1;
      }
    }
    return status;
  } catch (const pmbd::InputError& e) {
    std::fprintf(stderr, "pmbd_b200: %s\n", e.what());
    return 1;
  }
}
