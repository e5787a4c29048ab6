// Test driver for mbd_b200/host/pmbd_io.h (no GPU, no library): each
// subcommand runs one part of the header on files the test writes and prints
// the result for the test to compare.
//
//   host_io_check geometry FILE    parsed geometry, one value per line (%a)
//   host_io_check settings FILE    parsed settings
//   host_io_check report GEOM VALS format_report of GEOM fed the values in
//                                  VALS (hex floats: energy c6_mol nimag
//                                  sc1 sc2 sc3, c6_eff[N], alpha_eff[N],
//                                  molpol_eig[63] (eig[f + 21 k]), omega[21])
//   host_io_check edit FILE        lines "v w d" -> Fortran Ew.d and Fw.d of v
//   host_io_check sha256 FILE      hex digest of FILE
//   host_io_check network FILE     parameter count and the parameters (%a)
// Exit status 1 with the message on stderr when the header throws.
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "pmbd_io.h"

static std::string slurp(const char* path) {
  std::ifstream fh(path, std::ios::binary);
  if (!fh) throw pmbd::InputError(std::string(path) + ": cannot open");
  std::ostringstream ss;
  ss << fh.rdbuf();
  return ss.str();
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string cmd = argv[1];
  try {
    if (cmd == "geometry") {
      const pmbd::Geometry g = pmbd::parse_geometry(slurp(argv[2]));
      std::printf("%zu %d\n", g.names.size(), g.n_periodic);
      for (size_t i = 0; i < g.names.size(); ++i)
        std::printf("%s %a %a %a %a\n", g.names[i].c_str(), g.coords[3 * i], g.coords[3 * i + 1],
                    g.coords[3 * i + 2], g.hirshfeld[i]);
      for (double v : g.lattice) std::printf("%a\n", v);
    } else if (cmd == "settings") {
      const pmbd::Settings s = pmbd::parse_settings(slurp(argv[2]));
      std::printf("%d %a %a %a %d %d %d %d %d\n", s.xc, s.mbd_supercell_cutoff, s.mbd_cfdm_dip_cutoff,
                  s.mbd_scs_dip_cutoff, (int)s.mbd_scs_vacuum_axis[0], (int)s.mbd_scs_vacuum_axis[1],
                  (int)s.mbd_scs_vacuum_axis[2], s.nprow, s.npcol);
    } else if (cmd == "report") {
      if (argc < 4) return 2;
      const pmbd::Geometry g = pmbd::parse_geometry(slurp(argv[2]));
      std::istringstream in(slurp(argv[3]));
      auto next = [&] {
        std::string t;
        in >> t;
        return std::strtod(t.c_str(), nullptr);
      };
      pmbd::Report r;
      r.energy_Ha = next();
      r.c6_mol = next();
      r.nimag = (int)next();
      for (int& s : r.supercell) s = (int)next();
      const size_t n = g.names.size();
      for (size_t i = 0; i < n; ++i) r.c6_eff.push_back(next());
      for (size_t i = 0; i < n; ++i) r.alpha_eff.push_back(next());
      for (int i = 0; i < 63; ++i) r.molpol_eig.push_back(next());
      for (int i = 0; i < 21; ++i) r.omega.push_back(next());
      std::printf("%s\n", pmbd::format_report(g, r).c_str());
    } else if (cmd == "edit") {
      std::istringstream in(slurp(argv[2]));
      std::string v;
      int w, d;
      while (in >> v >> w >> d) {
        const double x = std::strtod(v.c_str(), nullptr);
        std::printf("%s|%s\n", pmbd::fortran_e(x, w, d).c_str(), pmbd::fortran_f(x, w, d).c_str());
      }
    } else if (cmd == "sha256") {
      const std::string data = slurp(argv[2]);
      for (uint8_t b : pmbd::Sha256::digest((const uint8_t*)data.data(), data.size())) std::printf("%02x", b);
      std::printf("\n");
    } else if (cmd == "network") {
      const std::vector<float> p = pmbd::read_network_file(argv[2]);
      std::printf("%zu\n", p.size());
      for (float v : p) std::printf("%a\n", (double)v);
    } else {
      return 2;
    }
  } catch (const pmbd::InputError& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
