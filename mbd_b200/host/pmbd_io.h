// Input files and the text report of pmbd.x, for the C++ host of the C ABI
// (pmbd_b200.cpp).  Header-only, no CUDA: the parsers and the report
// formatter are plain C++ so that they can be checked without a GPU.
//
//   parse_geometry  geometry.in as MBD_rsSCS.f90:66-89 reads it: the atom
//                   count, a skipped line, `name x y z hirshfeld` per atom
//                   (Angstrom; a Fortran 'd' exponent is accepted), then
//                   optional `lattice_vector ax ay az` records that make
//                   the system periodic.
//   parse_settings  setting.in as MBD_rsSCS.f90:98-135: on each line the
//                   first keyword that occurs in it (xc,
//                   mbd_supercell_cutoff, mbd_cfdm_dip_cutoff,
//                   mbd_scs_dip_cutoff, mbd_scs_vacuum_axis, nprow, npcol)
//                   takes the value(s) after the line's first token; nprow
//                   and npcol are accepted and ignored (no process grid).
//   format_report   the MBD section of the report (MBD_at_rsSCS,
//                   UTILS.f90:223-331, and get_mbd_rSCS, UTILS.f90:753-755,
//                   861), every line as output_string (UTILS.f90:1708-1714)
//                   prints it -- list-directed, so with a leading blank --
//                   with the reference's edit descriptors.
//   read_network_file  the learned warm start's network checkpoint: 8-byte
//                   magic "MBDNET\0\0", uint32 format version (1), uint32
//                   parameter count, the FP32 parameters (little-endian) and
//                   the SHA-256 of the parameter bytes, all checked.
#pragma once

#include <array>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

namespace pmbd {

struct InputError : std::runtime_error {
  explicit InputError(const std::string& m) : std::runtime_error(m) {}
};

struct Geometry {
  std::vector<std::string> names;   // CHARACTER*2 atom names
  std::vector<double> coords;       // [3 N], Angstrom, atom-major
  std::vector<double> hirshfeld;    // [N]
  double lattice[9] = {0};          // lattice[3 k + c]: vector k, Angstrom
  int n_periodic = 0;
};

struct Settings {
  int xc = 1;
  double mbd_supercell_cutoff = 25.0;   // UTILS.f90:81
  double mbd_cfdm_dip_cutoff = 100.0;   // UTILS.f90:82
  double mbd_scs_dip_cutoff = 120.0;    // UTILS.f90:83
  bool mbd_scs_vacuum_axis[3] = {false, false, false};
  int nprow = 1, npcol = 1;
};

// The numbers a report prints (C6_eff and alpha_eff per atom, the 3
// eigenvalues of the molecular polarizability per frequency: eig[f + 21 k]).
struct Report {
  double energy_Ha = 0.0, c6_mol = 0.0;
  int nimag = 0;
  int supercell[3] = {1, 1, 1};
  std::vector<double> c6_eff, alpha_eff, molpol_eig, omega;
};

inline std::vector<std::string> split_lines(const std::string& text) {
  // str.splitlines() for \n, \r\n and \r endings
  std::vector<std::string> out;
  std::string cur;
  for (size_t i = 0; i < text.size(); ++i) {
    const char ch = text[i];
    if (ch == '\n' || ch == '\r') {
      out.push_back(cur);
      cur.clear();
      if (ch == '\r' && i + 1 < text.size() && text[i + 1] == '\n') ++i;
    } else {
      cur += ch;
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

inline std::vector<std::string> tokens(const std::string& line) {
  // commas count as blanks (list-directed input)
  std::vector<std::string> out;
  std::string cur;
  for (char ch : line) {
    if (ch == ' ' || ch == '\t' || ch == ',' || ch == '\v' || ch == '\f') {
      if (!cur.empty()) out.push_back(cur);
      cur.clear();
    } else {
      cur += ch;
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

inline double to_real(std::string t) {
  for (char& ch : t)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* end = nullptr;
  const double v = std::strtod(t.c_str(), &end);
  if (t.empty() || end != t.c_str() + t.size()) throw InputError("not a real number: '" + t + "'");
  return v;
}

inline int to_int(const std::string& t) {
  char* end = nullptr;
  const long v = std::strtol(t.c_str(), &end, 10);
  if (t.empty() || end != t.c_str() + t.size()) throw InputError("not an integer: '" + t + "'");
  return (int)v;
}

inline bool to_logical(const std::string& t) {
  size_t i = 0;
  while (i < t.size() && t[i] == '.') ++i;
  const char c = i < t.size() ? (char)std::tolower((unsigned char)t[i]) : '\0';
  if (c != 't' && c != 'f') throw InputError("not a Fortran logical: '" + t + "'");
  return c == 't';
}

inline Geometry parse_geometry(const std::string& text) {
  const std::vector<std::string> lines = split_lines(text);
  Geometry g;
  int n = 0;
  try {
    n = to_int(tokens(lines.at(0)).at(0));
  } catch (const std::exception&) {
    throw InputError("geometry: first record must hold the atom count");
  }
  if (n < 1) throw InputError("geometry: atom count must be >= 1");
  size_t k = 2;
  for (int i = 0; i < n; ++i) {
    if (k >= lines.size())
      throw InputError("geometry: expected " + std::to_string(n) + " atoms, found " + std::to_string(i));
    const std::vector<std::string> tok = tokens(lines[k++]);
    if (tok.size() < 5)
      throw InputError("geometry: atom record " + std::to_string(i + 1) + " needs name x y z hirshfeld");
    g.names.push_back(tok[0].substr(0, 2));
    try {
      for (int c = 1; c <= 3; ++c) g.coords.push_back(to_real(tok[c]));
      g.hirshfeld.push_back(to_real(tok[4]));
    } catch (const InputError& e) {
      throw InputError("geometry: atom record " + std::to_string(i + 1) + ": " + e.what());
    }
  }
  if (k < lines.size() && lines[k].find("lattice_vector") != std::string::npos) {
    g.n_periodic = 3;
    for (int i = 0; i < 3; ++i) {
      if (k + i >= lines.size()) throw InputError("geometry: three lattice_vector records required");
      const std::vector<std::string> tok = tokens(lines[k + i]);
      if (tok.size() < 4) throw InputError("geometry: lattice_vector needs three components");
      try {
        for (int c = 0; c < 3; ++c) g.lattice[3 * i + c] = to_real(tok[1 + c]);
      } catch (const InputError& e) {
        throw InputError(std::string("geometry: lattice_vector: ") + e.what());
      }
    }
  }
  return g;
}

inline Settings parse_settings(const std::string& text) {
  Settings s;
  for (const std::string& line : split_lines(text)) {
    const std::vector<std::string> tok = tokens(line);
    auto has = [&](const char* key) { return line.find(key) != std::string::npos; };
    try {
      if (has("xc")) {
        s.xc = to_int(tok.at(1));
      } else if (has("mbd_supercell_cutoff")) {
        s.mbd_supercell_cutoff = to_real(tok.at(1));
      } else if (has("mbd_cfdm_dip_cutoff")) {
        s.mbd_cfdm_dip_cutoff = to_real(tok.at(1));
      } else if (has("mbd_scs_dip_cutoff")) {
        s.mbd_scs_dip_cutoff = to_real(tok.at(1));
      } else if (has("mbd_scs_vacuum_axis")) {
        for (int c = 0; c < 3; ++c) s.mbd_scs_vacuum_axis[c] = to_logical(tok.at(1 + c));
      } else if (has("nprow")) {
        s.nprow = to_int(tok.at(1));
      } else if (has("npcol")) {
        s.npcol = to_int(tok.at(1));
      }
    } catch (const std::exception&) {
      throw InputError("settings: cannot read '" + line + "'");
    }
  }
  return s;
}

// Fortran Fw.d (asterisks when the number does not fit)
inline std::string fortran_f(double v, int w, int d) {
  char buf[512];
  std::snprintf(buf, sizeof buf, "%*.*f", w, d, v);
  std::string t(buf);
  return (int)t.size() <= w ? t : std::string(w, '*');
}

// Fortran Ew.d: 0.ddd...E+ee (the E dropped for a three-digit exponent)
inline std::string fortran_e(double v, int w, int d) {
  std::string body;
  if (v == 0.0) {
    body = "0." + std::string(d, '0') + "E+00";
  } else if (!std::isfinite(v)) {
    body = std::isnan(v) ? "nan" : (v < 0 ? "-inf" : "inf");
  } else {
    char m[512];
    std::snprintf(m, sizeof m, "%.*E", d - 1, std::fabs(v));   // d.ddddE+xx
    const std::string ms(m);
    const size_t epos = ms.find('E');
    std::string digits = ms.substr(0, epos);
    const size_t dot = digits.find('.');   // none when d == 1
    if (dot != std::string::npos) digits.erase(dot, 1);
    const int ex = std::atoi(ms.c_str() + epos + 1) + 1;
    char eb[16];
    if (std::abs(ex) <= 99) std::snprintf(eb, sizeof eb, "E%+03d", ex);
    else std::snprintf(eb, sizeof eb, "%+04d", ex);
    body = std::string(v < 0 ? "-" : "") + "0." + digits + eb;
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

inline std::string rstrip(std::string s) {
  while (!s.empty() && (s.back() == ' ' || s.back() == '\t')) s.pop_back();
  return s;
}

inline std::string format_report(const Geometry& g, const Report& r) {
  const std::string rule = "| ---------------------------------------------------------------------------";
  std::string out;
  auto put = [&](const std::string& text) {
    if (!out.empty()) out += '\n';
    out += " " + rstrip(text);
  };
  char buf[256];
  put("  | Many-Body Dispersion (MBD@rsSCS) energy ");
  put("  | System dynamic molecular polarizability alpha(iw) (bohr^3)");
  put("  " + rule);
  put("  |  omega(Ha)   alpha_iso      alpha_xx       alpha_yy       alpha_zz");
  for (int f = 0; f < 21; ++f) {
    const double e0 = r.molpol_eig[f], e1 = r.molpol_eig[f + 21], e2 = r.molpol_eig[f + 42];
    put("  | " + fortran_f(r.omega[f], 10, 6) + fortran_e((e0 + e1 + e2) / 3.0, 15, 6) + fortran_e(e0, 15, 6) +
        fortran_e(e1, 15, 6) + fortran_e(e2, 15, 6));
  }
  put("  " + rule);
  put("  | System C6 coefficient    :  " + fortran_f(r.c6_mol, 20, 8) + "    hartree bohr^6");
  put("  " + rule);
  put("  | Partitioned C6 (hartree bohr^6) | alpha (bohr^3)  of atom in system");
  put("  " + rule);
  for (size_t i = 0; i < g.names.size(); ++i) {
    std::snprintf(buf, sizeof buf, "%4d  %-2.2s", (int)i + 1, g.names[i].c_str());
    put("  | ATOM " + std::string(buf) + fortran_f(r.c6_eff[i], 12, 6) + std::string(6, ' ') +
        fortran_f(r.alpha_eff[i], 12, 6));
  }
  put("  " + rule);
  std::snprintf(buf, sizeof buf, "%3d X %3d X %3d", r.supercell[0], r.supercell[1], r.supercell[2]);
  put("  | Creating super cell of dimension" + std::string(buf) + " in MBD calculation");
  std::snprintf(buf, sizeof buf, "%6d", (int)g.names.size() * r.supercell[0] * r.supercell[1] * r.supercell[2]);
  put("  | containing" + std::string(buf) + "  atom");
  if (r.nimag > 0) {
    std::snprintf(buf, sizeof buf, "%4d", r.nimag);
    put("***WARNING: found " + std::string(buf) + " negative eigenvalues in MBD energy calculation.");
  }
  // 27.211 is a REAL*4 literal (UTILS.f90:330)
  put("  | MBD@rsSCS energy   :" + fortran_f(r.energy_Ha, 20, 9) + " Ha     " +
      fortran_f(r.energy_Ha * (double)27.211f, 20, 9) + " eV");
  return out;
}

// SHA-256 as FIPS 180-4 specifies it.  The initial hash value and the round
// constants are, by that definition, the first 32 bits of the fractional
// parts of the square roots of the first 8 primes and of the cube roots of
// the first 64 primes; they are computed here from that definition in
// extended precision (64-bit mantissa: 35 significant bits are needed).
class Sha256 {
 public:
  static std::array<uint8_t, 32> digest(const uint8_t* data, size_t n) {
    const Tables& t = tables();
    uint32_t h[8];
    std::memcpy(h, t.h0, sizeof h);
    const uint64_t bits = (uint64_t)n * 8u;
    size_t full = n / 64;
    for (size_t b = 0; b < full; ++b) block(h, data + 64 * b, t.k);
    uint8_t tail[128] = {0};
    const size_t rest = n - 64 * full;
    if (rest) std::memcpy(tail, data + 64 * full, rest);
    tail[rest] = 0x80;
    const size_t tlen = rest + 1 + 8 <= 64 ? 64 : 128;
    for (int i = 0; i < 8; ++i) tail[tlen - 1 - i] = (uint8_t)(bits >> (8 * i));
    for (size_t b = 0; b < tlen; b += 64) block(h, tail + b, t.k);
    std::array<uint8_t, 32> out{};
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(h[i] >> (24 - 8 * j));
    return out;
  }

 private:
  struct Tables {
    uint32_t h0[8], k[64];
  };
  static uint32_t frac32(long double x) {
    return (uint32_t)std::floor((x - std::floor(x)) * 4294967296.0L);
  }
  static const Tables& tables() {
    static const Tables t = [] {
      Tables r{};
      int found = 0;
      for (int p = 2; found < 64; ++p) {
        bool prime = true;
        for (int d = 2; d * d <= p; ++d)
          if (p % d == 0) { prime = false; break; }
        if (!prime) continue;
        if (found < 8) r.h0[found] = frac32(std::sqrt((long double)p));
        r.k[found++] = frac32(std::cbrt((long double)p));
      }
      return r;
    }();
    return t;
  }
  static uint32_t rotr(uint32_t x, int s) { return (x >> s) | (x << (32 - s)); }
  static void block(uint32_t h[8], const uint8_t* m, const uint32_t k[64]) {
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
      w[i] = (uint32_t)m[4 * i] << 24 | (uint32_t)m[4 * i + 1] << 16 | (uint32_t)m[4 * i + 2] << 8 | m[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
      const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
      const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
      w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
      const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
      const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
  }
};

inline std::vector<float> read_network_file(const std::string& path) {
  std::ifstream fh(path, std::ios::binary);
  if (!fh) throw InputError(path + ": cannot open");
  const std::vector<uint8_t> data((std::istreambuf_iterator<char>(fh)), std::istreambuf_iterator<char>());
  static const uint8_t magic[8] = {'M', 'B', 'D', 'N', 'E', 'T', 0, 0};
  if (data.size() < 16 || std::memcmp(data.data(), magic, 8) != 0)
    throw InputError(path + ": not a network checkpoint");
  auto u32 = [&](size_t o) {
    return (uint32_t)data[o] | (uint32_t)data[o + 1] << 8 | (uint32_t)data[o + 2] << 16 | (uint32_t)data[o + 3] << 24;
  };
  const uint32_t version = u32(8), count = u32(12);
  if (version != 1)
    throw InputError(path + ": checkpoint format version " + std::to_string(version) + ", expected 1");
  const uint64_t body = 4ull * count;
  if (data.size() != 16 + body + 32 ||
      Sha256::digest(data.data() + 16, (size_t)body) !=
          [&] { std::array<uint8_t, 32> d{}; std::memcpy(d.data(), data.data() + 16 + body, 32); return d; }())
    throw InputError(path + ": checkpoint is truncated or corrupted (SHA-256 mismatch)");
  std::vector<float> p(count);
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t bitsv = u32(16 + 4 * (size_t)i);
    std::memcpy(&p[i], &bitsv, 4);
  }
  return p;
}

}  // namespace pmbd
