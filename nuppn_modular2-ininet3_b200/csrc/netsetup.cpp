// netsetup.cpp -- networksetup.txt reader and writer (host only).
//
// The reference writes its network to networksetup.txt (write_networksetup / output_network,
// physics/source/networksetup.F90:55-115) and can start from such a file instead of building the
// network (read_networksetup, :140-260). The file is fixed-column text in the Fortran edit
// descriptors of that module; this file writes the same columns and reads them back with the same
// column positions the reference's read formats use:
//   counts       '(7x,I5,16x,I5)'
//   species      (7X,I5,3X,A5,1X,L5,2X,0PF4.0,3X,F4.0,3x,I1)
//   reactions    (2X,I5,1X,L1,1X,I2,2X,A5,'  + ',I2,2X,A5,2X,'->',1X,I2,2X,A5,'  + ',I2,2X,A5,3X,
//                 ES9.3,2x,A5,2x,A5,2x,I2,2x,ES10.3,2x,ES10.3)
// A reaction line lists k2 zis(k1) + k4 zis(k3) -> k8 zis(k7) + k6 zis(k5).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "nuppn_internal.h"

namespace nuppn {

namespace {

// Fortran Ew.3 output of x in a field of w characters: [-]0.dddE+ee
std::string fortran_e3(double x, int w) {
  char buf[64];
  if (x == 0.0 || !std::isfinite(x)) {
    std::snprintf(buf, sizeof buf, "%s", x == 0.0 ? "0.000E+00" : "NaN");
  } else {
    char t[32];
    std::snprintf(t, sizeof t, "%.2e", std::fabs(x));  // a.bce+XX: the three significant digits
    const int ex = std::atoi(t + 5) + 1;                // 0.abc E(XX+1)
    std::snprintf(buf, sizeof buf, "%s0.%c%c%cE%c%02d", x < 0 ? "-" : "", t[0], t[2], t[3], ex < 0 ? '-' : '+',
                  ex < 0 ? -ex : ex);
  }
  std::string s(buf);
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

// Fortran ESw.3 output: [-]d.dddE+ee right-justified in w characters ([-]d.ddd+eee for a
// three-digit exponent, which drops the E as Fortran does)
std::string fortran_es3(double x, int w) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.3E", x);
  std::string s(buf);
  const size_t e = s.find('E');
  if (e != std::string::npos && s.size() - e - 2 >= 3) s.erase(e, 1);
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

std::string name5(const char *p) {
  std::string s(p, 5);
  for (char &c : s)
    if (c == '\0') c = ' ';
  return s;
}

std::string field(const std::string &line, int col, int width) {  // 1-based column
  if ((int)line.size() < col) return std::string();
  return line.substr(col - 1, width);
}

bool parse_int(const std::string &f, int &v) {
  const char *s = f.c_str();
  while (*s == ' ') ++s;
  if (!*s) { v = 0; return true; }  // a blank integer field reads as 0 (BLANK='NULL')
  char *end = nullptr;
  const long x = std::strtol(s, &end, 10);
  while (end && *end == ' ') ++end;
  if (!end || *end) return false;
  v = (int)x;
  return true;
}

bool parse_real(const std::string &f, double &v) {
  std::string t = f;
  // a Fortran exponent without its letter (0.123-100): put the E back before the exponent's sign
  const size_t sg = t.find_last_of("+-");
  if (sg != std::string::npos && sg > 0 && t.find_first_of("eEdD") == std::string::npos && std::isdigit((unsigned char)t[sg - 1]))
    t.insert(sg, "E");
  for (char &c : t)
    if (c == 'D' || c == 'd') c = 'E';
  const char *s = t.c_str();
  while (*s == ' ') ++s;
  if (!*s) { v = 0.0; return true; }
  char *end = nullptr;
  v = std::strtod(s, &end);
  while (end && *end == ' ') ++end;
  return end && !*end;
}

bool parse_logical(const std::string &f, bool &v) {
  for (char c : f) {
    if (c == ' ' || c == '.') continue;
    if (c == 'T' || c == 't') { v = true; return true; }
    if (c == 'F' || c == 'f') { v = false; return true; }
    return false;
  }
  return false;
}

}  // namespace

std::string write_networksetup(const char *path, const nuppn_netsetup &ns) {
  if (!path || ns.nsp < 0 || ns.nre < 0 || !ns.zis || !ns.considerisotope || !ns.anetw || !ns.znetw ||
      (ns.nre > 0 && (!ns.considerreaction || !ns.k)))
    return "networksetup: missing arrays";
  FILE *f = std::fopen(path, "w");
  if (!f) return std::string("networksetup: cannot write ") + path;
  const std::string stars(72, '*');
  std::fprintf(f, "%s\n", stars.c_str());
  std::fprintf(f, "        TABLE OF ISOTOPES %s %s\n", fortran_e3(ns.t9, 10).c_str(), fortran_e3(ns.rho, 10).c_str());
  std::fprintf(f, "\n");
  std::fprintf(f, "        NO. SYMBOL T/F MASSNR PROTON\n");
  std::fprintf(f, "       %5d =  NGIS        %5d =  ISOMERS\n", ns.nsp, ns.nisomers);
  for (int i = 0; i < ns.nsp; ++i)
    std::fprintf(f, "       %5d   %s %5s  %3d.   %3d.   %1d\n", i + 1, name5(ns.zis + 5 * i).c_str(),
                 ns.considerisotope[i] ? "T" : "F", (int)std::lround(ns.anetw[i]), (int)std::lround(ns.znetw[i]),
                 ns.isomeric_state ? ns.isomeric_state[i] : 1);
  std::fprintf(f, "%s\n\n", stars.c_str());
  std::fprintf(f, "%10s%s%35s%s\n\n", "", "REACTION NETWORK", "", "V(i) Nasv(*rho)");
  std::fprintf(f, "       %5d =  NGIR        %5d = + REAZ ISOMERS\n", ns.nre, ns.nreac_isomers);
  auto nm = [&](int s) { return (s >= 0 && s < ns.nsp) ? name5(ns.zis + 5 * s) : std::string("OOOOO"); };
  for (int l = 0; l < ns.nre; ++l) {
    const int32_t *k = ns.k + 8 * (size_t)l;
    std::fprintf(f, "  %5d %s %2d  %s  + %2d  %s  -> %2d  %s  + %2d  %s   %s  %s  %s  %2d  %s  %s\n", l + 1,
                 ns.considerreaction[l] ? "T" : "F", k[1], nm(k[0]).c_str(), k[3], nm(k[2]).c_str(), k[7],
                 nm(k[6]).c_str(), k[5], nm(k[4]).c_str(), fortran_es3(ns.v ? ns.v[l] : 0.0, 9).c_str(),
                 ns.lab ? name5(ns.lab + 5 * l).c_str() : "     ", ns.labb ? name5(ns.labb + 5 * l).c_str() : "     ",
                 ns.ilabb ? ns.ilabb[l] : 0, fortran_es3(ns.rfac ? ns.rfac[l] : 1.0, 10).c_str(),
                 fortran_es3(ns.bind_energy_diff ? ns.bind_energy_diff[l] : 0.0, 10).c_str());
  }
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? "" : "networksetup: write error";
}

std::string read_networksetup(const char *path, nuppn_netsetup &ns) {
  if (!path) return "networksetup: null path";
  FILE *f = std::fopen(path, "r");
  if (!f) return std::string("networksetup: cannot open ") + path;
  std::vector<std::string> lines;
  char buf[1024];
  while (std::fgets(buf, sizeof buf, f)) {
    std::string s(buf);
    while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) s.pop_back();
    lines.push_back(s);
  }
  std::fclose(f);
  auto bad = [&](size_t i) { return "networksetup: cannot parse line " + std::to_string(i + 1); };
  if (lines.size() < 5) return "networksetup: file too short";
  // header: '(a25,2(e11.3))'
  double t9 = 0, rho = 0;
  if (!parse_real(field(lines[1], 26, 11), t9) || !parse_real(field(lines[1], 37, 11), rho)) return bad(1);
  int nsp = 0, niso = 0;
  if (!parse_int(field(lines[4], 8, 5), nsp) || !parse_int(field(lines[4], 29, 5), niso) || nsp < 0) return bad(4);
  const size_t r0 = 5 + (size_t)nsp + 4;  // species lines, then 4 lines the reader skips
  if (lines.size() < r0 + 1) return "networksetup: file too short";
  int nre = 0, nreiso = 0;
  if (!parse_int(field(lines[r0], 8, 5), nre) || !parse_int(field(lines[r0], 29, 5), nreiso) || nre < 0) return bad(r0);
  if (lines.size() < r0 + 1 + (size_t)nre) return "networksetup: fewer reaction lines than NGIR";
  const bool sizing = !ns.zis && !ns.considerisotope && !ns.anetw && !ns.znetw && !ns.considerreaction && !ns.k;
  if (sizing) {
    ns.nsp = nsp; ns.nre = nre; ns.nisomers = niso; ns.nreac_isomers = nreiso; ns.t9 = t9; ns.rho = rho;
    return "";
  }
  if (ns.nsp != nsp || ns.nre != nre) return "networksetup: array sizes differ from the file's NGIS / NGIR";
  if (!ns.zis || !ns.considerisotope || !ns.anetw || !ns.znetw || (nre > 0 && (!ns.considerreaction || !ns.k)))
    return "networksetup: missing arrays";
  ns.nisomers = niso; ns.nreac_isomers = nreiso; ns.t9 = t9; ns.rho = rho;
  std::unordered_map<std::string, int> ispe;
  for (int i = 0; i < nsp; ++i) {  // (7X,I5,3X,A5,1X,L5,2X,0PF4.0,3X,F4.0,3x,I1)
    const std::string &L = lines[5 + i];
    const std::string name = field(L, 16, 5);
    bool t = false;
    double a = 0, z = 0;
    int iso = 0;
    if (name.size() < 5 || !parse_logical(field(L, 22, 5), t) || !parse_real(field(L, 29, 4), a) ||
        !parse_real(field(L, 36, 4), z) || !parse_int(field(L, 43, 1), iso))
      return bad(5 + i);
    std::memcpy(ns.zis + 5 * (size_t)i, name.data(), 5);
    ns.considerisotope[i] = t ? 1 : 0;
    ns.anetw[i] = a;
    ns.znetw[i] = z;
    if (ns.isomeric_state) ns.isomeric_state[i] = iso;
    ispe.emplace(name, i);  // the first species of a name, as ispe's hash lookup
  }
  auto idx = [&](const std::string &n) {
    auto it = ispe.find(n);
    return it == ispe.end() ? -1 : it->second;
  };
  for (int l = 0; l < nre; ++l) {  // fmtreactionread
    const std::string &L = lines[r0 + 1 + l];
    bool cr = false;
    int k2, k4, k8, k6, il = 0;
    double v = 0, rf = 0, be = 0;
    if (!parse_logical(field(L, 9, 1), cr) || !parse_int(field(L, 11, 2), k2) || !parse_int(field(L, 24, 2), k4) ||
        !parse_int(field(L, 38, 2), k8) || !parse_int(field(L, 51, 2), k6) || !parse_real(field(L, 63, 9), v) ||
        !parse_int(field(L, 88, 2), il) || !parse_real(field(L, 92, 10), rf) || !parse_real(field(L, 104, 10), be))
      return bad(r0 + 1 + l);
    int32_t *k = ns.k + 8 * (size_t)l;
    k[0] = idx(field(L, 15, 5)); k[1] = k2;
    k[2] = idx(field(L, 28, 5)); k[3] = k4;
    k[6] = idx(field(L, 42, 5)); k[7] = k8;
    k[4] = idx(field(L, 55, 5)); k[5] = k6;
    ns.considerreaction[l] = cr ? 1 : 0;
    if (ns.v) ns.v[l] = v;
    if (ns.lab) { const std::string s = field(L, 74, 5); std::memcpy(ns.lab + 5 * (size_t)l, (s + "     ").data(), 5); }
    if (ns.labb) { const std::string s = field(L, 81, 5); std::memcpy(ns.labb + 5 * (size_t)l, (s + "     ").data(), 5); }
    if (ns.ilabb) ns.ilabb[l] = il;
    if (ns.rfac) ns.rfac[l] = rf;
    if (ns.bind_energy_diff) ns.bind_energy_diff[l] = be;
  }
  // species switched off in the file switch off every reaction they take part in (networksetup.F90:226-240)
  const int gamma = idx("OOOOO");
  for (int i = 0; i < nsp; ++i) {
    if (ns.considerisotope[i] || i == gamma) continue;
    for (int l = 0; l < nre; ++l) {
      const int32_t *k = ns.k + 8 * (size_t)l;
      if (k[0] == i || k[2] == i || k[4] == i || k[6] == i) ns.considerreaction[l] = 0;
    }
  }
  return "";
}

}  // namespace nuppn
