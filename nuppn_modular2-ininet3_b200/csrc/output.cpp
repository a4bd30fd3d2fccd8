// output.cpp -- ppn's per-cycle output files, byte for byte (host only).
//
// printonecycle (frames/ppn/source/ppn.F90:431-539) writes, every print_cycles models,
//   iso_massf<mmmmm>.DAT  the abundances of the considered species (:519-536), and
//   flux_<mmmmm>.DAT      with iplot_flux_option = 1, the flux, energy and time scale of every
//                         network reaction (:496-510).
// Downstream NuGrid tools read these fixed-column files, so the writers below emit the same Fortran
// edit descriptors the reference uses:
//   iso_massf header  '(A1,1x,A3,2x,2(3X,A1,1x),A4,2x,A12,2x ,A5)'
//             model   '(1x,A,1x,I8,1x,A,1x,ES9.2,1x,A,1x,ES11.4)'
//             t9, rho '(2(1x,A,2x,ES10.3))'
//             dens*   '(1x,A,1x,ES12.5)'
//             species '(I5,2x,2(1X,F4.0),2x,I2,2x,ES12.5,2x,A5)'
//   flux      header  '(3x,a,2x,4(a,2x),6x,4(a,2x),2x,a,2(4x,a))'
//             reaction '(i5,4(2x,i3),8x,4(2x,i3),3(8x,ES12.5))'
// ESw.d is d.ddddE+ee right-justified in w characters; a three-digit exponent drops the E
// (d.dddd-100), as Fortran prints it. Values are clamped as the reference clamps them: abundances and
// fluxes to at least 1e-99, time scales to at least 1e99.
#include <cmath>
#include <cstdio>
#include <string>

#include "net_host.h"

namespace nuppn {

namespace {

std::string rjust(const std::string &s, int w) {
  return (int)s.size() >= w ? s : std::string(w - s.size(), ' ') + s;
}

// Fortran ESw.d
std::string fes(double x, int w, int d) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.*E", d, x);
  std::string s(buf);
  const size_t e = s.find('E');
  if (e != std::string::npos && s.size() - e - 2 >= 3) s.erase(e, 1);
  if ((int)s.size() > w) return std::string(w, '*');
  return rjust(s, w);
}

// Fortran Fw.0 of a whole number: ddd.
std::string ff0(double x, int w) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.0f.", x);
  std::string s(buf);
  if ((int)s.size() > w) return std::string(w, '*');
  return rjust(s, w);
}

std::string fi(long long v, int w) {
  std::string s = std::to_string(v);
  if ((int)s.size() > w) return std::string(w, '*');
  return rjust(s, w);
}

std::string name5(const char *p) {
  std::string s(p, 5);
  for (char &c : s)
    if (c == '\0') c = ' ';
  return s;
}

}  // namespace

bool write_iso_massf(const char *path, int model, double dzeit, double agej, double t9, double rho, double densn,
                     double densp, double densa, double total_energy_flux, int nsp, const double *z, const double *a,
                     const int *isomeric_state, const double *x, const char *names, const uint8_t *consider) {
  FILE *f = std::fopen(path, "w");
  if (!f) return false;
  std::fprintf(f, "H NUM     Z    A ISOM  ABUNDANCE_MF  ISOTP\n");
  std::fprintf(f, " # mod %s dzeit %s agej %s\n", fi(model, 8).c_str(), fes(dzeit, 9, 2).c_str(),
               fes(agej, 11, 4).c_str());
  std::fprintf(f, " # t9 =   %s rho =   %s\n", fes(t9, 10, 3).c_str(), fes(rho, 10, 3).c_str());
  std::fprintf(f, " # densn %s\n", fes(densn, 12, 5).c_str());
  std::fprintf(f, " # densp %s\n", fes(densp, 12, 5).c_str());
  std::fprintf(f, " # densa %s\n", fes(densa, 12, 5).c_str());
  std::fprintf(f, " # total_energy_flux_[erg/(g*s)] %s\n", fes(total_energy_flux, 12, 5).c_str());
  for (int i = 0; i < nsp; ++i) {
    if (consider && !consider[i]) continue;
    std::fprintf(f, "%s   %s %s  %s  %s  %s\n", fi(i + 1, 5).c_str(), ff0(z[i], 4).c_str(), ff0(a[i], 4).c_str(),
                 fi(isomeric_state ? isomeric_state[i] : 1, 2).c_str(), fes(std::fmax(x[i], 1.0e-99), 12, 5).c_str(),
                 name5(names + 5 * (size_t)i).c_str());
  }
  return std::fclose(f) == 0;
}

bool write_flux(const char *path, int nreac, const int *k, const double *z, const double *a, const double *flux,
                const double *energy, const double *timescale) {
  FILE *f = std::fopen(path, "w");
  if (!f) return false;
  std::fprintf(f, "   #  Z_k1  A_k1  Z_k3  A_k3        Z_k5  A_k5  Z_k7  A_k7    flux [dY/dt]    "
                  "energy [erg/(g*s)]    timescale reac [s]\n");
  for (int i = 0; i < nreac; ++i) {
    const int *kk = k + (size_t)i * 8;
    std::string line = fi(i + 1, 5);
    for (int s : {0, 2}) line += "  " + fi((long long)z[kk[s]], 3) + "  " + fi((long long)a[kk[s]], 3);
    line += "        ";
    for (int s : {4, 6}) line += "  " + fi((long long)z[kk[s]], 3) + "  " + fi((long long)a[kk[s]], 3);
    line += "        " + fes(std::fmax(1.0e-99, flux[i]), 12, 5);
    line += "        " + fes(std::fmax(1.0e-99, energy[i]), 12, 5);
    line += "        " + fes(std::fmax(1.0e99, timescale[i]), 12, 5);
    std::fprintf(f, "%s\n", line.c_str());
  }
  return std::fclose(f) == 0;
}

}  // namespace nuppn
