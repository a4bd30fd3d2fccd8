// tppnp_io.cpp -- tppnp's binary trajectory input (host only).
//
// traj_data_bin_init / read_bin_trajectory (frames/tppnp/source/traj_data.F90:73-168) read an
// unformatted stream file (access = "stream", no record markers, the machine's byte order: the
// run template's tp.lsb is little-endian) laid out as
//   header      num_tracers, nsteps_min, nsteps_max                      3 x int32
//   per tracer  pnum, ntimesteps                                          2 x int32
//               mass                                                      float64
//               posini(3), posfin(3)                                      6 x float64
//               time(nt) [s], temp(nt) [K], dens(nt) [g/cm^3]             3 x nt float64
//               pnum, niso                                                2 x int32
//               xini_a(niso), xini_z(niso)                                2 x niso int32
//               xini_zis(niso)                                            niso x 5 characters
//               xini_x(niso)                                              niso float64
// read_trajectory then divides the temperatures by 1e9 (T9), which this reader does too.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "net_host.h"

namespace nuppn {

namespace {

struct File {
  FILE *f = nullptr;
  explicit File(const char *path) : f(std::fopen(path, "rb")) {}
  ~File() {
    if (f) std::fclose(f);
  }
  bool read(void *p, size_t bytes) { return bytes == 0 || std::fread(p, 1, bytes, f) == bytes; }
  bool skip(size_t bytes) { return std::fseek(f, (long)bytes, SEEK_CUR) == 0; }
};

}  // namespace

std::string tppnp_header(const char *path, int *num_tracers, int *nsteps_min, int *nsteps_max) {
  File F(path);
  if (!F.f) return std::string("cannot open ") + path;
  int32_t h[3];
  if (!F.read(h, sizeof h)) return "tppnp file: short header";
  if (h[0] < 0 || h[1] < 0 || h[2] < h[1]) return "tppnp file: bad header";
  *num_tracers = h[0];
  *nsteps_min = h[1];
  *nsteps_max = h[2];
  return std::string();
}

std::string tppnp_next(const char *path, int64_t *pos, int *pnum, int *nsteps, int *niso, double *mass,
                       double *posini, double *posfin, double *time, double *t9, double *rho, int *a, int *z,
                       char *zis, double *x) {
  File F(path);
  if (!F.f) return std::string("cannot open ") + path;
  const int64_t at = *pos > 0 ? *pos : 12;  // 0: the first tracer, after the 3-integer header
  if (std::fseek(F.f, (long)at, SEEK_SET) != 0) return "tppnp file: bad offset";
  int32_t pn[2];
  if (!F.read(pn, sizeof pn)) return "tppnp file: no tracer at this offset";
  const int nt = pn[1];
  if (nt < 0 || nt > (1 << 26)) return "tppnp file: bad time-step count";
  double m = 0.0, pi[3], pf[3];
  if (!F.read(&m, 8) || !F.read(pi, 24) || !F.read(pf, 24)) return "tppnp file: short tracer record";
  const bool fill = time && t9 && rho && a && z && zis && x;
  if (fill) {
    if (!F.read(time, 8 * (size_t)nt) || !F.read(t9, 8 * (size_t)nt) || !F.read(rho, 8 * (size_t)nt))
      return "tppnp file: short trajectory";
    for (int i = 0; i < nt; ++i) t9[i] = t9[i] / 1.e9;  // K -> GK, as read_trajectory does
  } else if (!F.skip(24 * (size_t)nt)) {
    return "tppnp file: short trajectory";
  }
  int32_t pn2[2];
  if (!F.read(pn2, sizeof pn2)) return "tppnp file: short abundance record";
  const int ni = pn2[1];
  if (ni < 0 || ni > (1 << 20)) return "tppnp file: bad isotope count";
  if (fill) {
    if (!F.read(a, 4 * (size_t)ni) || !F.read(z, 4 * (size_t)ni) || !F.read(zis, 5 * (size_t)ni) ||
        !F.read(x, 8 * (size_t)ni))
      return "tppnp file: short abundance record";
  } else if (!F.skip(17 * (size_t)ni)) {
    return "tppnp file: short abundance record";
  }
  *pnum = pn[0];
  *nsteps = nt;
  *niso = ni;
  if (mass) *mass = m;
  if (posini) std::memcpy(posini, pi, sizeof pi);
  if (posfin) std::memcpy(posfin, pf, sizeof pf);
  if (fill) *pos = (int64_t)std::ftell(F.f);
  return std::string();
}

}  // namespace nuppn
