// net_host.h -- one-time host analysis of a network description.
//
// Everything the reference recomputes per call or keeps in module state is prepared here once:
// the static Jacobian pattern of makemap (jac_rhs.F90:461-540), the accumulation orders of
// calculate_dxdt / calculate_jacobian (jac_rhs.F90:243-262, 363-392) turned into per-target gather
// lists, and a static-pivot sparse LU (fill-reducing order, filled pattern, update map and level
// schedules) that takes the place of SuperLU's per-call COLAMD + symbolic analysis
// (c_fortran_dgssv.c:110-119).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "nuppn_internal.h"

namespace nuppn {

struct HostNet {
  nuppn_knobs kn;
  int nsp = 0, nre = 0, ig = 0, nact = 0, nsys = 0, nnzJ = 0, nnzLU = 0, ihe4 = -1, ibe8 = -1;
  int nvar = 0;
  std::vector<double> an, zn, gspin_nse;
  // NSE set (nse_init, nse_swj.F90:208-245): species, nuclear mass (g), binding energy (MeV), 2J+1,
  // Z, N, Z/A, partition row (-1: none); positions of the proton and of Ni56 in the set (-1: absent)
  std::vector<int> nse_idx, nse_part;
  std::vector<double> nse_m, nse_q, nse_g, nse_z, nse_n, nse_zoa;
  int nse_iprot = -1, nse_ini56 = -1, nse_p2 = 1;
  std::vector<uint8_t> ciso, crea, rev_target;
  std::vector<int> spart, src, sidx, ilabb, scr_mode, irev, rev_sp, rev_kind;
  std::vector<double> rfac, scr_z1, scr_z2, rev_mc, rev_Q;
  std::vector<int> act_slot, act_k, act_ice;
  // raw k of all slots (for the pattern query)
  std::vector<int> k_all;
  // REACLIB
  int nc = 0, nr = 0;
  std::vector<int> rl_first, rl_info, rl_part;
  std::vector<double> rl_a;
  int npart = 0;
  std::vector<double> pt9, pval;
  int nv = 0;
  std::vector<int> vfirst, vxfac, vform;
  std::vector<double> vterms, vdpow;
  int ngk = 0, ngn = 0, ngd = 1;
  std::vector<double> ngt8, ngl10t8, ngflag, ngane, ngl10v;
  std::vector<int> ngndata;
  int ffv = 0, fft = 0, ffr = 0;
  std::vector<double> fft9, ffrho, ffl10v;
  int kdn = 0, kde = 0;
  std::vector<double> kdE, kdcoef;
  std::vector<double> constr;
  // pattern
  std::vector<int> jrow, jcol, jdiag, dmap_all;  // dmap_all[nre*8] (-1 for unconsidered)
  std::vector<int> jg_ptr, jg_item, dg_ptr, dg_item, jg_long, dg_long;
  std::vector<int> jg_oth;        // per jg item: the reaction's other reactant (the one not differentiated), -1 for gamma
  std::vector<int> k1_ptr, k1_list;  // species -> considered reactions it leads as k1, in order
  std::vector<double> dg_coef;
  // system / LU
  std::vector<int> sys_of_sp, sp_of_sys, pos_of_entry, lu_src;
  std::vector<int> lu_rowptr, lu_diag, lu_col, upd_start;
  std::vector<uint16_t> upd_off;
  std::vector<int> lvL_ptr, lvL_rows, lvL_grp, lvU_ptr, lvU_rows, lvU_grp;
  int64_t lu_flops = 0;
  // BD constants
  int nseq[kMaxLevels + 2];
  double bd_a[kMaxLevels + 2];
  double alf[kMaxLevels + 1][kMaxLevels + 1];
  int kmax = 0, kopt0 = 0;
};

// Builds the analysis; returns an empty string on success or a message describing the problem.
std::string build_host_net(const nuppn_net_desc &d, const nuppn_knobs &kn, HostNet &H);
void bd_constants(HostNet &H);

// One entry of an isotope database file (physics/run_template/isotopedatabase*.txt).
struct IsotopeEntry {
  int z = 0, a = 0;
  char elem[3] = {0, 0, 0};
  double amin = 0.0;  // the fourth column, a reference mass number
  bool consider = false;
};
// The first nnn entries of an isotope database file (read_isotopedatabase, nuc_data.F90:50-95):
// three header lines, then per line Z, A, element symbol, the reference mass number and a T/F flag,
// separated by blanks or tabs. Returns "" or what went wrong (the file cannot be opened, a line does
// not parse, or the file has fewer than nnn entries, where the reference stops the run).
std::string read_isotope_database(const char *path, int nnn, std::vector<IsotopeEntry> &out);

// networksetup.txt (netsetup.cpp): write_networksetup / read_networksetup of networksetup.F90.
std::string write_networksetup(const char *path, const nuppn_netsetup &ns);
std::string read_networksetup(const char *path, nuppn_netsetup &ns);

// ppn's per-cycle output files (output.cpp)
bool write_iso_massf(const char *path, int model, double dzeit, double agej, double t9, double rho, double densn,
                     double densp, double densa, double total_energy_flux, int nsp, const double *z, const double *a,
                     const int *isomeric_state, const double *x, const char *names, const uint8_t *consider);
bool write_flux(const char *path, int nreac, const int *k, const double *z, const double *a, const double *flux,
                const double *energy, const double *timescale);

// mppnp's diffusive mixing (mixing.cu): Lagrangian coefficient, the step's tridiagonal matrix and
// its factorization on the host; an empty string on success, else the reason
std::string mix_d_lagrangian(int m, const double *d_eul, const double *rho, const double *rad, double *d_lagr);
std::string mix_matrix(int m, const double *xm, const double *dq, double *d, double h, double sig, bool mesa,
                       std::vector<double> &a, std::vector<double> &b, std::vector<double> &c);
std::string tridag_factor(int m, const std::vector<double> &a, const std::vector<double> &b,
                          const std::vector<double> &c, std::vector<double> &gam, std::vector<double> &bet);

// tppnp's binary trajectory input (tppnp_io.cpp); an empty string on success, else the reason
std::string tppnp_header(const char *path, int *num_tracers, int *nsteps_min, int *nsteps_max);
std::string tppnp_next(const char *path, int64_t *pos, int *pnum, int *nsteps, int *niso, double *mass,
                       double *posini, double *posfin, double *time, double *t9, double *rho, int *a, int *z,
                       char *zis, double *x);

}  // namespace nuppn
