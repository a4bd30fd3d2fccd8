// oracle.cpp -- CPU checker for the device solver. TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Restates, in the reference's evaluation order, NuPPN's FP64 per-zone path:
//   evaluate_all_rates        physics/source/evaluate_rates.F90:14-196
//   reaclib rates/partition   physics/source/reaclib.F90:431-605
//   netgen / fuller / kadonis physics/source/netgen.F90:179-310, fuller.F90:92-122, kadonis.F90:150-187,
//                             utils/source/akima.F90:22-191, utils/source/utils.F90:624-722
//   reverse rates             physics/source/reverse.F90:107-335
//   screening (Chugunov)      physics/source/screening.F90:60-80, screening_chugunov.F90:67-234
//   calculate_dxdt            solver/source/jac_rhs.F90:217-278
//   calculate_jacobian        solver/source/jac_rhs.F90:282-455
//   makemap / dns2csr         solver/source/jac_rhs.F90:461-561
//   reduce_jacobian etc.      solver/source/jac_rhs.F90:97-213, 584-608
//   backward Euler Newton     solver/source/backward_euler.F90:29-176
//   Bader-Deuflhard           solver/source/bader_deuflhard.F90:66-488
//   integrate_network         solver/source/solver.F90:53-274
//   utils                     utils/source/utils.F90:481-553, 726-740, sort.F90:73-127, interp.F90:29-50
// and calls the reference's SuperLU (slu_solve, c_fortran_dgssv_) for every LU.
//
// VITAL rates are evaluated from analytic templates (see nuppn.h); every other formula follows the
// cited lines. Zone state is per call, so zones run on independent host threads.
#include "oracle.h"

#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <tuple>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

namespace {

using std::vector;

// ---- constants (utils/source/constants.F90) ---------------------------------------------------
const double ev2erg = 1.602177e-12, mev2erg = ev2erg * 1.0e6, erg2mev = 1.0 / mev2erg;
const double kev2erg = ev2erg * 1.0e3;
const double pi = 3.141592653589793238462643383279502884;  // acos(-1)
const double clight = 2.99792458e10, clight2 = clight * clight;
const double avogadro = 6.022140857e23, boltzmann = 1.3806485279e-16;
const double planck_mev = 4.135667662e-21, planck_erg = planck_mev * mev2erg;
const double hbar_erg = planck_erg / 2.0 / pi;
const double amu = 1.6605402e-24, mp_mev = 938.27231, mn_mev = 939.56563, me_g = 9.10938356e-28;
const double qe = 4.80320425e-10, qe2 = qe * qe;
const double ZERO = 0.0, ONE = 1.0, TWO = 2.0, THREE = 3.0, FOUR = 4.0, HALF = 0.5;
const double THIRD = 1.0 / 3.0, FOURTH = 1.0 / 4.0, FIFTH = 1.0 / 5.0, SIXTH = 1.0 / 6.0;
const double SMALL = 1.e-30;
const double SUM_TOL = 1.e-6;

// error codes, errors.F90:5-21
enum { SLV_CNVRG = 1, MAX_SUBSTEPS, BAD_STEP, NEG_ABUNDS, HUGE_ABUNDS, SUM_X, GOT_NAN, BAD_YE,
       NSE_CNVRG, NSE_WEAK, SMALL_DT };
// reaction types, reaction_info.F90:8-34
enum { i_ng = 1, i_gn, i_np, i_na, i_pg, i_gp, i_pn, i_pa, i_ag, i_ga, i_an, i_ap, i_bm, i_ec, i_bn,
       i_bp, i_ba, i_ve, i_vp, i_vsp, i_vsn, i_vsa };

// ---- reference SuperLU ------------------------------------------------------------------------
typedef void (*slu_solve_t)(int, int, int, int, double *, int *, int *, double *, int *);
typedef void (*dgssv_t)(int *, int *, int *, int *, double *, int *, int *, double *, int *,
                        long long *, int *);
slu_solve_t g_slu_solve = nullptr;
dgssv_t g_dgssv = nullptr;

// gfortran's integer power (libgcc __powidf2): square-and-multiply.
inline double powi(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

// NR indexx heapsort (sort.F90:73-127), 1-based in the original.
void indexx(int n, const double *arrin, vector<int> &indx) {
  indx.resize(n + 1);
  for (int j = 1; j <= n; ++j) indx[j] = j;
  if (n == 1) return;
  int l = n / 2 + 1, ir = n, indxt, i, j;
  double q;
  for (;;) {
    if (l > 1) {
      l = l - 1;
      indxt = indx[l];
      q = arrin[indxt - 1];
    } else {
      indxt = indx[ir];
      q = arrin[indxt - 1];
      indx[ir] = indx[1];
      ir = ir - 1;
      if (ir == 1) {
        indx[1] = indxt;
        return;
      }
    }
    i = l;
    j = l + l;
    while (j <= ir) {
      if (j < ir) {
        if (arrin[indx[j] - 1] < arrin[indx[j + 1] - 1]) j = j + 1;
      }
      if (q < arrin[indx[j] - 1]) {
        indx[i] = indx[j];
        i = j;
        j = j + j;
      } else {
        j = ir + 1;
      }
    }
    indx[i] = indxt;
  }
}

double sortedsum(const double *a, int n) {  // utils.F90:481-501
  vector<int> idx;
  indexx(n, a, idx);
  double s = 0.0;
  for (int i = 1; i <= n; ++i) s = s + a[idx[i] - 1];
  return s;
}

// bsearch_r8 (utils.F90:687-722): closest index (1-based) with arr(idx) <= val; arr 1-based via ptr-1
int bsearch_r8(const double *arr, int siz, double val) {
  int a = 1, b = siz, r = b - a, m = (a + b) / 2;
  while (val != arr[m - 1] && r > 1) {
    if (arr[m - 1] > val) b = m; else a = m;
    r = b - a;
    m = (a + b) / 2;
  }
  if (arr[m - 1] > val) m = m - 1;
  return m;
}

struct Akima {  // akima.F90 coefficients for one table
  vector<double> p0, p1, p2, p3;
};

void akima_setup(int n, const double *xpt, const double *ypt, Akima &ai) {  // akima.F90:78-132
  const double eps = 1e-30, delta_x = 0.1;
  vector<double> mm(n + 3), t(n + 1);
  auto m = [&](int i) -> double & { return mm[i + 1]; };  // m(-1:n+1)
  for (int i = 1; i <= n - 1; ++i) m(i) = (ypt[i] - ypt[i - 1]) / (xpt[i] - xpt[i - 1]);
  m(0) = 2.0 * m(1) - m(2);
  m(-1) = 2.0 * m(0) - m(1);
  m(n) = 2.0 * m(n - 1) - m(n - 2);
  m(n + 1) = 2.0 * m(n) - m(n - 1);
  auto abs_smooth = [&](double x) {
    if (x >= delta_x) return x;
    if (x <= -delta_x) return -x;
    return x * x / (2.0 * delta_x) + delta_x / 2.0;
  };
  for (int i = 1; i <= n; ++i) {
    double m1 = m(i - 2), m2 = m(i - 1), m3 = m(i), m4 = m(i + 1);
    double w1 = abs_smooth(m4 - m3), w2 = abs_smooth(m2 - m1);
    if (w1 < eps && w2 < eps) t[i] = 0.5 * (m2 + m3);
    else t[i] = (w1 * m2 + w2 * m3) / (w1 + w2);
  }
  ai.p0.resize(n); ai.p1.resize(n); ai.p2.resize(n); ai.p3.resize(n);
  for (int i = 1; i <= n - 1; ++i) {
    double dx = xpt[i] - xpt[i - 1], t1 = t[i], t2 = t[i + 1];
    ai.p0[i] = ypt[i - 1];
    ai.p1[i] = t1;
    ai.p2[i] = (3.0 * m(i) - 2.0 * t1 - t2) / dx;
    ai.p3[i] = (t1 + t2 - 2.0 * m(i)) / powi(dx, 2);
  }
}

double akima_eval(const Akima &ai, int npt, const double *xpt, double xx_in) {  // akima.F90:35-47,135-170
  double xx = std::max(xx_in, xpt[0]);
  xx = std::min(xx, xpt[npt - 1]);
  int j;
  if (xx < xpt[0]) {
    j = 1;
  } else {
    for (j = npt - 1; j >= 1; --j)
      if (xx >= xpt[j - 1]) break;
  }
  double dx = xx - xpt[j - 1];
  return ai.p0[j] + ai.p1[j] * dx + ai.p2[j] * powi(dx, 2) + ai.p3[j] * powi(dx, 3);
}

// ---- network -----------------------------------------------------------------------------------
struct Net {
  nuppn_knobs kn;
  int rhs_noise = -1;  // >= 0: seed of the dX/dt rounding perturbation (oracle_set_rhs_noise), else off
  int lu_permute = -1; // >= 0: seed of the LU elimination-order permutation (oracle_set_lu_permute), else off
  int nsp, nre, ig;
  vector<double> an, zn, exmass, gspin;
  vector<uint8_t> ciso, crea;
  vector<int> spart, k, ilabb, src, sidx, irev;
  vector<double> rfac;
  vector<uint8_t> rev_target;  // lab == 'RVRSE' (reverse.F90:73-74): gathered as 0
  // reaclib
  int nc, nr;
  vector<double> rla;
  vector<int> rlrate, rlchap, rlnireac, rlpart;
  vector<uint8_t> rlv, rlec;
  int npart;
  vector<double> pt9, pval;
  // vital
  int nv;
  vector<int> vfirst, vxfac, vform;
  vector<double> vterms, vdpow;
  // netgen
  int ngk, ngn, ngd;
  vector<double> ngt8, ngl10t8, ngflag, ngane, ngl10v;
  vector<int> ngndata;
  // fuller
  int ffv, fft, ffr;
  vector<double> fft9, ffrho, ffl10v;
  // kadonis
  int kdn, kde;
  vector<double> kdE, kdrate;
  vector<Akima> kdak;
  vector<double> constr;
  // derived nuclear data (nse_swj.F90:174-196)
  vector<double> ppn_m, ppn_q, ppn_g;
  // makemap
  int nnz;
  vector<int> jrow, jcol, dmap;  // 0-based species; dmap[l*8+s] 0-based entry or -1
  vector<int> rowptr;             // CSR of the full pattern (row-major numbering)
  // Bader-Deuflhard constants (bader_deuflhard.F90:66-124)
  int nseq[10];
  double a[10];
  double alf[9][9];
  int kmax, kopt0;
  // special species
  int ihe4, ibe8;
  // NSE set (nse_init, nse_swj.F90:208-245): species indices, positions of p, n, Ni56 in it
  vector<int> nse_idx;
  int nse_iprot = -1, nse_ineut = -1, nse_ini56 = -1;
};

template <class T>
vector<T> cp(const T *p, size_t n) {
  return p ? vector<T>(p, p + n) : vector<T>(n, T(0));
}

void bd_init(Net &N) {  // bader_deuflhard.F90:66-124
  const double cf = 1, cj = 0.0 * cf, cs = 10, clr = cj, safe1 = FOURTH;
  const double alpha = 5.0 / 7.0;
  const int nlevels = 8;
  N.nseq[1] = 2; N.nseq[2] = 6; N.nseq[3] = 10;
  for (int i = 4; i <= nlevels + 1; ++i) N.nseq[i] = (int)std::lround((double)N.nseq[i - 1] / alpha);
  N.a[1] = cj + clr + (N.nseq[1] + 1) * (cf + cs);
  for (int i = 2; i <= nlevels; ++i) N.a[i] = N.a[i - 1] + N.nseq[i] * (cf + cs) + clr + cs;
  N.a[nlevels + 1] = 0.0;  // never set by the reference when use_weights (only read via kopt+1<=kmax+1)
  for (int iq = 2; iq <= nlevels; ++iq)
    for (int k = 1; k <= iq - 1; ++k)
      N.alf[k][iq] = std::pow(N.kn.dgrd * safe1,
                              (N.a[k + 1] - N.a[iq + 1]) / ((N.a[iq + 1] - N.a[1] + ONE) * (TWO * k + 1)));
  int kopt;
  N.kmax = 0;
  for (kopt = 2; kopt <= nlevels - 1; ++kopt) {
    if (N.a[kopt + 1] > N.a[kopt] * N.alf[kopt - 1][kopt]) {
      N.kmax = kopt;
      break;
    }
  }
  N.kopt0 = kopt;
}

void makemap(Net &N) {  // jac_rhs.F90:461-540
  int n = N.nsp;
  vector<int> tmp((size_t)n * n, -1);
  for (int i = 0; i < N.nre; ++i) {
    if (!N.crea[i]) continue;
    const int *kk = &N.k[i * 8];
    int in1 = kk[0], in2 = kk[2], out1 = kk[4], out2 = kk[6];
    int r[4] = {in1, in2, out1, out2};
    for (int c : {in1, in2})
      for (int rr : r) tmp[(size_t)rr * n + c] = 1;
  }
  for (int i = 0; i < n; ++i)
    if (N.ciso[i]) tmp[(size_t)i * n + i] = 1;
  int cnt = 0;
  N.jrow.clear(); N.jcol.clear();
  N.rowptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    N.rowptr[i] = cnt;
    for (int j = 0; j < n; ++j)
      if (tmp[(size_t)i * n + j] != -1) {
        tmp[(size_t)i * n + j] = cnt++;
        N.jrow.push_back(i);
        N.jcol.push_back(j);
      }
  }
  N.rowptr[n] = cnt;
  N.nnz = cnt;
  N.dmap.assign((size_t)N.nre * 8, -1);
  for (int i = 0; i < N.nre; ++i) {
    if (!N.crea[i]) continue;
    const int *kk = &N.k[i * 8];
    int in1 = kk[0], in2 = kk[2], out1 = kk[4], out2 = kk[6];
    // slot order in1in1, in2in1, out1in1, out2in1, in1in2, in2in2, out1in2, out2in2 (jac_rhs.F90:72-80)
    int rr[8] = {in1, in2, out1, out2, in1, in2, out1, out2};
    int cc[8] = {in1, in1, in1, in1, in2, in2, in2, in2};
    for (int s = 0; s < 8; ++s) N.dmap[i * 8 + s] = tmp[(size_t)rr[s] * n + cc[s]];
  }
}

// ---- zone scratch ------------------------------------------------------------------------------
struct Zone {
  const Net *N;
  vector<double> v, v_rev, rv, reacv, partinter, xn, dxdt, jac, jacval_cpy;
  vector<int> jrow_flag;  // jac_coo%row: -1 = unset, else set (row index)
  vector<uint8_t> mask;
  int nvar1 = 0;
  // screening precalc state (screening_chugunov.F90:21-35)
  double abar, zbar, a_av, ntot, tp, wp, tk, tn, gamfac, zeta;
  // BD state
  int kopt;
  double qcol[9][1], xhist[9];
  vector<double> qc, ye_rr;  // qcol(nsp,8), yerr(nsp,8) flattened [k*nsp + i]
  double err[9], errmax, abuerr, negerr, sumerr;
  bool reduce = false;
  // NSE state (nse_swj.F90 module variables): work arrays and the last converged guess
  vector<double> nse_x, nse_gtot, nse_mucoul, lm_ov_a;
  double mu_p_coul = 0.0, nse_mu[2] = {0.0, 0.0}, nse_mu_last[2] = {-9.0, -9.0}, nse_the = 0.0, nse_phi = 0.0;
  bool nse_first = true;
  unsigned long long noise = 0;  // generator state of the dX/dt perturbation (oracle_set_rhs_noise)
  // stats
  nuppn_zone_stats st;
  explicit Zone(const Net *n) : N(n) {
    nse_x.assign(N->nse_idx.size(), 0.0); nse_gtot.assign(N->nse_idx.size(), 0.0);
    nse_mucoul.assign(N->nse_idx.size(), 0.0); lm_ov_a.assign(N->nsp, 0.0);
    v.assign(N->nre, 0.0); v_rev.assign(N->nre, 0.0);
    rv.assign(N->nr, 0.0); reacv.assign(N->nr, 0.0);
    partinter.assign(N->npart, 1.0);
    xn.assign(N->nsp, 0.0); dxdt.assign(N->nsp, 0.0);
    jac.assign(N->nnz, 0.0); jacval_cpy.assign(N->nnz, 0.0); jrow_flag.assign(N->nnz, -1);
    mask.assign(N->nsp, 0);
    qc.assign((size_t)9 * N->nsp, 0.0); ye_rr.assign((size_t)9 * N->nsp, 0.0);
    kopt = N->kopt0;
    sumerr = 0.0;
    memset(&st, 0, sizeof(st));
  }
};

// ---- rates -------------------------------------------------------------------------------------
void reaclib_partition(Zone &Z, double t9_in) {  // reaclib.F90:586-605
  const Net &N = *Z.N;
  if (N.npart == 0) return;
  const int pd = (int)N.pt9.size();
  double t9 = std::max(N.pt9[0], std::min(t9_in, N.pt9[pd - 1]));
  int i0 = bsearch_r8(N.pt9.data(), pd, t9);
  int i1 = i0 + 1;
  double t90 = N.pt9[i0 - 1], t91 = N.pt9[i1 - 1];
  double Dt9 = (t9 - t90) / (t91 - t90);
  for (int i = 0; i < N.npart; ++i) {
    const double *p = &N.pval[(size_t)i * pd];
    Z.partinter[i] = p[i0 - 1] + (p[i1 - 1] - p[i0 - 1]) * Dt9;
  }
}

void reaclib_rates(Zone &Z, double t9in, double rhoin, double yein) {  // reaclib.F90:431-582
  const Net &N = *Z.N;
  double t9 = std::max(t9in, 0.01);
  double rhoye = rhoin * yein;
  double t9inv = ONE / t9, t9pow13 = std::pow(t9, THIRD), t9pow13inv = ONE / t9pow13;
  double t9pow23 = t9pow13 * t9pow13, t9pow43 = t9 * t9pow13, t9pow53 = t9pow13 * t9pow43;
  (void)t9pow23;
  double lnt9 = std::log(t9);
  std::fill(Z.reacv.begin(), Z.reacv.end(), 0.0);
  for (int i = 0; i < N.nc; ++i) {
    const double *a = &N.rla[(size_t)i * 7];
    double r0 = a[0] + a[1] * t9inv + a[2] * t9pow13inv + a[3] * t9pow13 + a[4] * t9 + a[5] * t9pow53 +
                a[6] * lnt9;
    r0 = std::exp(r0);
    Z.reacv[N.rlrate[i]] = Z.reacv[N.rlrate[i]] + r0;
  }
  for (int j = 0; j < N.nr; ++j) {
    double Gfac = ONE;
    if (N.rlv[j]) {
      double g[6];
      for (int s = 0; s < 6; ++s) {
        int p = N.rlpart[j * 6 + s];
        g[s] = p < 0 ? 1.0 : Z.partinter[p];
      }
      double g1 = g[0], g2 = g[1], g3 = g[2], g4 = g[3], g5 = g[4], g6 = g[5];
      switch (N.rlchap[j]) {
        case 1: Gfac = g2 / g1; break;
        case 2: Gfac = g2 * g3 / g1; break;
        case 3: Gfac = g2 * g3 * g4 / g1; break;
        case 4: Gfac = g3 / (g1 * g2); break;
        case 5: Gfac = g3 * g4 / (g1 * g2); break;
        case 6: Gfac = g3 * g4 * g5 / (g1 * g2); break;
        case 7: Gfac = g3 * g4 * g5 * g6 / (g1 * g2); break;
        case 8: Gfac = g4 / (g1 * g2 * g3); break;
        case 9: Gfac = g4 * g5 / (g1 * g2 * g3); break;
        case 10: Gfac = g5 * g6 / (g1 * g2 * g3 * g4); break;
        case 11: Gfac = g2 * g3 * g4 * g5 * g6 / g1; break;
        default: Gfac = ONE;
      }
    }
    double rv_ = Z.reacv[j] * Gfac;
    switch (N.rlnireac[j]) {
      case i_bm: case i_gn: case i_bn: case i_bp: case i_gp: case i_ga: Z.rv[j] = rv_; break;
      case i_ec: Z.rv[j] = N.rlec[j] ? rv_ * rhoye : rv_; break;
      case i_ng: case i_pg: case i_ag: case i_np: case i_na: case i_pn: case i_pa: case i_an: case i_ap:
        Z.rv[j] = rv_ * rhoin; break;
      default: Z.rv[j] = 1.e-99;
    }
    Z.rv[j] = std::max(Z.rv[j], 1e-99);
  }
}

double exv(double x) {  // vital.F90:2583-2593
  if (x > 200.0) return (x - 200.0) * std::exp(200.0);
  if (x < -200.0) return -std::exp(-200.0) / (x + 200.0);
  return std::exp(x);
}

// vital_calculate_rates (vital.F90:239-569), the slots restated here: v(5) at every T9 (:340-343);
// for T9 >= 0.001 (:364) and 1.2e-3 < T9 < T9PPMAX (:366) V(1) :379, V(2) :395, V(3) :419, V(4)
// :442-445, V(6) :468-473, V(7) :478, V(9) :481-482, V(8) :487 (IPPIV = 0 leaves V(10)-V(13) zero);
// for T9 > 5e-3 (:532) V(14) :540-543 (the second fit replaces the first), V(73) :548, V(15) :556-558
// (likewise), V(16) :563-565, V(17) :568-571. Every other slot stays zero (:322).
double vital_reference(int slot, double T9, double RHO, double xprot) {
  const double THIRD = ONE / 3.0, FOURTH = ONE / 4.0, SIXTH = ONE / 6.0, FIVE_SIXTHS = 5.0 * SIXTH;
  const double T9PPMAX = 10.0, PROTOFAK = ONE;
  const double TP13 = std::pow(T9, THIRD), TP14 = std::pow(T9, FOURTH);
  const double TP12 = TP14 * TP14, TP23 = TP13 * TP13, TP32 = T9 * TP12, TP43 = T9 * TP13, TP53 = T9 * TP23;
  const double TM13 = ONE / TP13, TM23 = ONE / TP23, TM32 = ONE / TP32, t9inv = ONE / T9;
  double V[74] = {0.0};
  const double FABE7 = HALF * (ONE + xprot);
  V[5] = 1.34e-10 / TP12 * (ONE - 0.537 * TP13 + 3.86 * TP23 + 0.0027 * t9inv * exv(2.515e-03 * t9inv)) * RHO * FABE7;
  if (T9 < 1.e-03 || T9 > T9PPMAX) V[5] = std::min(V[5], 1.51e-07);
  if (T9 >= 0.001) {
    if (T9 > 1.2e-3 && T9 < T9PPMAX) {
      V[1] = (4.01e-15 * TM23 * exv(-3.380 * TM13) * (ONE + 0.123 * TP13 + 1.09 * TP23 + 0.938 * T9)) * RHO * PROTOFAK;
      V[2] = (2.24e+03 * TM23 * exv(-3.720 * TM13) * (ONE + 0.112 * TP13 + 3.38 * TP23 + 2.65 * T9)) * RHO * PROTOFAK;
      V[3] = (6.04e+10 * TM23 * exv(-12.276 * TM13) *
              (1.0 + 0.034 * TP13 - 0.522 * TP23 - 0.124 * T9 + 0.353 * TP43 + 0.213 * TP53)) * RHO;
      const double TT = T9 / (ONE + 4.95e-02 * T9);
      const double T56 = std::pow(TT, FIVE_SIXTHS), T13 = std::pow(TT, THIRD);
      V[4] = (5.61e+06 * T56 / TP32 * exv(-12.826 / T13)) * RHO;
      const double T9A = T9 / (ONE + 0.759 * T9);
      const double T9A13 = std::pow(T9A, THIRD), T9A56 = std::pow(T9A, FIVE_SIXTHS);
      V[6] = (1.096e+09 / TP23 * exv(-8.472 / TP13) - 4.83e+08 * T9A56 / TP32 * exv(-8.472 / T9A13) +
              1.06e+10 / TP32 * exv(-30.442 / T9)) * RHO * PROTOFAK;
      V[7] = (3.11e5 / TP23 * exv(-10.262 / TP13) + 2.53e3 / TP32 * exv(-7.306 / T9)) * RHO * PROTOFAK;
      const double REV = 1.30e+10 * TP32 * exv(-1.595 / T9) / (RHO);
      V[9] = REV * V[7];
      V[8] = 8.96e-1;
    }
    if (T9 > 5.e-3) {
      V[14] = (2.00e+07 * TM23 * exv(-13.692 * TM13 - (T9 / 0.46) * (T9 / 0.46)) *
                   (1.0 + 9.89 * T9 - 59.8 * T9 * T9 + 266.0 * T9 * T9 * T9) +
               1.00e+05 * TM32 * exv(-4.913 / T9) + 4.24e+05 * TM32 * exv(-21.62 / T9));
      V[14] = V[14] * RHO * PROTOFAK;
      V[73] = V[14] / (RHO * PROTOFAK) * 8.84e+09 * TP32 * exv(-22.553 / T9);
      V[15] = (9.57e+07 * TM23 * exv(-13.720 * TM13 - T9 * T9) * (1 + 3.56 * T9) + 1.50e+06 * TM32 * exv(-5.930 / T9) +
               std::exp(-12.057 / T9) * 6.83e+05 / std::pow(T9, 0.864)) * RHO * PROTOFAK;
      V[16] = 4.04e+07 * TM23 * exv(-15.202 * TM13 - (T9 / 1.191) * (T9 / 1.191)) *
                  (1.0 + 0.027 * TP13 - 0.803 * TP23 - 0.154 * T9 + 5.00 * TP43 + 2.44 * TP53) +
              2.43e+05 * TM32 * exv(-6.348 / T9) * RHO * PROTOFAK;
      V[17] = (4.90e7 / TP23 * exv(-15.228 / TP13 - (T9 / 3.294) * (T9 / 3.294)) *
                   (ONE + 0.027 * TP13 - 0.778 * TP23 - 0.149 * T9 + 0.261 * TP43 + 0.127 * TP53) +
               2.37e3 / TP32 * exv(-3.011 / T9) + 2.19e4 * exv(-12.530 / T9)) * RHO * PROTOFAK;
    }
  }
  return (slot >= 1 && slot <= 73) ? V[slot] : 0.0;
}

double vital_rate(const Net &N, int r, double t9_in, double rho, const double *x) {
  double t9 = std::min(t9_in, 10.0);  // vital.F90:230
  if (N.vform[r] > 0) return vital_reference(N.vform[r], t9, rho, N.vxfac[r] >= 0 ? x[N.vxfac[r]] : 0.0);
  // analytic template: rho^dpow * xfac * sum c*T9^p*exp(d*T9^(-1/3) + f/T9 + g*T9)
  double tm13 = ONE / std::pow(t9, THIRD);
  double s = 0.0;
  for (int t = N.vfirst[r]; t < N.vfirst[r + 1]; ++t) {
    const double *c = &N.vterms[(size_t)t * 5];
    s = s + c[0] * std::pow(t9, c[1]) * std::exp(c[2] * tm13 + c[3] / t9 + c[4] * t9);
  }
  double f = std::pow(rho, N.vdpow[r]);
  if (N.vxfac[r] >= 0) f = f * (HALF * (ONE + x[N.vxfac[r]]));
  return s * f;
}

void netgen_rates(const Net &N, double t9, double rho, double ye, double *out) {  // netgen.F90:179-310
  if (N.ngn == 0) return;
  double t8 = t9 * 10.0, rhoye = rho * ye, ane_in = rhoye * avogadro;
  double rhop2 = rho * rho, rhop3 = rho * rho * rho;
  double mxr = -ONE, flg = -ONE;
  int ndt = -1;
  t8 = std::min(std::max(t8, N.ngt8[0]), N.ngt8[N.ngk - 1]);
  int k = bsearch_r8(N.ngt8.data(), N.ngk, t8);
  int klo = k, khi = klo + 1;
  double h = N.ngl10t8[khi - 1] - N.ngl10t8[klo - 1];
  double b = (std::log10(t8) - N.ngl10t8[klo - 1]) / h;
  int jlo = 1, jhi = 2;
  double anelo = 0, anehi = 0, dane = 0, deltagrid = 1;
  auto L = [&](int kk, int i, int j) { return N.ngl10v[((size_t)(kk - 1) * N.ngn + i) * N.ngd + (j - 1)]; };
  for (int i = 0; i < N.ngn; ++i) {
    double v = 0.0;
    // vgrid(k,i,1) <= 0 test: tables hold log10 values; the linear grid is 10**l10v > 0 always
    if (N.ngflag[i] <= ZERO) {
      double lo = L(klo, i, 1), hi = L(khi, i, 1);
      double l10rate = lo + b * (hi - lo);
      switch ((int)std::lround(N.ngflag[i])) {
        case -14:
          v = std::pow(10.0, l10rate) * rhoye;
          if (t8 < 0.01) v = std::min(v, 1.51e-7 / rhoye);
          break;
        case -13: v = std::pow(10.0, l10rate) * rhoye; break;
        case -11: v = std::pow(10.0, l10rate); break;
        case -10: v = std::pow(10.0, l10rate) * rho / 1.0 / 1.0; break;
        case -100: v = std::pow(10.0, l10rate) * rhop2 / 1.0 / 1.0; break;
        case -200: v = std::pow(10.0, l10rate) * rhop3 / 1.0 / 1.0; break;
        default: v = ZERO;
      }
    } else {
      double oldflg = flg; flg = N.ngflag[i];
      int oldndt = ndt; ndt = N.ngndata[i];
      double oldmxr = mxr; mxr = N.ngane[(size_t)i * N.ngd + ndt - 1];
      if (flg != oldflg || ndt != oldndt || oldmxr != mxr) {
        double ane = std::min(std::max(ane_in, flg), mxr);
        int j = bsearch_r8(&N.ngane[(size_t)i * N.ngd], ndt, ane);
        jlo = j; jhi = jlo + 1;
        anelo = N.ngane[(size_t)i * N.ngd + jlo - 1];
        anehi = N.ngane[(size_t)i * N.ngd + jhi - 1];
        dane = ane - anelo;
        deltagrid = anehi - anelo;
      }
      double vlow = L(klo, i, jlo) + b * (L(khi, i, jlo) - L(klo, i, jlo));
      double vhigh = L(klo, i, jhi) + b * (L(khi, i, jhi) - L(klo, i, jhi));
      vlow = std::pow(10.0, vlow);
      vhigh = std::pow(10.0, vhigh);
      v = (vhigh - vlow) / deltagrid * dane + vlow;
    }
    out[i] = std::max(v, 1e-99);
  }
}

void fuller_rates(const Net &N, double t9in, double rhoin, double yein, double *out) {  // fuller.F90:92-122
  if (N.ffv == 0) return;
  double t90 = std::log10(t9in), rho0 = std::log10(rhoin * yein);
  t90 = std::min(std::max(t90, N.fft9[0]), N.fft9[N.fft - 1]);
  rho0 = std::min(std::max(rho0, N.ffrho[0]), N.ffrho[N.ffr - 1]);
  int ix1 = bsearch_r8(N.fft9.data(), N.fft, t90), iy1 = bsearch_r8(N.ffrho.data(), N.ffr, rho0);
  int ix2 = ix1 + 1, iy2 = iy1 + 1;
  // generic_interp_2d (utils.F90:624-666)
  double x1 = N.fft9[ix1 - 1], x2 = N.fft9[ix2 - 1], y1 = N.ffrho[iy1 - 1], y2 = N.ffrho[iy2 - 1];
  double dx = x2 - x1, dy = y2 - y1;
  double xb = (t90 - x1) / dx, xa = 1.0 - xb, yb = (rho0 - y1) / dy, ya = 1.0 - yb;
  for (int v = 0; v < N.ffv; ++v) {
    auto F = [&](int ix, int iy) { return N.ffl10v[((size_t)v * N.fft + (ix - 1)) * N.ffr + (iy - 1)]; };
    double f11 = F(ix1, iy1), f21 = F(ix2, iy1), f12 = F(ix1, iy2), f22 = F(ix2, iy2);
    double fA = f11 * ya + f12 * yb;
    double fC = f21 * ya + f22 * yb;
    double res = fA * xa + fC * xb;
    out[v] = std::pow(10.0, res);
  }
}

void kadonis_rates(const Net &N, double t9, double rho, double *out) {  // kadonis.F90:150-187
  if (N.kdn == 0) return;
  double Ekev_in = t9 * 1e9 * (boltzmann / kev2erg);
  double Ekev = std::min(std::max(Ekev_in, N.kdE[0]), N.kdE[N.kde - 1]);
  for (int i = 0; i < N.kdn; ++i) out[i] = akima_eval(N.kdak[i], N.kde, N.kdE.data(), Ekev) * rho;
}

// screening_chugunov.F90:67-134
void screen_precalc(Zone &Z, const double *x, double tkin, double rho) {
  const Net &N = *Z.N;
  // calculate_azbar (utils.F90:504-525): sums over the mask in index order
  double ytot = 0, sa = 0, sz = 0;
  for (int i = 0; i < N.nsp; ++i) {
    if (!N.ciso[i]) continue;
    double y = x[i] / N.an[i];
    ytot += y;
  }
  for (int i = 0; i < N.nsp; ++i) {
    if (!N.ciso[i]) continue;
    double y = x[i] / N.an[i];
    sa += N.an[i] * y;
  }
  for (int i = 0; i < N.nsp; ++i) {
    if (!N.ciso[i]) continue;
    double y = x[i] / N.an[i];
    sz += N.zn[i] * y;
  }
  Z.abar = sa / ytot;
  Z.zbar = sz / ytot;
  const double fourov3pi = FOUR / (THREE * pi * pi), fourpiqe2 = FOUR * pi * qe2;
  const double t1 = 0.1, t2 = 0.2, t0 = (t1 + t2) * HALF;
  Z.ntot = rho / (Z.abar * amu);
  double denom = std::pow(THREE / (FOUR * pi * Z.zbar * Z.ntot), THIRD);
  Z.a_av = denom * std::pow(Z.zbar, THIRD);
  Z.wp = std::pow(fourpiqe2 * Z.zbar * Z.zbar * Z.ntot / (Z.abar * amu), HALF);
  Z.tp = hbar_erg * Z.wp / boltzmann;
  Z.tn = tkin / Z.tp;
  if (Z.tn >= TWO * t2) {
    Z.tk = tkin;
  } else if (Z.tn <= HALF * t1) {
    Z.tk = t1 * Z.tp;
  } else {
    double s = ONE / (ONE + std::exp(-(Z.tn - t0) / 0.01));
    Z.tn = (ONE - s) * t1 + s * Z.tn;
    Z.tk = Z.tn * Z.tp;
  }
  Z.gamfac = qe2 / (Z.a_av * Z.tk) / boltzmann;
  Z.zeta = std::pow(fourov3pi * Z.tp * Z.tp / Z.tk / Z.tk, THIRD);
}

double screen_factor(const Zone &Z, double z1, double z2) {  // screening_chugunov.F90:140-234
  const double c_a1 = 2.7822, c_a2 = 98.34, c_a3 = std::sqrt(THREE) - c_a1 / std::sqrt(c_a2);
  const double c_b1 = -1.7476, c_b2 = 66.07, c_b3 = 1.12, c_b4 = 65.0, alfa = 0.022;
  const double gamfitlim = 600.0, g0 = 599.0;
  if (z1 <= ZERO || z2 <= ZERO) return ONE;
  double z1z2 = z1 * z2;
  double gam = z1z2 * Z.gamfac;
  double beta = 0.41 - 0.6 / gam, gama = 0.06 + 2.2 / gam;
  double gamtild = gam / std::pow(ONE + alfa * Z.zeta + beta * powi(Z.zeta, 2) + gama * powi(Z.zeta, 3), THIRD);
  if (gamtild >= 650) {
    gamtild = gamfitlim;
  } else if (gamtild <= 550) {
  } else {
    double s = ONE / (ONE + std::exp(-(gamtild - g0) / ONE));
    gamtild = s * gamfitlim + (1 - s) * gamtild;
  }
  double gamtild2 = gamtild * gamtild;
  double t1 = std::pow(gamtild, THREE * HALF) * (c_a1 / std::sqrt(c_a2 + gamtild) + c_a3 / (1 + gamtild));
  double t2 = c_b1 * gamtild2 / (c_b2 + gamtild);
  double t3 = c_b3 * gamtild2 / (c_b4 + gamtild2);
  double screen = std::exp(t1 + t2 + t3);
  screen = std::min(screen, 1e30);
  return screen;
}

double calc_screening(const Zone &Z, int r1, int r2) {  // screening.F90:60-80
  const Net &N = *Z.N;
  double screen;
  switch (N.kn.screen_option) {
    case 0: screen = ONE; break;
    case 2: screen = screen_factor(Z, N.zn[r1], N.zn[r2]); break;
    default: screen = ONE;  // Graboske (option 1) is not part of the default path
  }
  return std::min(screen, 1.e30);
}

// reverse.F90:178-335 (Coulomb corrections off: use_coulomb_corrections = .false.)
bool reverse_rate(const Zone &Z, int idx, double rho, double t9, const double *G, double &fac) {
  const Net &N = *Z.N;
  double kTerg = boltzmann * t9 * 1.e9, kTMeV = kTerg * erg2mev;
  const int *kk = &N.k[idx * 8];
  int a1 = kk[0], a2 = kk[2], b1 = kk[4], b2 = kk[6];
  int na1 = kk[1], nb1 = kk[5], nb2 = kk[7];
  double G_a1 = G[a1], m_a1 = N.ppn_m[a1], G_a2, m_a2, G_b1, m_b1;
  if (na1 == 1) { G_a2 = G[a2]; m_a2 = N.ppn_m[a2]; }
  else if (na1 == 2) { G_a2 = G_a1; m_a2 = m_a1; }
  else return false;
  double G_b2 = G[b2], m_b2 = N.ppn_m[b2];
  if (nb2 == 1) {
    if (nb1 == 1) { G_b1 = G[b1]; m_b1 = N.ppn_m[b1]; }
    else { G_b1 = ZERO; m_b1 = ZERO; }  // nb1 == 0 (other values leave them undefined in the reference)
  } else if (nb2 == 2) { G_b1 = G_b2; m_b1 = m_b2; }
  else return false;
  double pfac, mfac, Q, rhofac;
  switch (N.ilabb[idx]) {
    case i_ng: case i_pg: case i_ag:
      pfac = G_a1 * G_a2 / G_b2;
      mfac = std::pow(m_a1 * m_a2 / m_b2 * kTerg * TWO * pi / planck_erg / planck_erg, 1.5);
      Q = -N.ppn_q[a1] - N.ppn_q[a2] + N.ppn_q[b2];
      rhofac = ONE / rho / avogadro;
      break;
    default:
      pfac = G_a1 * G_a2 / G_b1 / G_b2;
      mfac = std::pow(m_a1 * m_a2 / m_b1 / m_b2, 1.5);
      Q = -N.ppn_q[a1] - N.ppn_q[a2] + N.ppn_q[b1] + N.ppn_q[b2];
      rhofac = ONE;
  }
  double x = std::min(-Q / kTMeV, 200.0);
  double efac = std::exp(x);
  fac = mfac * efac * rhofac;
  fac = fac * pfac;
  fac = std::min(std::max(fac, 1e-99), 1e99);
  return true;
}

void evaluate_all_rates(Zone &Z, double ye, double rho, double t9, const double *yps) {
  const Net &N = *Z.N;
  vector<double> &v = Z.v;
  // rnetw2008 (ppn_physics.F90:1025-1119): v = 0, VITAL, networkII gather, alpha decays
  std::fill(v.begin(), v.end(), 0.0);
  reaclib_partition(Z, t9);
  reaclib_rates(Z, t9, rho, ye);
  vector<double> ng(N.ngn, 0.0), ff(N.ffv, 0.0), kd(N.kdn, 0.0);
  netgen_rates(N, t9, rho, ye, ng.data());
  fuller_rates(N, t9, rho, ye, ff.data());
  if (t9 > 0.001) kadonis_rates(N, t9, rho, kd.data());  // t9_netgen_limit (netgen.F90:42)
  for (int l = 0; l < N.nre; ++l) {
    if (N.rev_target[l]) { v[l] = 0.0; continue; }  // lab 'RVRSE': not gathered
    int i = N.sidx[l];
    switch (N.src[l]) {
      case NUPPN_SRC_VITAL: v[l] = vital_rate(N, i, t9, rho, yps); break;
      case NUPPN_SRC_REACLIB: v[l] = Z.rv[i]; break;
      case NUPPN_SRC_NETGEN: v[l] = ng[i]; break;
      case NUPPN_SRC_FULLER: v[l] = ff[i]; break;
      case NUPPN_SRC_KADONIS: v[l] = kd[i]; break;
      case NUPPN_SRC_CONST: v[l] = N.constr[i]; break;
      default: v[l] = 0.0;
    }
  }
  // apply_rate_factors (evaluate_rates.F90:176-196), networksetup factors only
  for (int l = 0; l < N.nre; ++l) v[l] = std::max(v[l] * N.rfac[l], 1.e-99);
  // calculate_reverse_rates (reverse.F90:107-174)
  if (N.kn.detailed_balance) {
    reaclib_partition(Z, t9);
    vector<double> G(N.nsp, ONE);
    for (int i = 0; i < N.nsp; ++i)
      if (N.ppn_g[i] != 0.0 && i != N.ig && N.ciso[i] && N.an[i] != 0)  // nse_mask
        G[i] = (N.spart[i] >= 0 ? Z.partinter[N.spart[i]] : ONE) * N.ppn_g[i];
    for (int i = 0; i < N.nre; ++i) {
      if (!N.crea[i] || N.irev[i] == -1) continue;
      if (v[i] > 1.e-97) {
        double fac;
        if (!reverse_rate(Z, i, rho, t9, G.data(), fac)) continue;
        Z.v_rev[i] = std::max(v[i] * fac, 1e-99);
        v[N.irev[i]] = Z.v_rev[i];
      }
    }
  }
  // screening (evaluate_rates.F90:58-121)
  double tk = t9 * 1.e9;
  if (N.kn.screen_option == 2) screen_precalc(Z, yps, tk, rho);
  for (int i = 0; i < N.nre; ++i) {
    if (!N.crea[i] && i + 1 > 110) continue;
    if (v[i] <= 1.e-99) continue;
    double Fs, Fa;
    if (i + 1 == 43) {
      Fs = calc_screening(Z, N.ihe4, N.ihe4);
      Fa = calc_screening(Z, N.ihe4, N.ibe8);
      v[i] = v[i] * Fs * Fa;
    } else if (i + 1 == 109) {
      Fs = calc_screening(Z, N.ihe4, N.ihe4);
      v[i] = v[i] * Fs;
    } else {
      const int *kk = &N.k[i * 8];
      if (kk[1] == 2) Fs = calc_screening(Z, kk[0], kk[0]);
      else Fs = calc_screening(Z, kk[0], kk[2]);
      v[i] = v[i] * Fs;
    }
  }
  auto weak = [](int t) {
    return t == i_ec || t == i_bm || t == i_bn || t == i_bp || t == i_ve || t == i_vp || t == i_vsp ||
           t == i_vsn || t == i_vsa;
  };
  if (!N.kn.weak_rates)
    for (int i = 0; i < N.nre; ++i)
      if (N.crea[i] && weak(N.ilabb[i])) v[i] = 1.e-99;
  if (!N.kn.strong_rates)
    for (int i = 0; i < N.nre; ++i)
      if (N.crea[i] && !weak(N.ilabb[i])) v[i] = 1.e-99;
  if (N.kn.decay)
    for (int i = 0; i < N.nre; ++i) {
      if (!N.crea[i]) continue;
      int t = N.ilabb[i];
      if (t == i_ec || t == i_bm || t == i_bn || t == i_bp || t == i_ba) continue;
      v[i] = 1.e-99;
    }
  for (int i = 0; i < N.nre; ++i) v[i] = std::max(v[i], 1.e-99);
}

// ---- RHS and Jacobian --------------------------------------------------------------------------
const double fact[5] = {ONE, ONE, HALF, SIXTH, ONE / 24.0};

// Test infrastructure, off unless oracle_set_rhs_noise was called: every dX/dt entry scaled by
// 1 - 2^-52, 1 or 1 + 2^-52 at random, a change of the size of one rounding of the sum. An
// implementation that sums the same terms in another order differs from the reference by such
// amounts; the spread of the checker's results under this perturbation is how far the reference's
// own answer depends on them. Each zone draws from its own generator (seed, zone), so results do not
// depend on the thread count.
static unsigned long long noise_state(int seed, int z) {
  unsigned long long x = 0x9E3779B97F4A7C15ull * (unsigned long long)(seed + 1) + 0xD1B54A32D192ED03ull * (unsigned long long)(z + 1);
  x ^= x >> 31;
  return x | 1ull;
}

static void rhs_perturb(Zone &Z) {
  for (int i = 0; i < Z.N->nsp; ++i) {
    Z.noise = Z.noise * 6364136223846793005ull + 1442695040888963407ull;
    const int u = (int)((Z.noise >> 33) % 3ull) - 1;
    Z.dxdt[i] = Z.dxdt[i] * (1.0 + u * 2.220446049250313e-16);
  }
}

void calculate_dxdt(Zone &Z, const double *x_in) {  // jac_rhs.F90:217-278
  const Net &N = *Z.N;
  std::fill(Z.dxdt.begin(), Z.dxdt.end(), 0.0);
  std::fill(Z.xn.begin(), Z.xn.end(), 0.0);
  for (int i = 0; i < N.nsp; ++i)
    if (N.ciso[i] && N.an[i] != 0) Z.xn[i] = x_in[i] / N.an[i];
  Z.xn[N.ig] = ONE;
  for (int i = 0; i < N.nre; ++i) {
    if (!N.crea[i]) continue;
    const int *kk = &N.k[i * 8];
    double vx = fact[kk[1]] * Z.v[i] * powi(Z.xn[kk[0]], kk[1]) * Z.xn[kk[2]];
    double dx1dt = (double)(-kk[1]) * vx, dx3dt = -vx, dx5dt = (double)kk[5] * vx, dx7dt = (double)kk[7] * vx;
    Z.dxdt[kk[0]] = Z.dxdt[kk[0]] + dx1dt;
    Z.dxdt[kk[2]] = Z.dxdt[kk[2]] + dx3dt;
    Z.dxdt[kk[4]] = Z.dxdt[kk[4]] + dx5dt;
    Z.dxdt[kk[6]] = Z.dxdt[kk[6]] + dx7dt;
  }
  for (int i = 0; i < N.nsp; ++i)
    if (N.ciso[i]) Z.dxdt[i] = Z.dxdt[i] * N.an[i];
  Z.xn[N.ig] = ZERO;
  Z.dxdt[N.ig] = ZERO;
  if (N.rhs_noise >= 0) rhs_perturb(Z);
}

void calculate_jacobian(Zone &Z, double dzeit, const double *x_in) {  // jac_rhs.F90:282-455
  const Net &N = *Z.N;
  const int g = N.ig;
  vector<double> &jac = Z.jac;
  vector<int> &row = Z.jrow_flag;
  vector<uint8_t> &mask = Z.mask;
  std::fill(mask.begin(), mask.end(), 0);
  double dfdNmin = N.kn.cyminformal / dzeit;
  std::fill(jac.begin(), jac.end(), 1.e-99);
  std::fill(row.begin(), row.end(), -1);
  for (int i = 0; i < N.nsp; ++i)
    if (N.ciso[i] && N.an[i] > ZERO) Z.xn[i] = x_in[i] / N.an[i];
  Z.xn[g] = ONE;
  for (int l = 0; l < N.nre; ++l) {
    if (!N.crea[l]) continue;
    if (std::fabs(Z.v[l]) / dzeit <= N.kn.min_rate_ov_dt) continue;
    const int *kk = &N.k[l * 8];
    int in1 = kk[0], in2 = kk[2], out1 = kk[4], out2 = kk[6];
    int Nin1 = kk[1], Nin2 = kk[3], Nout1 = kk[5], Nout2 = kk[7];
    double ain1 = N.an[in1], ain2 = N.an[in2], aout1 = N.an[out1], aout2 = N.an[out2];
    double y1 = Z.xn[in1], y2 = Z.xn[in2];
    const int *ice = &N.dmap[l * 8];
    int ice1 = ice[0], ice2 = ice[1], ice3 = ice[4], ice4 = ice[2], ice5 = ice[3], ice6 = ice[5],
        ice7 = ice[6], ice8 = ice[7];
    double stem = fact[Nin1] * fact[Nin2] * Z.v[l];
    double dfdN = stem * powi(y1, Nin1) * y2;
    if (std::fabs(dfdN) > dfdNmin) {
      mask[in1] = 1; mask[in2] = 1; mask[out1] = 1; mask[out2] = 1;
    }
    stem = (double)Nin1 * fact[Nin1] * fact[Nin2] * powi(y2, Nin2) * powi(y1, Nin1 - 1) * Z.v[l];
    double dfin1dy1 = (double)(-Nin1) * stem, dfin2dy1 = (double)(-Nin2) * stem;
    double dfout1dy1 = (double)Nout1 * stem, dfout2dy1 = (double)Nout2 * stem;
    stem = (double)Nin2 * fact[Nin1] * fact[Nin2] * powi(y1, Nin1) * powi(y2, Nin2 - 1) * Z.v[l];
    double dfin1dy2 = (double)(-Nin1) * stem, dfin2dy2 = (double)(-Nin2) * stem;
    double dfout1dy2 = (double)Nout1 * stem, dfout2dy2 = (double)Nout2 * stem;
    if (in1 != g) jac[ice1] = jac[ice1] + dfin1dy1 * ain1 / ain1;
    if (in1 != g && in2 != g) {
      jac[ice2] = jac[ice2] + dfin2dy1 * ain2 / ain1;
      jac[ice3] = jac[ice3] + dfin1dy2 * ain1 / ain2;
    }
    if (in1 != g && out1 != g) jac[ice4] = jac[ice4] + dfout1dy1 * aout1 / ain1;
    if (in1 != g && out2 != g) jac[ice5] = jac[ice5] + dfout2dy1 * aout2 / ain1;
    if (in2 != g) jac[ice6] = jac[ice6] + dfin2dy2 * ain2 / ain2;
    if (in2 != g && out1 != g) jac[ice7] = jac[ice7] + dfout1dy2 * aout1 / ain2;
    if (in2 != g && out2 != g) jac[ice8] = jac[ice8] + dfout2dy2 * aout2 / ain2;
    if (in2 != g && !mask[in2]) continue;
    if (out1 != g && !mask[out1]) continue;
    if (mask[in1] && mask[out2]) {
      if (in1 != g) row[ice1] = in1;
      if (in1 != g && in2 != g) { row[ice2] = in2; row[ice3] = in1; }
      if (in1 != g && out1 != g) row[ice4] = out1;
      if (in1 != g && out2 != g) row[ice5] = out2;
      if (in2 != g) row[ice6] = in2;
      if (in2 != g && out1 != g) row[ice7] = out1;
      if (in2 != g && out2 != g) row[ice8] = out2;
    }
  }
  Z.xn[g] = ZERO;
  mask[g] = 0;
}

// reduce_jacobian (jac_rhs.F90:134-197) on Z.jac (already scaled by -dt or -h) + coocsr; 1-based CSR
void reduce_jacobian(Zone &Z, vector<double> &val, vector<int> &colind, vector<int> &rowptr, int &nvar1) {
  const Net &N = *Z.N;
  vector<double> &jac = Z.jac;
  vector<int> &row = Z.jrow_flag;
  for (int i = 0; i < N.nnz; ++i)
    if ((std::fabs(jac[i]) == ZERO || jac[i] == -ONE) && row[i] != -1) row[i] = -1;
  nvar1 = 0;
  vector<int> iexpand(N.nsp, -1);
  for (int i = 0; i < N.nsp; ++i) {
    if (!Z.mask[i]) continue;
    nvar1 = nvar1 + 1;
    iexpand[i] = nvar1;
    int ice = N.rowptr[i];  // dns2csr(i,i): diagonal entry of row i
    while (N.jcol[ice] != i) ++ice;
    row[ice] = i;
    jac[ice] = jac[ice] + ONE;
  }
  // pack in COO (= row-major) order; coocsr keeps the within-row order
  rowptr.assign(nvar1 + 1, 0);
  val.clear(); colind.clear();
  vector<int> cnt(nvar1 + 2, 0);
  vector<int> rr, cc; vector<double> vv;
  for (int e = 0; e < N.nnz; ++e) {
    if (row[e] == -1) continue;
    int r = iexpand[N.jrow[e]], c = iexpand[N.jcol[e]];
    rr.push_back(r); cc.push_back(c); vv.push_back(jac[e]);
  }
  int n_ice = (int)rr.size();
  // coocsr (sparsekit_module.F90:152): counting sort by row, stable
  vector<int> iao(nvar1 + 2, 0);
  for (int k = 0; k < n_ice; ++k) iao[rr[k]] += 1;
  int k0 = 1;
  for (int j = 1; j <= nvar1 + 1; ++j) { int k1 = iao[j]; iao[j] = k0; k0 = k0 + k1; }
  val.assign(n_ice, 0.0); colind.assign(n_ice, 0);
  for (int k = 0; k < n_ice; ++k) {
    int i = rr[k], j = cc[k], iad = iao[i];
    val[iad - 1] = vv[k];
    colind[iad - 1] = j;
    iao[i] = iad + 1;
  }
  for (int j = nvar1; j >= 1; --j) iao[j + 1] = iao[j];
  iao[1] = 1;
  rowptr.assign(iao.begin() + 1, iao.begin() + nvar1 + 2);
}

// csrcsc (sparsekit) for the BD factorization, 1-based in/out
void csr_to_csc(int n, const vector<double> &a, const vector<int> &ja, const vector<int> &ia,
                vector<double> &ao, vector<int> &jao, vector<int> &iao) {
  int nnz = ia[n] - 1;
  iao.assign(n + 2, 0);
  for (int i = 1; i <= n; ++i)
    for (int k = ia[i - 1]; k <= ia[i] - 1; ++k) iao[ja[k - 1] + 1] += 1;
  iao[1] = 1;
  for (int i = 1; i <= n; ++i) iao[i + 1] = iao[i] + iao[i + 1];
  ao.assign(nnz, 0.0); jao.assign(nnz, 0);
  for (int i = 1; i <= n; ++i)
    for (int k = ia[i - 1]; k <= ia[i] - 1; ++k) {
      int j = ja[k - 1], next = iao[j];
      ao[next - 1] = a[k - 1];
      jao[next - 1] = i;
      iao[j] = next + 1;
    }
  for (int i = n; i >= 1; --i) iao[i + 1] = iao[i];
  iao[1] = 1;
  iao.erase(iao.begin());
  iao.resize(n + 1);
}

void ypsplus(vector<double> &yps) {  // utils.F90:726-740
  const double yminformal = 1.e-27;
  for (double &y : yps) if (y < -yminformal) y = 1.e-99;
  for (double &y : yps) if (y < yminformal) y = 1.e-99;
}

double seqsum(const vector<double> &a) {
  double s = 0.0;
  for (double x : a) s = s + x;
  return s;
}

double maxval_neg(const vector<double> &y) {
  double m = -1.7976931348623157e308;
  for (double x : y) m = std::max(m, -x);
  return m;
}

// ---- backward Euler (backward_euler.F90:29-176) --------------------------------------------------
int newton_iteration(Zone &Z, const vector<double> &y_old, const vector<double> &y_cur, double dt,
                     double &grd, vector<double> &y_new) {
  const Net &N = *Z.N;
  calculate_jacobian(Z, dt, y_cur.data());
  for (double &j : Z.jac) j = j * (-dt);
  vector<double> val; vector<int> colind, rowptr;
  int nvar1;
  reduce_jacobian(Z, val, colind, rowptr, nvar1);
  Z.nvar1 = nvar1;
  calculate_dxdt(Z, y_cur.data());
  vector<double> rhs(N.nsp);
  for (int i = 0; i < N.nsp; ++i) rhs[i] = y_old[i] - y_cur[i] + dt * Z.dxdt[i];
  vector<double> rrhs, ry_cur;
  for (int i = 0; i < N.nsp; ++i)
    if (Z.mask[i]) { rrhs.push_back(rhs[i]); ry_cur.push_back(y_cur[i]); }
  int ierr = 0;
  if (nvar1 > 0) {
    int nnz = (int)val.size();
    g_slu_solve(nvar1, nnz, 1, 1, val.data(), colind.data(), rowptr.data(), rrhs.data(), &ierr);
  }
  Z.st.nfact++; Z.st.nsolve++;
  if (ierr != 0) return -1;  // the reference stops (linalg.F90:120-123)
  int icons = 0;
  for (int i = 0; i < N.nsp; ++i)
    if (Z.mask[i]) { y_new[i] = ry_cur[icons] + rrhs[icons]; ++icons; }
  grd = 0.0;
  for (int i = 0; i < N.nsp; ++i) {
    double g = 0.0;
    if (y_cur[i] > N.kn.grdthreshold) g = std::fabs((y_new[i] - y_cur[i]) / y_cur[i]);
    grd = std::max(grd, g);
  }
  return 0;
}

int backward_euler_newton(Zone &Z, int nvar, vector<double> &yps, double dt, double &dtrcmd) {
  const Net &N = *Z.N;
  const double rmin = 0.2, rmax = 2;
  const double dgrd = N.kn.dgrd;
  double sum_check = N.kn.grdthreshold * nvar * dgrd;
  vector<double> y_new = yps, y_old = yps, y_cur = yps;
  int iter = 0, ierr = 0;
  double grd = 0, err, tol;
  for (;;) {
    if (iter > N.kn.ittd) {
      if (maxval_neg(y_new) >= sum_check) {
        err = maxval_neg(y_new); tol = sum_check; ierr = NEG_ABUNDS;
      } else if (std::fabs(ONE - seqsum(y_new)) > SUM_TOL) {
        err = std::fabs(ONE - seqsum(y_new)); tol = SUM_TOL; ierr = SUM_X;
      } else {
        err = grd; tol = dgrd; ierr = SLV_CNVRG;
      }
      dtrcmd = std::max(std::min(std::pow(tol / std::max(err, SMALL), HALF), rmax), rmin) * dt;
      return ierr;
    }
    if (newton_iteration(Z, y_old, y_cur, dt, grd, y_new) != 0) return BAD_STEP;
    iter = iter + 1;
    Z.st.newton_iters++;
    if (grd <= dgrd && maxval_neg(y_new) < sum_check && std::fabs(ONE - seqsum(y_new)) <= SUM_TOL) {
      yps = y_new;
      dtrcmd = TWO * std::max(std::min(std::pow(dgrd / std::max(grd, SMALL), HALF), rmax), rmin) * dt;
      ypsplus(yps);
      return 0;
    }
    y_cur = y_new;
  }
}

// ---- Bader-Deuflhard (bader_deuflhard.F90:139-488) ----------------------------------------------
struct SluFactors {
  long long h = 0;
  bool live = false;
};

// Test infrastructure, off unless oracle_set_lu_permute was called: hand SuperLU the reduced system
// of every Bader-Deuflhard level under a seeded symmetric permutation P A P^T (and P b, the solution
// permuted back). The system is the same; only the elimination order, and so the rounding, changes.
// The spread of the checker's results under it is how far the reference's answer depends on the
// LU's rounding, which any other factorization changes.
static vector<int> lu_permutation(int n, int seed) {
  vector<int> p(n);
  for (int i = 0; i < n; ++i) p[i] = i;
  unsigned long long st = 0x9E3779B97F4A7C15ull * (unsigned long long)(seed + 1) + (unsigned long long)n;
  for (int i = n - 1; i > 0; --i) {  // Fisher-Yates with a 64-bit LCG
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    const int j = (int)((st >> 33) % (unsigned long long)(i + 1));
    std::swap(p[i], p[j]);
  }
  return p;
}

// CSC (1-based, as the shim takes it) of P A P^T: entry (i, j) moves to (p[i], p[j]).
static void permute_csc(int n, const vector<double> &val, const vector<int> &row, const vector<int> &col,
                        const vector<int> &p, vector<double> &pv, vector<int> &pr, vector<int> &pc) {
  vector<std::tuple<int, int, double>> e;
  for (int j = 0; j < n; ++j)
    for (int q = col[j] - 1; q < col[j + 1] - 1; ++q) e.emplace_back(p[j], p[row[q] - 1], val[q]);
  std::sort(e.begin(), e.end(), [](const auto &a, const auto &b) {
    return std::get<0>(a) != std::get<0>(b) ? std::get<0>(a) < std::get<0>(b) : std::get<1>(a) < std::get<1>(b);
  });
  pv.resize(e.size());
  pr.resize(e.size());
  pc.assign(n + 1, 0);
  for (size_t q = 0; q < e.size(); ++q) {
    pv[q] = std::get<2>(e[q]);
    pr[q] = std::get<1>(e[q]) + 1;
    pc[std::get<0>(e[q]) + 1]++;
  }
  for (int j = 0; j < n; ++j) pc[j + 1] += pc[j];
  for (int j = 0; j <= n; ++j) pc[j] += 1;
}

int bd_step(Zone &Z, vector<double> &y_k, vector<double> &delta_k, double h, int nvar1, int stage,
            const vector<double> &cval_in, vector<int> &crow_in, vector<int> &ccol_in, SluFactors &F) {
  const int pseed = Z.N->lu_permute;
  vector<int> perm;
  vector<double> pval;
  vector<int> prow, pcol;
  if (pseed >= 0 && nvar1 > 0) {
    perm = lu_permutation(nvar1, pseed);
    permute_csc(nvar1, cval_in, crow_in, ccol_in, perm, pval, prow, pcol);
  }
  const vector<double> &cval = perm.empty() ? cval_in : pval;
  vector<int> &crow = perm.empty() ? crow_in : prow;
  vector<int> &ccol = perm.empty() ? ccol_in : pcol;
  const Net &N = *Z.N;
  enum { FIRST = 1, MID = 2, LAST = 3 };
  int ierr = 0;
  vector<double> x(N.nsp, 0.0), rhs(N.nsp);
  calculate_dxdt(Z, y_k.data());
  if (stage == FIRST) for (int i = 0; i < N.nsp; ++i) rhs[i] = h * Z.dxdt[i];
  else for (int i = 0; i < N.nsp; ++i) rhs[i] = h * Z.dxdt[i] - delta_k[i];
  vector<double> rr;
  for (int i = 0; i < N.nsp; ++i) if (Z.mask[i]) rr.push_back(rhs[i]);
  int n = nvar1, nnz = (int)cval.size(), nrhs = 1, ldb = nvar1, info = 0, iopt;
  vector<double> vals = cval;  // dgssv reads values only
  if (n == 0) {  // empty dynamic network: nothing to solve
    rr.clear();
  } else if (stage == FIRST) {
    iopt = 1;
    g_dgssv(&iopt, &n, &nnz, &nrhs, vals.data(), crow.data(), ccol.data(), rr.data(), &ldb, &F.h, &info);
    F.live = true;
    Z.st.nfact++;
  }
  if (n > 0) {
    iopt = 2;
    if (!perm.empty()) {
      vector<double> t(n);
      for (int i = 0; i < n; ++i) t[perm[i]] = rr[i];
      rr = t;
    }
    g_dgssv(&iopt, &n, &nnz, &nrhs, vals.data(), crow.data(), ccol.data(), rr.data(), &ldb, &F.h, &info);
    if (!perm.empty()) {
      vector<double> t(n);
      for (int i = 0; i < n; ++i) t[i] = rr[perm[i]];
      rr = t;
    }
  }
  Z.st.nsolve++;
  int icons = 0;
  for (int i = 0; i < N.nsp; ++i)
    if (Z.mask[i]) x[i] = rr[icons++];
  if (stage == FIRST || stage == LAST) delta_k = x;
  else for (int i = 0; i < N.nsp; ++i) delta_k[i] = delta_k[i] + TWO * x[i];
  for (int i = 0; i < N.nsp; ++i) y_k[i] = y_k[i] + delta_k[i];
  if (stage == LAST && F.live) {
    iopt = 3;
    g_dgssv(&iopt, &n, &nnz, &nrhs, vals.data(), crow.data(), ccol.data(), rr.data(), &ldb, &F.h, &info);
    F.live = false;
  }
  bool huge = false;
  for (double y : y_k) if (y > TWO) huge = true;
  if (huge) {
    ierr = HUGE_ABUNDS;
    if (stage != LAST && F.live) {
      iopt = 3;
      g_dgssv(&iopt, &n, &nnz, &nrhs, vals.data(), crow.data(), ccol.data(), rr.data(), &ldb, &F.h, &info);
      F.live = false;
    }
  }
  return ierr;
}

int semi_implicit_extrapolation(Zone &Z, double time_step, int k, vector<double> &y_k, double &xest) {
  const Net &N = *Z.N;
  double h = time_step / (double)N.nseq[k];
  xest = powi(h / N.nseq[k], 2);
  for (int e = 0; e < N.nnz; ++e) Z.jac[e] = Z.jacval_cpy[e] * (-h);
  vector<double> val; vector<int> colind, rowptr;
  int nvar1;
  reduce_jacobian(Z, val, colind, rowptr, nvar1);
  Z.nvar1 = nvar1;
  vector<double> cval; vector<int> crow, ccol;
  csr_to_csc(nvar1, val, colind, rowptr, cval, crow, ccol);
  vector<double> delta_k(N.nsp, 0.0);
  SluFactors F;
  int ierr = bd_step(Z, y_k, delta_k, h, nvar1, 1, cval, crow, ccol, F);
  if (ierr) return ierr;
  for (int i = 1; i <= N.nseq[k] - 1; ++i) {
    ierr = bd_step(Z, y_k, delta_k, h, nvar1, 2, cval, crow, ccol, F);
    if (ierr) return ierr;
  }
  return bd_step(Z, y_k, delta_k, h, nvar1, 3, cval, crow, ccol, F);
}

void extrapolate(Zone &Z, int k, const vector<double> &yest, vector<double> &y_extrap, double xest) {
  const Net &N = *Z.N;
  const int n = N.nsp;
  double *qcol = Z.qc.data(), *yerr = Z.ye_rr.data();
  auto Q = [&](int i, int kk) -> double & { return qcol[(size_t)kk * n + i]; };
  auto E = [&](int i, int kk) -> double & { return yerr[(size_t)kk * n + i]; };
  Z.xhist[k] = xest;
  vector<double> yz = yest;
  for (int j = 0; j < n; ++j) E(j, k) = yest[j];
  if (k == 1) {
    for (int j = 0; j < n; ++j) Q(j, k) = yest[j];
    y_extrap = yest;
    return;
  }
  vector<double> d = yest;
  for (int k1 = 1; k1 <= k - 1; ++k1) {
    double delta = ONE / (Z.xhist[k - k1] - xest);
    double f1 = xest * delta, f2 = Z.xhist[k - k1] * delta;
    for (int j = 0; j < n; ++j) {
      double q = Q(j, k1);
      Q(j, k1) = E(j, k);
      double dl = d[j] - q;
      E(j, k) = f1 * dl;
      d[j] = f2 * dl;
      yz[j] = yz[j] + E(j, k);
    }
  }
  for (int j = 0; j < n; ++j) Q(j, k) = E(j, k);
  y_extrap = yz;
}

void compute_error(Zone &Z, int k, const vector<double> &y_k, const vector<double> &yscal) {
  const Net &N = *Z.N;
  const int n = N.nsp;
  double am = -1.7976931348623157e308;
  for (int i = 0; i < n; ++i)
    if (y_k[i] > 1e-27) am = std::max(am, std::fabs(Z.ye_rr[(size_t)k * n + i] / yscal[i]));
  Z.abuerr = am / N.kn.dgrd;
  double nm = -1.7976931348623157e308;
  for (int i = 0; i < n; ++i)
    if (y_k[i] < N.kn.grdthreshold) nm = std::max(nm, -y_k[i]);
  Z.negerr = nm / N.kn.grdthreshold;
  if (Z.abuerr < 1e-3) {
    Z.errmax = Z.abuerr;
  } else {
    Z.sumerr = std::fabs(ONE - sortedsum(y_k.data(), n)) / SUM_TOL;
    Z.errmax = std::max(Z.abuerr, Z.sumerr);
  }
  Z.errmax = std::max(Z.errmax, Z.negerr);
}

int bader_deuflhard_integration(Zone &Z, vector<double> &yps, double dt, double &dtrcmd, bool frst) {
  const Net &N = *Z.N;
  const double safe1 = FOURTH, safe2 = 0.7, redmin = 0.7, redmax = 1.e-5, scalmx = 0.25;
  int ierr = 0, km = -1, k;
  double scal = ONE, red = -ONE;
  vector<double> y_k = yps, y_extrap, yscal(N.nsp);
  calculate_jacobian(Z, dt, yps.data());
  Z.jacval_cpy = Z.jac;
  for (k = 1; k <= N.kmax; ++k) {
    y_k = yps;
    double xest;
    ierr = semi_implicit_extrapolation(Z, dt, k, y_k, xest);
    if (ierr != 0) {
      dtrcmd = dt * FIFTH;
      return ierr;
    }
    Z.st.newton_iters += N.nseq[k];
    extrapolate(Z, k, y_k, y_extrap, xest);
    y_k = y_extrap;
    bool nan = false;
    for (double y : y_k) if (y != y) nan = true;
    if (nan) {
      dtrcmd = dt * FIFTH;
      return GOT_NAN;
    }
    for (int i = 0; i < N.nsp; ++i) yscal[i] = std::max(std::fabs(y_k[i]), N.kn.grdthreshold);
    if (k != 1) {
      compute_error(Z, k, y_k, yscal);
      km = k - 1;
      Z.err[km] = std::pow(Z.errmax / safe1, ONE / (TWO * km + ONE));
    }
    if (k != 1 && (k >= Z.kopt - 1 || frst)) {
      if (Z.errmax <= ONE) {
        Z.reduce = false;
        break;
      } else {
        if (k == N.kmax || k == Z.kopt + 1) {
          Z.reduce = true; red = safe2 / Z.err[km];
        } else if (k == Z.kopt) {
          if (N.alf[Z.kopt - 1][Z.kopt] < Z.err[km]) { Z.reduce = true; red = safe2 / Z.err[km]; }
        } else if (Z.kopt == N.kmax) {
          if (N.alf[km][N.kmax - 1] < Z.err[km]) { Z.reduce = true; red = N.alf[km][N.kmax - 1] * safe2 / Z.err[km]; }
        } else if (N.alf[km][Z.kopt] < Z.err[km]) {
          Z.reduce = true; red = N.alf[km][Z.kopt - 1] / Z.err[km];
        }
      }
    }
  }
  if (k > N.kmax) k = N.kmax + 1;  // Fortran DO leaves k = kmax+1 after normal completion
  if (Z.reduce) {
    red = std::max(redmax, std::min(red, redmin));
    dtrcmd = dt * red;
    if (Z.negerr > Z.sumerr && Z.negerr > Z.abuerr) ierr = NEG_ABUNDS;
    else if (Z.sumerr > Z.abuerr) ierr = SUM_X;
    else ierr = SLV_CNVRG;
  } else {
    double workmin = 1.e35, fct, work;
    for (int kk = 1; kk <= km; ++kk) {
      fct = std::max(Z.err[kk], scalmx);
      work = fct * N.a[kk + 1];
      if (work < workmin) { scal = fct; workmin = work; Z.kopt = kk + 1; }
    }
    dtrcmd = TWO * dt / scal;
    if (Z.kopt >= k && Z.kopt != N.kmax) {
      fct = std::max(scal / N.alf[Z.kopt - 1][Z.kopt], scalmx);
      if (N.a[Z.kopt + 1] * fct <= workmin) {
        dtrcmd = dtrcmd * scal / fct;
        Z.kopt = Z.kopt + 1;
      }
    }
  }
  yps = y_k;
  return ierr;
}

double calculate_ye(const Net &N, const double *x) {  // utils.F90:537-553
  vector<double> eta(N.nsp, 0.0);
  for (int i = 0; i < N.nsp; ++i)
    if (N.ciso[i]) eta[i] = (N.an[i] - 2.0 * N.zn[i]) * x[i] / N.an[i];
  return (1.0 - sortedsum(eta.data(), N.nsp)) * 0.5;
}

// ---- NSE (physics/source/nse_swj.F90:272-625, solver/source/nse_solver.F90:33-291) ------------
const double twopi = 2.0 * pi, FIVE_THIRDS = 5.0 * THIRD, SIX_FIFTHS = 6.0 * FIFTH;
const double ye_tol = 1.e-5;  // solver_knobs.F90:13

void nse_coulomb(Zone &Z, double t9, double rho, double ye) {  // coulomb_corrections, nse_swj.F90:545-580
  const Net &N = *Z.N;
  const double a1 = -0.9052, a2 = 0.6322, a3 = -HALF * std::sqrt(THREE) - a1 / std::sqrt(a2);
  const double kT_erg = boltzmann * t9 * 1.e9, kT_mev = kT_erg * erg2mev;
  const double ae = std::pow(FOUR * pi * rho * ye * avogadro / THREE, -THIRD);
  const double Gam_e = qe * qe / kT_erg / ae;
  for (size_t j = 0; j < N.nse_idx.size(); ++j) {
    const double G = Gam_e * std::pow(N.zn[N.nse_idx[j]], FIVE_THIRDS);
    double mc = a1 * (std::sqrt(G * (a2 + G)) - a2 * std::log(std::sqrt(G / a2) + std::sqrt(ONE + G / a2))) +
                TWO * a3 * (std::sqrt(G) - std::atan(std::sqrt(G)));
    Z.nse_mucoul[j] = mc * kT_mev;
  }
  Z.mu_p_coul = Z.nse_mucoul[N.nse_iprot];
}

void nse_partition(Zone &Z, double t9) {  // partition_functions, nse_swj.F90:585-597
  const Net &N = *Z.N;
  reaclib_partition(Z, t9);
  for (size_t j = 0; j < N.nse_idx.size(); ++j) {
    const int i = N.nse_idx[j];
    Z.nse_gtot[j] = (N.spart[i] >= 0 ? Z.partinter[N.spart[i]] : ONE) * N.ppn_g[i];
  }
}

void nse_distribution(Zone &Z, double mu_p, double mu_n, double t9, double rho, double *out) {  // :524-541
  const Net &N = *Z.N;
  const double kT_erg = boltzmann * t9 * 1.e9, kT_mev = kT_erg * erg2mev;
  for (size_t j = 0; j < N.nse_idx.size(); ++j) {
    const int i = N.nse_idx[j];
    const double m = N.ppn_m[i], z = N.zn[i], n = N.an[i] - N.zn[i];
    const double lam = std::sqrt(planck_erg * planck_erg / (twopi * m * kT_erg));
    const double fac = z * (mu_p + Z.mu_p_coul) + n * mu_n - Z.nse_mucoul[j] + N.ppn_q[i];
    const double pre = m / rho * Z.nse_gtot[j] / (lam * lam * lam);
    out[j] = pre * std::exp(fac / kT_mev);
  }
}

void nse_rhs(Zone &Z, double ye) {  // calculate_rhs, nse_swj.F90:510-520
  const Net &N = *Z.N;
  const int n = (int)N.nse_idx.size();
  vector<double> zx(n);
  for (int j = 0; j < n; ++j) zx[j] = (N.zn[N.nse_idx[j]] / N.an[N.nse_idx[j]]) * Z.nse_x[j];
  Z.nse_the = sortedsum(Z.nse_x.data(), n) - ONE;
  Z.nse_phi = sortedsum(zx.data(), n) - ye;
}

void nse_jac(Zone &Z, double t9, double jac[2][2]) {  // calculate_jac, nse_swj.F90:483-506
  const Net &N = *Z.N;
  const int n = (int)N.nse_idx.size();
  const double kT_mev = boltzmann * t9 * 1.e9 * erg2mev;
  vector<double> dp(n), dn(n), zp(n), zn(n);
  for (int j = 0; j < n; ++j) {
    const int i = N.nse_idx[j];
    const double zoa = N.zn[i] / N.an[i];
    dp[j] = Z.nse_x[j] * N.zn[i] / kT_mev;
    dn[j] = Z.nse_x[j] * (N.an[i] - N.zn[i]) / kT_mev;
    zp[j] = zoa * dp[j];
    zn[j] = zoa * dn[j];
  }
  jac[0][0] = sortedsum(dp.data(), n); jac[0][1] = sortedsum(dn.data(), n);
  jac[1][0] = sortedsum(zp.data(), n); jac[1][1] = sortedsum(zn.data(), n);
}

// Crout LU with implicit partial pivoting, and its back substitution, for the 2x2 NSE Jacobian
// (ludcmp_nse / lubksb_nse, nse_swj.F90:751-883). Returns false for a zero row.
bool nse_lu2(double a[2][2], int indx[2]) {
  const int n = 2;
  double vv[2];
  for (int i = 0; i < n; ++i) {
    double aamax = 0.0;
    for (int j = 0; j < n; ++j) aamax = std::max(aamax, std::fabs(a[i][j]));
    if (aamax == ZERO) return false;
    vv[i] = 1.0 / aamax;
  }
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) {
      double sum = a[i][j];
      for (int k = 0; k < i; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
    }
    double aamax = 0.0;
    int imax = j;
    for (int i = j; i < n; ++i) {
      double sum = a[i][j];
      for (int k = 0; k < j; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
      const double dum = vv[i] * std::fabs(sum);
      if (dum >= aamax) { imax = i; aamax = dum; }
    }
    if (j != imax) {
      for (int k = 0; k < n; ++k) std::swap(a[imax][k], a[j][k]);
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (a[j][j] == ZERO) a[j][j] = 1.0e-20;
    if (j != n - 1) {
      const double dum = 1.0 / a[j][j];
      for (int i = j + 1; i < n; ++i) a[i][j] = a[i][j] * dum;
    }
  }
  return true;
}

void nse_lub2(const double a[2][2], const int indx[2], double b[2]) {
  const int n = 2;
  int ii = -1;
  for (int i = 0; i < n; ++i) {
    const int ll = indx[i];
    double sum = b[ll];
    b[ll] = b[i];
    if (ii >= 0) {
      for (int j = ii; j < i; ++j) sum = sum - a[i][j] * b[j];
    } else if (sum != ZERO) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = n - 1; i >= 0; --i) {
    double sum = b[i];
    for (int j = i + 1; j < n; ++j) sum = sum - a[i][j] * b[j];
    b[i] = sum / a[i][i];
  }
}

// solve_nse (nse_swj.F90:388-460): Newton on (theta, phi) in (mu_p, mu_n) with a x1e-2 line search.
int solve_nse(Zone &Z, double t9, double rho, double ye, double &mu_p, double &mu_n, int &it, int max_iter) {
  const int lnsrchmax = 100;
  Z.nse_mu[0] = mu_p;
  Z.nse_mu[1] = mu_n;
  for (int i = 1; i <= max_iter; ++i) {
    it = i;
    const double mu_old[2] = {Z.nse_mu[0], Z.nse_mu[1]};
    nse_rhs(Z, ye);
    const double the_old = Z.nse_the, phi_old = Z.nse_phi;
    double jac[2][2];
    nse_jac(Z, t9, jac);
    int indx[2];
    if (!nse_lu2(jac, indx)) return BAD_STEP;
    double del[2] = {Z.nse_the, Z.nse_phi};
    nse_lub2(jac, indx, del);
    double gamma = ONE;
    for (int j = 1; j <= lnsrchmax; ++j) {
      if (j == lnsrchmax) return NSE_CNVRG;
      Z.nse_mu[0] = mu_old[0] - gamma * del[0];
      Z.nse_mu[1] = mu_old[1] - gamma * del[1];
      nse_distribution(Z, Z.nse_mu[0], Z.nse_mu[1], t9, rho, Z.nse_x.data());
      nse_rhs(Z, ye);
      if (std::fabs(Z.nse_the) > 1.e10 * std::fabs(the_old) + 1.e-10 ||
          std::fabs(Z.nse_phi) > 1.e10 * std::fabs(phi_old) + 1.e-10)
        gamma = gamma * 1.e-2;
      else
        break;
    }
    if (std::fabs(Z.nse_the) <= 1.e-9 && std::fabs(Z.nse_phi) <= 1.e-9) break;
    if (i == max_iter) return NSE_CNVRG;
  }
  mu_p = Z.nse_mu[0];
  mu_n = Z.nse_mu[1];
  return 0;
}

// initial_guess with ni56_initial (nse_swj.F90:466-478): X(Ni56) = 1 and mu_p = mu_n, or the last
// converged solution.
void nse_initial_guess(Zone &Z, double &mu_p, double &mu_n, double t9, double rho) {
  const Net &N = *Z.N;
  if (!Z.nse_first) {
    Z.nse_mu[0] = Z.nse_mu_last[0]; Z.nse_mu[1] = Z.nse_mu_last[1];
    mu_p = Z.nse_mu[0]; mu_n = Z.nse_mu[1];
    return;
  }
  const double kT_erg = boltzmann * t9 * 1.e9, kT_mev = kT_erg * erg2mev;
  const int j = N.nse_ini56, i = N.nse_idx[j];
  const double lam = std::sqrt(planck_erg * planck_erg / (twopi * N.ppn_m[i] * kT_erg));
  mu_p = kT_mev * std::log(ONE * rho * powi(lam, 3) / Z.nse_gtot[j] / N.ppn_m[i]) - N.ppn_q[i] + Z.nse_mucoul[j] -
         N.zn[i] * Z.mu_p_coul;
  mu_p = mu_p / N.an[i];
  mu_n = mu_p;
}

// compute_nse (nse_swj.F90:272-384). The reference stops the run when the temperature descent also
// fails; here the failure comes back as the error code.
int compute_nse(Zone &Z, double t9in, double rho, double ye, double *yps, double &mu_p, double &mu_n, int &iter) {
  const Net &N = *Z.N;
  const int nn = (int)N.nse_idx.size();
  if (ye <= ZERO || ye >= ONE) return BAD_YE;
  mu_n = ZERO; mu_p = ZERO; iter = 0;
  for (int i = 0; i < N.nsp; ++i) yps[i] = ZERO;
  int it = 0;
  double t9 = t9in;
  auto finish = [&]() {
    nse_distribution(Z, mu_p, mu_n, t9, rho, Z.nse_x.data());
    for (int i = 0; i < N.nsp; ++i) yps[i] = 1.e-99;
    for (int j = 0; j < nn; ++j) yps[N.nse_idx[j]] = std::max(Z.nse_x[j], 1e-99);
    Z.nse_mu_last[0] = Z.nse_mu[0]; Z.nse_mu_last[1] = Z.nse_mu[1];
    Z.nse_first = false;
    return 0;
  };
  nse_coulomb(Z, t9, rho, ye);
  nse_partition(Z, t9);
  nse_initial_guess(Z, mu_p, mu_n, t9, rho);
  nse_distribution(Z, mu_p, mu_n, t9, rho, Z.nse_x.data());
  int ierr = solve_nse(Z, t9, rho, ye, mu_p, mu_n, it, 100);
  iter += it;
  if (ierr == 0) return finish();
  // temperature descent from T9 = 100
  const int tsteps = 10;
  const double coeff = std::pow(100.0 / t9in, ONE / ((double)tsteps - ONE));
  for (int i = 1; i <= tsteps; ++i) {
    t9 = t9in * powi(coeff, tsteps - i);
    nse_coulomb(Z, t9, rho, ye);
    nse_partition(Z, t9);
    if (i == 1) nse_initial_guess(Z, mu_p, mu_n, t9, rho);
    nse_distribution(Z, mu_p, mu_n, t9, rho, Z.nse_x.data());
    ierr = solve_nse(Z, t9, rho, ye, mu_p, mu_n, it, 500);
    iter += it;
  }
  if (ierr == 0) return finish();
  return ierr == BAD_STEP ? BAD_STEP : NSE_CNVRG;
}

// nse_solver_cache_lm_ov_a (nse_solver.F90:33-66): keep only the weak rates, and per parent
// (lambda_beta - lambda_ec) / A.
void nse_cache_lm_ov_a(Zone &Z) {
  const Net &N = *Z.N;
  for (int l = 0; l < N.nre; ++l) {
    const int lab = N.ilabb[l];
    if (!(lab == i_bm || lab == i_ec || lab == i_ve || lab == i_vp)) Z.v[l] = ZERO;
  }
  for (double &x : Z.lm_ov_a) x = ZERO;
  for (int l = 0; l < N.nre; ++l) {
    if (!N.crea[l] || Z.v[l] == ZERO) continue;
    const int par = N.k[(size_t)l * 8 + 0], dau = N.k[(size_t)l * 8 + 6];
    const double lm = Z.v[l], a = N.an[par];
    if (N.zn[par] < N.zn[dau]) Z.lm_ov_a[par] = Z.lm_ov_a[par] + lm / a;
    else Z.lm_ov_a[par] = Z.lm_ov_a[par] - lm / a;
  }
}

// yedot (nse_solver.F90:104-113): sortedsum(x * lm_ov_a, mask = considerisotope). The reference's
// sortedsum applies the mask by sorted position (utils.F90:489-495), restated as is.
double nse_yedot(const Zone &Z, const double *x) {
  const Net &N = *Z.N;
  vector<double> t(N.nsp);
  for (int i = 0; i < N.nsp; ++i) t[i] = x[i] * Z.lm_ov_a[i];
  vector<int> idx;
  indexx(N.nsp, t.data(), idx);
  double s = 0.0;
  for (int i = 1; i <= N.nsp; ++i)
    if (N.ciso[i - 1]) s = s + t[idx[i] - 1];
  return s;
}

// rk4_nse_step (nse_solver.F90:116-238): Cash-Karp Runge-Kutta for Ye in NSE.
int rk4_nse_step(Zone &Z, double dt, double rho, double t9, double &ye, vector<double> &y1, double &error) {
  const double b21 = FIFTH, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0, b41 = 3.0 / 10.0, b42 = -9.0 / 10.0, b43 = SIX_FIFTHS,
               b51 = -11.0 / 54.0, b52 = 5.0 * HALF, b53 = -70.0 / 27.0, b54 = 35.0 / 27.0, b61 = 1631.0 / 55296.0,
               b62 = 175.0 / 512.0, b63 = 575.0 / 13824.0, b64 = 44275.0 / 110592.0, b65 = 253.0 / 4096.0,
               c1 = 37.0 / 378.0, c1s = 2825.0 / 27648.0, c2 = ZERO, c2s = ZERO, c3 = 250.0 / 621.0,
               c3s = 18575.0 / 48384.0, c4 = 125.0 / 594.0, c4s = 13525.0 / 55296.0, c5 = ZERO,
               c5s = 277.0 / 14336.0, c6 = 512.0 / 1771.0, c6s = FOURTH;
  double mu_p, mu_n;
  int iters, ierr;
  const double ye_0 = ye;
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  const double k1 = dt * nse_yedot(Z, y1.data());
  ye = ye_0 + (b21 * k1);
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  const double k2 = dt * nse_yedot(Z, y1.data());
  ye = ye_0 + (b31 * k1 + b32 * k2);
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  const double k3 = dt * nse_yedot(Z, y1.data());
  ye = ye_0 + (b41 * k1 + b42 * k2 + b43 * k3);
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  const double k4 = dt * nse_yedot(Z, y1.data());
  ye = ye_0 + (b51 * k1 + b52 * k2 + b53 * k3 + b54 * k4);
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  const double k5 = dt * nse_yedot(Z, y1.data());
  ye = ye_0 + (b61 * k1 + b62 * k2 + b63 * k3 + b64 * k4 + b65 * k5);
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  const double k6 = dt * nse_yedot(Z, y1.data());
  const double ye_5th = ye_0 + c1 * k1 + c2 * k2 + c3 * k3 + c4 * k4 + c5 * k5 + c6 * k6;
  const double ye_4th = ye_0 + c1s * k1 + c2s * k2 + c3s * k3 + c4s * k4 + c5s * k5 + c6s * k6;
  ye = ye_5th;
  if ((ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters)) != 0) return ierr;
  error = std::fabs(ye_5th - ye_4th);
  return 0;
}

// nse_yedot_rk4 (nse_solver.F90:72-101)
int nse_yedot_rk4(Zone &Z, vector<double> &yps, double t9, double rho, double &ye, double dt, double &dtrcmd) {
  const double maxfac = 2.0, minfac = 0.1;
  const double ye_old = ye;
  vector<double> y1 = yps;
  double error = 0.0, fac;
  int ierr = rk4_nse_step(Z, dt, rho, t9, ye, y1, error);
  if (ierr != 0) error = ye_old;
  if (ierr != 0 || ye < ZERO || ye > ONE) {
    ierr = BAD_YE;
    fac = HALF * std::pow(std::fabs(ye_tol * ye_old / std::max(error, SMALL)), FIFTH);
  } else if (error / ye > ye_tol) {
    ierr = NSE_WEAK;
    fac = HALF * std::pow(std::fabs(ye_tol * ye / std::max(error, SMALL)), FIFTH);
  } else {
    ierr = 0;
    fac = std::pow(std::fabs(ye_tol * ye / std::max(error, SMALL)), FIFTH);
    yps = y1;
  }
  dtrcmd = dt * std::max(std::min(fac, maxfac), minfac);
  return ierr;
}

// nse_yedot_euler (nse_solver.F90:241-289)
int nse_yedot_euler(Zone &Z, vector<double> &yps, double t9, double rho, double &ye, double dt, double &dtrcmd) {
  const double deltamax = 1.e-5;
  vector<double> y1(yps.size());
  double mu_p, mu_n;
  int iters;
  int ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters);
  if (ierr != 0 || ye < ZERO || ye > ONE) {
    dtrcmd = 0.1 * dt;
    return BAD_STEP;
  }
  const double dyedt = nse_yedot(Z, y1.data());
  const double d_ye = dyedt * dt;
  if (d_ye > deltamax) {
    dtrcmd = deltamax / std::fabs(dyedt);
    return NSE_WEAK;
  }
  ye = ye + d_ye;
  ierr = compute_nse(Z, t9, rho, ye, y1.data(), mu_p, mu_n, iters);
  if (ierr == 0) yps = y1;
  else ierr = NSE_CNVRG;
  dtrcmd = deltamax / std::fabs(dyedt);
  return ierr;
}

double interp2(double x0, double x1, double y0, double y1, double xw) {  // interp.F90:29-50
  double xwant = std::max(xw, x0);
  xwant = std::min(xwant, x1);
  return y0 + (y1 - y0) * (xwant - x0) / (x1 - x0);
}

// integrate_network (solver.F90:53-238) for one zone
int integrate_zone(Zone &Z, double *yps_io, double t9_0, double t9_1, double rho_0, double rho_1,
                   double &ye, double dtwant, int32_t *bd_state) {
  const Net &N = *Z.N;
  const int nsp = N.nsp;
  const nuppn_knobs &kn = N.kn;
  int nvar = 0;
  for (int i = 0; i < nsp; ++i) nvar += N.ciso[i] ? 1 : 0;
  bool frst = true;
  if (bd_state && *bd_state > 0) { frst = false; Z.kopt = *bd_state; }
  vector<double> yps(yps_io, yps_io + nsp), yps_old = yps;
  double ye_old = ye, dtdone = ZERO, dtrcmd = ZERO, dttry = dtwant;
  double my_t9_last = HALF * (t9_0 + t9_1), my_rho_last = HALF * (rho_0 + rho_1);
  // the frame's evaluate_all_rates right before the call (ppn.F90:298, mppnp.F90:719)
  evaluate_all_rates(Z, ye, my_rho_last, my_t9_last, yps.data());
  int ierr = 0;
  int i;
  for (i = 1; i <= kn.max_sub_steps; ++i) {
    if (i > 1) frst = false;
    double my_t9_0 = 0, my_t9_1 = 0, my_t9, my_rho_0 = 0, my_rho_1 = 0, my_rho;
    double t_0 = dtdone, t_1 = std::min(dtdone + dttry, dtwant);
    if (kn.interpolate_temp) {
      my_t9_0 = interp2(ZERO, dtwant, t9_0, t9_1, t_0);
      my_t9_1 = interp2(ZERO, dtwant, t9_0, t9_1, t_1);
      my_t9 = HALF * (my_t9_0 + my_t9_1);
    } else {
      my_t9 = HALF * (t9_0 + t9_1);
    }
    if (kn.interpolate_dens) {
      my_rho_0 = interp2(ZERO, dtwant, rho_0, rho_1, t_0);
      my_rho_1 = interp2(ZERO, dtwant, rho_0, rho_1, t_1);
      my_rho = HALF * (my_rho_0 + my_rho_1);
    } else {
      my_rho = HALF * (rho_0 + rho_1);
    }
    double diff = std::fabs(my_t9_0 - my_t9_1) / my_t9_0;
    diff = std::max(diff, std::fabs(my_rho_0 - my_rho_1) / my_rho_0);
    if (diff > kn.delta_state_max && t9_0 > kn.min_t9_for_slv && t9_1 > kn.min_t9_for_slv) {
      dttry = HALF * dttry;
      continue;
    }
    if (my_t9 != my_t9_last || my_rho != my_rho_last) {
      evaluate_all_rates(Z, ye, my_rho, my_t9, yps.data());
      my_rho_last = my_rho; my_t9_last = my_t9;
    }
    // NSE above nse_min_t9 (solver.F90:153-158, do_one_time_step :260-266)
    const bool do_nse = kn.i_nse == 1 && my_t9 >= kn.nse_min_t9;
    if (do_nse) nse_cache_lm_ov_a(Z);
    ierr = 0;
    if (my_t9 >= kn.min_t9_for_slv) {
      if (do_nse) {
        if (kn.nse_weak_method == 0) ierr = nse_yedot_euler(Z, yps, my_t9, my_rho, ye, dttry, dtrcmd);
        else ierr = nse_yedot_rk4(Z, yps, my_t9, my_rho, ye, dttry, dtrcmd);
      } else {
        if (kn.integration_method == 0) ierr = backward_euler_newton(Z, nvar, yps, dttry, dtrcmd);
        else ierr = bader_deuflhard_integration(Z, yps, dttry, dtrcmd, frst);
        ye = calculate_ye(N, yps.data());
      }
      if (dttry < SMALL) {
        std::copy(yps.begin(), yps.end(), yps_io);
        if (bd_state) *bd_state = Z.kopt;
        return SMALL_DT;
      }
    } else {
      ierr = 0;
    }
    if (ierr == 0) {
      dtdone = dtdone + dttry;
      for (double &y : yps) y = std::max(y, 1.e-99);
      yps_old = yps;
      ye_old = ye;
      Z.st.nsucc++;
      if (dtdone >= dtwant) break;
    } else {
      yps = yps_old;
      ye = ye_old;
      Z.st.nfail++;
    }
    dttry = std::min(dtrcmd, dtwant - dtdone);
    if (i == kn.max_sub_steps) {
      std::copy(yps.begin(), yps.end(), yps_io);
      if (bd_state) *bd_state = Z.kopt;
      return MAX_SUBSTEPS;
    }
  }
  if (kn.integration_method == 1) {
    double s = seqsum(yps);
    for (double &y : yps) y = y / s;
  }
  for (double &y : yps) y = std::max(y, 1.e-99);
  std::copy(yps.begin(), yps.end(), yps_io);
  Z.st.nvar1_last = Z.nvar1;
  if (bd_state) *bd_state = Z.kopt;
  return 0;
}

}  // namespace

// ---- C API --------------------------------------------------------------------------------------
extern "C" {

int oracle_load_superlu(const char *path) {
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  g_slu_solve = (slu_solve_t)dlsym(h, "slu_solve");
  g_dgssv = (dgssv_t)dlsym(h, "c_fortran_dgssv_");
  return (g_slu_solve && g_dgssv) ? 0 : -2;
}

void *oracle_net_create(const nuppn_net_desc *d, const nuppn_knobs *kn) {
  Net *N = new Net();
  N->kn = *kn;
  N->nsp = d->nsp; N->nre = d->nre; N->ig = d->igamma;
  N->an = cp(d->anetw, d->nsp); N->zn = cp(d->znetw, d->nsp);
  N->ciso = cp(d->considerisotope, d->nsp);
  N->exmass = cp(d->exmass, d->nsp); N->gspin = cp(d->gspin, d->nsp);
  N->spart = cp(d->spec_part, d->nsp);
  N->k = cp(d->k, (size_t)d->nre * 8);
  N->ilabb = cp(d->ilabb, d->nre); N->crea = cp(d->considerreaction, d->nre);
  N->rfac = cp(d->rfac, d->nre); N->src = cp(d->src, d->nre); N->sidx = cp(d->src_idx, d->nre);
  N->irev = cp(d->irev, d->nre);
  N->rev_target.assign(d->nre, 0);
  for (int i = 0; i < d->nre; ++i)
    if (N->crea[i] && N->irev[i] >= 0) N->rev_target[N->irev[i]] = 1;
  N->nc = d->rl_ncontrib; N->nr = d->rl_nrate;
  N->rla = cp(d->rl_a, (size_t)N->nc * 7); N->rlrate = cp(d->rl_rate, N->nc);
  N->rlchap = cp(d->rl_chapter, N->nr); N->rlv = cp(d->rl_vflag, N->nr);
  N->rlec = cp(d->rl_ecflag, N->nr); N->rlnireac = cp(d->rl_nireac, N->nr);
  N->rlpart = cp(d->rl_part, (size_t)N->nr * 6);
  N->npart = d->npart; N->pt9 = cp(d->part_t9, 24); N->pval = cp(d->part_val, (size_t)d->npart * 24);
  N->nv = d->vt_nrate; N->vfirst = cp(d->vt_first, N->nv + 1);
  N->vterms = cp(d->vt_terms, (size_t)d->vt_nterm * 5); N->vdpow = cp(d->vt_dpow, N->nv);
  N->vxfac = cp(d->vt_xfac, N->nv);
  N->vform = d->vt_form ? cp(d->vt_form, N->nv) : vector<int>(N->nv, 0);
  N->ngk = d->ng_kgrid; N->ngn = d->ng_nreac; N->ngd = d->ng_ndmax;
  N->ngt8 = cp(d->ng_t8, N->ngk); N->ngflag = cp(d->ng_flag, N->ngn);
  N->ngndata = cp(d->ng_ndata, N->ngn); N->ngane = cp(d->ng_ane, (size_t)N->ngn * N->ngd);
  N->ngl10v = cp(d->ng_l10v, (size_t)N->ngk * N->ngn * N->ngd);
  N->ngl10t8.resize(N->ngk);
  for (int i = 0; i < N->ngk; ++i) N->ngl10t8[i] = std::log10(N->ngt8[i]);
  N->ffv = d->ff_nv; N->fft = d->ff_nt; N->ffr = d->ff_nr;
  N->fft9 = cp(d->ff_t9coo, N->fft); N->ffrho = cp(d->ff_rhocoo, N->ffr);
  N->ffl10v = cp(d->ff_l10v, (size_t)N->ffv * N->fft * N->ffr);
  N->kdn = d->kd_n; N->kde = d->kd_ne; N->kdE = cp(d->kd_e, N->kde);
  N->kdrate = cp(d->kd_rate, (size_t)N->kdn * N->kde);
  N->kdak.resize(N->kdn);
  for (int i = 0; i < N->kdn; ++i) akima_setup(N->kde, N->kdE.data(), &N->kdrate[(size_t)i * N->kde], N->kdak[i]);
  N->constr = cp(d->const_rate, d->nconst);
  // nuclear data (nse_swj.F90:186-196)
  N->ppn_m.assign(N->nsp, 0.0); N->ppn_q.assign(N->nsp, 0.0); N->ppn_g.assign(N->nsp, 0.0);
  for (int i = 0; i < N->nsp; ++i) {
    if (i == N->ig) continue;
    double z = N->zn[i], n = N->an[i] - N->zn[i];
    N->ppn_g[i] = N->gspin[i];
    N->ppn_m[i] = N->exmass[i] * mev2erg / clight2 + N->an[i] * amu;
    N->ppn_m[i] = N->ppn_m[i] - z * me_g;
    N->ppn_q[i] = z * mp_mev + n * mn_mev - N->ppn_m[i] * clight2 * erg2mev;
    if (N->an[i] == 1.0 && (z == 0.0 || z == 1.0)) N->ppn_q[i] = ZERO;  // NEUT, PROT
  }
  N->ihe4 = N->ibe8 = -1;
  for (int i = 0; i < N->nsp; ++i) {
    if (N->zn[i] == 2 && N->an[i] == 4) N->ihe4 = i;
    if (N->zn[i] == 4 && N->an[i] == 8) N->ibe8 = i;
  }
  for (int i = 0; i < N->nsp; ++i)
    if (N->ciso[i] && N->an[i] != 0.0 && N->ppn_g[i] != 0.0 && N->ppn_m[i] != 0.0) {
      const int j = (int)N->nse_idx.size();
      N->nse_idx.push_back(i);
      if (N->zn[i] == 28 && N->an[i] == 56) N->nse_ini56 = j;
      if (N->zn[i] == 1 && N->an[i] == 1) N->nse_iprot = j;
      if (N->zn[i] == 0 && N->an[i] == 1) N->nse_ineut = j;
    }
  makemap(*N);
  bd_init(*N);
  return N;
}

void oracle_net_destroy(void *net) { delete (Net *)net; }
int oracle_nnz(void *net) { return ((Net *)net)->nnz; }

int oracle_jac_pattern(void *net, int32_t *row, int32_t *col, int32_t *map) {
  Net &N = *(Net *)net;
  for (int e = 0; e < N.nnz; ++e) { row[e] = N.jrow[e]; col[e] = N.jcol[e]; }
  for (size_t i = 0; i < N.dmap.size(); ++i) map[i] = N.dmap[i];
  return 0;
}

int oracle_eval_rates(void *net, double t9, double rho, double ye, const double *X, double *v) {
  Zone Z((Net *)net);
  evaluate_all_rates(Z, ye, rho, t9, X);
  std::copy(Z.v.begin(), Z.v.end(), v);
  return 0;
}

int oracle_dxdt(void *net, const double *v, const double *X, double *dxdt) {
  Zone Z((Net *)net);
  std::copy(v, v + Z.N->nre, Z.v.begin());
  calculate_dxdt(Z, X);
  std::copy(Z.dxdt.begin(), Z.dxdt.end(), dxdt);
  return 0;
}

int oracle_jacobian(void *net, const double *v, const double *X, double dt, double *jac,
                    uint8_t *entry_set, uint8_t *mask) {
  Zone Z((Net *)net);
  std::copy(v, v + Z.N->nre, Z.v.begin());
  calculate_jacobian(Z, dt, X);
  std::copy(Z.jac.begin(), Z.jac.end(), jac);
  for (int e = 0; e < Z.N->nnz; ++e) entry_set[e] = Z.jrow_flag[e] != -1;
  std::copy(Z.mask.begin(), Z.mask.end(), mask);
  return 0;
}

int oracle_solve_reduced(void *net, const double *jac, const uint8_t *entry_set, const uint8_t *mask,
                         double dt, const double *b, double *x) {
  Zone Z((Net *)net);
  const Net &N = *Z.N;
  for (int e = 0; e < N.nnz; ++e) {
    Z.jac[e] = jac[e] * (-dt);
    Z.jrow_flag[e] = entry_set[e] ? N.jrow[e] : -1;
  }
  std::copy(mask, mask + N.nsp, Z.mask.begin());
  vector<double> val; vector<int> colind, rowptr;
  int nvar1;
  reduce_jacobian(Z, val, colind, rowptr, nvar1);
  vector<double> rr;
  for (int i = 0; i < N.nsp; ++i) if (Z.mask[i]) rr.push_back(b[i]);
  int ierr = 0;
  if (nvar1 > 0) g_slu_solve(nvar1, (int)val.size(), 1, 1, val.data(), colind.data(), rowptr.data(), rr.data(), &ierr);
  int c = 0;
  for (int i = 0; i < N.nsp; ++i) x[i] = Z.mask[i] ? rr[c++] : 0.0;
  return ierr;
}

int oracle_integrate(void *net, int32_t nz, double *X, int32_t ldx, const double *t9_0,
                     const double *t9_1, const double *rho_0, const double *rho_1, double *ye,
                     const double *dtwant, int32_t *ierr, nuppn_zone_stats *stats, int32_t *bd_state,
                     int32_t nthreads) {
  Net *N = (Net *)net;
  if (!g_slu_solve) return -1;
  std::atomic<int> next(0);
  auto worker = [&]() {
    for (;;) {
      int z = next.fetch_add(1);
      if (z >= nz) break;
      Zone Zn(N);
      if (N->rhs_noise >= 0) Zn.noise = noise_state(N->rhs_noise, z);
      double yez = ye[z];
      ierr[z] = integrate_zone(Zn, X + (size_t)z * ldx, t9_0[z], t9_1[z], rho_0[z], rho_1[z], yez, dtwant[z],
                               bd_state ? bd_state + z : nullptr);
      ye[z] = yez;
      if (stats) stats[z] = Zn.st;
    }
  };
  int nt = std::max(1, (int)nthreads);
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(worker);
  worker();
  for (auto &t : th) t.join();
  return 0;
}

double oracle_calculate_ye(void *net, const double *X) { return calculate_ye(*(Net *)net, X); }

// The trajectory loop of tppnp (frames/tppnp/source/tppnp.F90:131-168) per zone.
int oracle_integrate_trajectories(void *net, int32_t nz, int32_t npts, double *X, int32_t ldx, const double *time,
                                  const double *t9, const double *rho, double *ye, int32_t *ierr, int32_t *fail,
                                  nuppn_zone_stats *stats, int32_t nthreads) {
  Net *N = (Net *)net;
  if (!g_slu_solve) return -1;
  auto ksum = [](const double *a, int n) {  // utils.F90:670-685
    double c = 0.0, s = 0.0;
    for (int i = 0; i < n; ++i) {
      const double y = a[i] - c;
      const double t = s + y;
      c = (t - s) - y;
      s = t;
    }
    return s;
  };
  std::atomic<int> next(0);
  auto worker = [&]() {
    for (;;) {
      const int z = next.fetch_add(1);
      if (z >= nz) break;
      Zone Zn(N);
      if (N->rhs_noise >= 0) Zn.noise = noise_state(N->rhs_noise, z);
      double *y = X + (size_t)z * ldx;
      const double *tt = time + (size_t)z * npts, *tp = t9 + (size_t)z * npts, *tr = rho + (size_t)z * npts;
      if (std::fabs(ONE - sortedsum(y, N->nsp)) > 1.e-8) {  // check_2d_mass_cons(.true.), renorm_2d
        const double s = ksum(y, N->nsp);
        for (int i = 0; i < N->nsp; ++i) y[i] = y[i] / s;
      }
      int32_t bd = 0;
      int r = 0, f = -1;
      double yez = ye[z];
      for (int i = 1; i < npts; ++i) {
        yez = calculate_ye(*N, y);
        r = integrate_zone(Zn, y, tp[i - 1], tp[i], tr[i - 1], tr[i], yez, tt[i] - tt[i - 1], &bd);
        if (r != 0) {
          f = i - 1;
          break;
        }
        double s = 0.0;  // check_1d_mass_cons(.false.)
        for (int q = 0; q < N->nsp; ++q) s += y[q];
        if (std::fabs(ONE - s) > 5.e-7) {
          const double k = ksum(y, N->nsp);
          for (int q = 0; q < N->nsp; ++q) y[q] = y[q] / k;
        }
      }
      ye[z] = yez;
      ierr[z] = r;
      if (fail) fail[z] = f;
      if (stats) stats[z] = Zn.st;
    }
  };
  const int nt = std::max(1, (int)nthreads);
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(worker);
  worker();
  for (auto &t : th) t.join();
  return 0;
}

int oracle_nse(void *net, int32_t nz, const double *t9, const double *rho, const double *ye, double *X,
               int32_t ldx, double *mu_p, double *mu_n, int32_t *iters, int32_t *ierr) {
  Net *N = (Net *)net;
  if (N->nse_iprot < 0 || N->nse_ini56 < 0) return -1;
  for (int z = 0; z < nz; ++z) {
    Zone Zn(N);
    int it = 0;
    ierr[z] = compute_nse(Zn, t9[z], rho[z], ye[z], X + (size_t)z * ldx, mu_p[z], mu_n[z], it);
    iters[z] = it;
  }
  return 0;
}
double oracle_sortedsum(const double *a, int32_t n) { return sortedsum(a, n); }

// ---- mppnp's diffusive mixing (frames/mppnp/source/mixing.F90), restated per species as the
// reference runs it: mix_calculate_D_Lagrangian :60-98, matrixdiffus :176-250, matrixdiffus_mesa
// :254-323 with reduce_term :327-340, and mixdiff08 :104-146 calling tridag :150-174 for every
// considered species 1 .. NSP-1 (0-based 0 .. nsp-2) on a fresh copy of the matrix.
void oracle_mix_d_lagrangian(int32_t m, const double *d_eul, const double *rho, const double *rad, double *d_lagr) {
  const double dconst = 3.0589703419947736e-11;
  for (int j = 1; j <= m; ++j) {
    d_lagr[j - 1] = ZERO;
    if (d_eul[j - 1] <= ZERO) continue;
    double lnrho, lnrad;
    if (j == 1) {
      lnrho = std::log(rho[j - 1]);
      lnrad = std::log(rad[j - 1]);
    } else {
      lnrho = (std::log(rho[j - 1]) + std::log(rho[j - 2])) / TWO;
      lnrad = (std::log(rad[j - 1]) + std::log(rad[j - 2])) / TWO;
    }
    d_lagr[j - 1] = d_eul[j - 1] * std::pow(dconst, TWO) * std::exp(TWO * (TWO * lnrad + lnrho));
  }
}

// tridag with 1-based arrays as in the reference; returns nonzero for a zero pivot
static int tridag_ref(const vector<double> &a, const vector<double> &b, const vector<double> &c,
                      const vector<double> &r, vector<double> &u, int n) {
  vector<double> gam(n + 1, ZERO);
  if (b[1] == ZERO) return 1;
  double bet = b[1];
  u[1] = r[1] / bet;
  for (int j = 2; j <= n; ++j) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    if (bet == ZERO) return 2;
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 1; j >= 1; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
  return 0;
}

int oracle_mix_diffusion(int32_t m, int32_t nsp, double *X, int32_t ldx, const double *xm_in, const double *dq_in,
                         double *d_io, double h, double sig, int32_t mesa, const uint8_t *consider) {
  if (m < 2) return -1;
  vector<double> a(m + 1, ZERO), b(m + 1, ZERO), c(m + 1, ZERO), D(m + 1, ZERO);
  for (int j = 1; j <= m; ++j) D[j] = d_io[j - 1];
  if (!mesa) {
    vector<double> xm(m + 1);
    for (int j = 1; j <= m; ++j) xm[j] = xm_in[j - 1];
    double xr = xm[2] - xm[1], alpha = D[2] * h / (xr * xr);
    if (sig < alpha) alpha = sig;
    a[1] = ZERO; b[1] = ONE + alpha; c[1] = -ONE * alpha;
    for (int j = 2; j <= m - 1; ++j) {
      const double xl = xm[j] - xm[j - 1];
      xr = xm[j + 1] - xm[j];
      const double xmm = HALF * (xm[j + 1] - xm[j - 1]);
      alpha = h / xmm;
      if (sig < D[j + 1] * alpha / xr) D[j + 1] = sig / alpha * xr;
      a[j] = -ONE * D[j] * alpha / xl;
      b[j] = ONE + (D[j + 1] / xr + D[j] / xl) * alpha;
      c[j] = -ONE * D[j + 1] * alpha / xr;
      if (xl == ZERO || xr == ZERO) return -2;
    }
    const double xl = xm[m] - xm[m - 1];
    alpha = D[m] * h / (xl * xl);
    a[m] = -ONE * alpha; b[m] = ONE + alpha; c[m] = ZERO;
    if (xl == ZERO || xr == ZERO) return -2;
  } else {
    vector<double> dq(m + 1), dr(m + 1, ZERO);
    for (int j = 1; j <= m; ++j) dq[j] = dq_in[j - 1];
    if (!(dq[1] > ZERO)) return -2;
    auto reduce = [&](double alpha, double onedxr, double &dc) {
      if (alpha * onedxr * dc > sig) dc = sig / (alpha * onedxr);
    };
    dr[1] = D[1];
    double xr = dq[1], alpha = h / xr, term_c = ONE / xr, dc = D[2];
    reduce(alpha, term_c, dc);
    dr[2] = dc;
    a[1] = ZERO; b[1] = ONE + term_c * alpha * dr[2]; c[1] = -ONE * term_c * alpha * dr[2];
    for (int j = 2; j <= m - 1; ++j) {
      const double xl = dq[j - 1];
      xr = dq[j];
      const double xmm = HALF * (dq[j] + dq[j - 1]);
      alpha = h / xmm;
      const double term_a = ONE / xl;
      term_c = ONE / xr;
      dc = D[j + 1];
      reduce(alpha, term_c, dc);
      dr[j + 1] = dc;
      const double term_b = term_c * dr[j + 1] + term_a * dr[j];
      a[j] = -ONE * term_a * dr[j] * alpha;
      b[j] = ONE + term_b * alpha;
      c[j] = -ONE * term_c * dr[j + 1] * alpha;
    }
    const double xl = dq[m];
    alpha = h / (xl * xl);
    a[m] = -ONE * alpha * D[m]; b[m] = ONE + alpha * D[m]; c[m] = ZERO;
  }
  vector<double> r(m + 1), u(m + 1);
  for (int s = 0; s < nsp - 1; ++s) {
    if (consider && !consider[s]) continue;
    for (int j = 1; j <= m; ++j) r[j] = X[(size_t)(j - 1) * ldx + s];
    const int e = tridag_ref(a, b, c, r, u, m);
    if (e) return -3;
    for (int j = 1; j <= m; ++j) X[(size_t)(j - 1) * ldx + s] = u[j];
  }
  for (int j = 1; j <= m; ++j) d_io[j - 1] = D[j];
  return 0;
}
void oracle_set_rhs_noise(void *net, int32_t seed) { ((Net *)net)->rhs_noise = seed < 0 ? -1 : seed; }
void oracle_set_lu_permute(void *net, int32_t seed) { ((Net *)net)->lu_permute = seed < 0 ? -1 : seed; }

}  // extern "C"

extern "C" double oracle_vital_reference(int32_t slot, double t9, double rho, double xprot) {
  return vital_reference(slot, std::min(t9, 10.0), rho, xprot);
}
