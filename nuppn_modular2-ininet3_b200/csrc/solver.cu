// solver.cu -- device kernels of the B200 reaction-network solver (sm_100a).
//
// One CTA integrates one zone at a time (persistent over a zone queue). Phases, each a block-wide
// loop over contiguous per-zone arrays followed by a barrier:
//   rates       evaluate_all_rates          physics/source/evaluate_rates.F90:14-174
//   dxdt        calculate_dxdt              solver/source/jac_rhs.F90:217-278
//   jacobian    calculate_jacobian          solver/source/jac_rhs.F90:282-455
//   assemble    reduce_jacobian as I-hJ     solver/source/jac_rhs.F90:134-197
//   factor      static-order LU of the active subsystem, dense tile up to 64 rows, sparse above
//               (replaces SuperLU dgstrf, c_fortran_dgssv.c:80-155)
//   solve       column-oriented substitution in registers (tile) or row-oriented sparse solves
//               (replaces SuperLU dgstrs, c_fortran_dgssv.c:157-174)
// and the step control of backward_euler.F90:29-176, bader_deuflhard.F90:139-488 and
// solver.F90:53-238 evaluated uniformly by every thread.
//
// Summation orders: dxdt and Jacobian entries are accumulated in the reference's order (reaction
// order, then the slot order of the reference's scatter) for every target whose list is short; the
// few long lists (the n, p, alpha rows and columns) are summed by a warp with a fixed tree.
#include <cuda_runtime.h>

#include "solver.cuh"

NUPPN_BEGIN

__constant__ double c_fact[5] = {1.0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0};

// physical constants (utils/source/constants.F90)
#define K_EV2ERG 1.602177e-12
#define K_MEV2ERG (K_EV2ERG * 1.0e6)
#define K_ERG2MEV (1.0 / K_MEV2ERG)
#define K_KEV2ERG (K_EV2ERG * 1.0e3)
#define K_PI 3.141592653589793238462643383279502884
#define K_AVOGADRO 6.022140857e23
#define K_BOLTZMANN 1.3806485279e-16
#define K_PLANCK_ERG (4.135667662e-21 * K_MEV2ERG)
#define K_HBAR_ERG (K_PLANCK_ERG / 2.0 / K_PI)
#define K_AMU 1.6605402e-24
#define K_QE 4.80320425e-10
#define K_QE2 (K_QE * K_QE)
#define K_SMALL 1.e-30
#define K_SUM_TOL 1.e-6

enum { i_ng = 1, i_gn, i_np, i_na, i_pg, i_gp, i_pn, i_pa, i_ag, i_ga, i_an, i_ap, i_bm, i_ec, i_bn, i_bp,
       i_ba, i_ve, i_vp, i_vsp, i_vsn, i_vsa };
enum { SLV_CNVRG = 1, MAX_SUBSTEPS, BAD_STEP, NEG_ABUNDS, HUGE_ABUNDS, SUM_X, GOT_NAN, BAD_YE, NSE_CNVRG,
       NSE_WEAK, SMALL_DT };

// ---------------------------------------------------------------------------------------------
// block helpers
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(NUPPN_FULL, v, o);
  return v;
}

struct Red {
  double *buf;  // shared, >= 32 doubles
};

// Every thread returns the same value (partials combined in a fixed order).
__device__ double block_sum(double v, double *sbuf) {
  v = warp_sum(v);
#if NUPPN_GROUP_WARP
  return v;  // the xor butterfly leaves the same sum in every lane
#endif
  GSYNC();
  if ((GT & 31) == 0) sbuf[GT >> 5] = v;
  GSYNC();
  double r = 0.0;
  const int nw = GN >> 5;
  for (int i = 0; i < nw; ++i) r += sbuf[i];
  return r;
}

__device__ double block_max(double v, double *sbuf) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(NUPPN_FULL, v, o));
#if NUPPN_GROUP_WARP
  return v;
#endif
  GSYNC();
  if ((GT & 31) == 0) sbuf[GT >> 5] = v;
  GSYNC();
  double r = -DBL_MAX;
  const int nw = GN >> 5;
  for (int i = 0; i < nw; ++i) r = fmax(r, sbuf[i]);
  return r;
}

__device__ bool block_any(bool p) { return g_or(p ? 1 : 0) != 0; }

// gfortran integer power (square-and-multiply, libgcc __powidf2)
__device__ __forceinline__ double powi(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
  double y = (n & 1u) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n & 1u) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

// bsearch_r8 (utils.F90:687-722), returns a 1-based index
__device__ int bsearch_r8(const double *arr, int siz, double val) {
  int a = 1, b = siz, r = b - a, m = (a + b) / 2;
  while (val != arr[m - 1] && r > 1) {
    if (arr[m - 1] > val) b = m; else a = m;
    r = b - a;
    m = (a + b) / 2;
  }
  if (arr[m - 1] > val) m = m - 1;
  return m;
}

// ---------------------------------------------------------------------------------------------
// rates
struct Screen {
  double gamfac, zeta;
};

__device__ double chugunov(const Screen &S, double z1, double z2) {  // screening_chugunov.F90:140-234
  const double c_a1 = 2.7822, c_a2 = 98.34, c_b1 = -1.7476, c_b2 = 66.07, c_b3 = 1.12, c_b4 = 65.0,
               alfa = 0.022, gamfitlim = 600.0, g0 = 599.0;
  const double c_a3 = sqrt(3.0) - c_a1 / sqrt(c_a2);
  if (z1 <= 0.0 || z2 <= 0.0) return 1.0;
  double gam = z1 * z2 * S.gamfac;
  double beta = 0.41 - 0.6 / gam, gama = 0.06 + 2.2 / gam;
  double gamtild = gam / pow(1.0 + alfa * S.zeta + beta * powi(S.zeta, 2) + gama * powi(S.zeta, 3), 1.0 / 3.0);
  if (gamtild >= 650) {
    gamtild = gamfitlim;
  } else if (gamtild > 550) {
    double s = 1.0 / (1.0 + exp(-(gamtild - g0) / 1.0));
    gamtild = s * gamfitlim + (1 - s) * gamtild;
  }
  double g2 = gamtild * gamtild;
  double t1 = pow(gamtild, 1.5) * (c_a1 / sqrt(c_a2 + gamtild) + c_a3 / (1 + gamtild));
  double t2 = c_b1 * g2 / (c_b2 + gamtild);
  double t3 = c_b3 * g2 / (c_b4 + g2);
  return fmin(exp(t1 + t2 + t3), 1e30);
}

__device__ __forceinline__ double screening(const DevNet &N, const Screen &S, double z1, double z2) {
  double f = N.kn.screen_option == 2 ? chugunov(S, z1, z2) : 1.0;
  return fmin(f, 1.e30);
}

// exv (vital.F90:2583-2593): exp with linear continuation beyond |x| = 200
__device__ __forceinline__ double vital_exv(double x) {
  if (x > 200.0) return (x - 200.0) * exp(200.0);
  if (x < -200.0) return -exp(-200.0) / (x + 200.0);
  return exp(x);
}

// The reference's own VITAL formulas (vital_calculate_rates, vital.F90:339-569) for the pp chains
// (slots 1-9; 10-13 are off with IPPIV = 0) and the first CNO reactions (14-17, 73), at the clipped
// t9 (<= 10), in the reference's order of operations. PROTOFAK is 1; FABE7 reads X(p) = xprot.
// Not inlined: the integration kernels that evaluate rates keep their own register allocation.
__device__ __noinline__ double vital_formula(int slot, double t9, double rho, double xprot) {
  const double third = 1.0 / 3.0, fourth = 1.0 / 4.0, sixth = 1.0 / 6.0;
  const double five_sixths = 5.0 * sixth, t9ppmax = 10.0, protofak = 1.0;
  const double tp13 = pow(t9, third), tp14 = pow(t9, fourth), tp12 = tp14 * tp14, tp23 = tp13 * tp13;
  const double tp32 = t9 * tp12, tp43 = t9 * tp13, tp53 = t9 * tp23;
  const double tm13 = 1.0 / tp13, tm23 = 1.0 / tp23, tm32 = 1.0 / tp32, t9inv = 1.0 / t9;
  if (slot == 5) {  // Be7(e-,nu)Li7, CF88, computed at every t9 (:340-343); the rest from T9 >= 0.001 (:364)
    const double fabe7 = 0.5 * (1.0 + xprot);
    double v = 1.34e-10 / tp12 * (1.0 - 0.537 * tp13 + 3.86 * tp23 + 0.0027 * t9inv * vital_exv(2.515e-03 * t9inv)) *
               rho * fabe7;
    if (t9 < 1.e-03 || t9 > t9ppmax) v = fmin(v, 1.51e-07);
    return v;
  }
  if (!(t9 >= 0.001)) return 0.0;
  if (slot <= 9) {  // pp I-III (:366-487), 1.2e-3 < T9 < T9PPMAX
    if (!(t9 > 1.2e-3 && t9 < t9ppmax)) return 0.0;
    switch (slot) {
      case 1:
        return (4.01e-15 * tm23 * vital_exv(-3.380 * tm13) * (1.0 + 0.123 * tp13 + 1.09 * tp23 + 0.938 * t9)) * rho *
               protofak;
      case 2:
        return (2.24e+03 * tm23 * vital_exv(-3.720 * tm13) * (1.0 + 0.112 * tp13 + 3.38 * tp23 + 2.65 * t9)) * rho *
               protofak;
      case 3:
        return (6.04e+10 * tm23 * vital_exv(-12.276 * tm13) *
                (1.0 + 0.034 * tp13 - 0.522 * tp23 - 0.124 * t9 + 0.353 * tp43 + 0.213 * tp53)) *
               rho;
      case 4: {
        const double tt = t9 / (1.0 + 4.95e-02 * t9), t56 = pow(tt, five_sixths), t13 = pow(tt, third);
        return (5.61e+06 * t56 / tp32 * vital_exv(-12.826 / t13)) * rho;
      }
      case 6: {
        const double t9a = t9 / (1.0 + 0.759 * t9), t9a13 = pow(t9a, third), t9a56 = pow(t9a, five_sixths);
        return (1.096e+09 / tp23 * vital_exv(-8.472 / tp13) - 4.83e+08 * t9a56 / tp32 * vital_exv(-8.472 / t9a13) +
                1.06e+10 / tp32 * vital_exv(-30.442 / t9)) *
               rho * protofak;
      }
      case 7:
      case 9: {
        const double v7 =
            (3.11e5 / tp23 * vital_exv(-10.262 / tp13) + 2.53e3 / tp32 * vital_exv(-7.306 / t9)) * rho * protofak;
        if (slot == 7) return v7;
        const double rev = 1.30e+10 * tp32 * vital_exv(-1.595 / t9) / (rho);
        return rev * v7;
      }
      case 8: return 8.96e-1;
      default: return 0.0;
    }
  }
  if (!(t9 > 5.e-3)) return 0.0;  // CNO (:532-571)
  switch (slot) {
    case 14:
    case 73: {
      const double q = t9 / 0.46;
      double v14 = (2.00e+07 * tm23 * vital_exv(-13.692 * tm13 - q * q) *
                        (1.0 + 9.89 * t9 - 59.8 * t9 * t9 + 266.0 * t9 * t9 * t9) +
                    1.00e+05 * tm32 * vital_exv(-4.913 / t9) + 4.24e+05 * tm32 * vital_exv(-21.62 / t9));
      v14 = v14 * rho * protofak;
      if (slot == 14) return v14;
      return v14 / (rho * protofak) * 8.84e+09 * tp32 * vital_exv(-22.553 / t9);
    }
    case 15:
      return (9.57e+07 * tm23 * vital_exv(-13.720 * tm13 - t9 * t9) * (1.0 + 3.56 * t9) +
              1.50e+06 * tm32 * vital_exv(-5.930 / t9) + exp(-12.057 / t9) * 6.83e+05 / pow(t9, 0.864)) *
             rho * protofak;
    case 16: {  // RHO*PROTOFAK multiplies the second term only, as the reference writes it
      const double q = t9 / 1.191;
      return 4.04e+07 * tm23 * vital_exv(-15.202 * tm13 - q * q) *
                 (1.0 + 0.027 * tp13 - 0.803 * tp23 - 0.154 * t9 + 5.00 * tp43 + 2.44 * tp53) +
             2.43e+05 * tm32 * vital_exv(-6.348 / t9) * rho * protofak;
    }
    case 17: {
      const double q = t9 / 3.294;
      return (4.90e7 / tp23 * vital_exv(-15.228 / tp13 - q * q) *
                  (1.0 + 0.027 * tp13 - 0.778 * tp23 - 0.149 * t9 + 0.261 * tp43 + 0.127 * tp53) +
              2.37e3 / tp32 * vital_exv(-3.011 / t9) + 2.19e4 * vital_exv(-12.530 / t9)) *
             rho * protofak;
    }
    default: return 0.0;
  }
}

// evaluate_all_rates for the CTA's zone; y = mass fractions (read for screening and VITAL)
__device__ void dev_eval_rates(const DevNet &N, const Ws &W, double t9, double rho, double ye, const double *y,
                               double *sred) {
  const int tid = GT, nt = GN;
  // partition functions (reaclib.F90:586-605)
  if (N.npart > 0) {
    double t9c = fmax(N.pt9[0], fmin(t9, N.pt9[kPartDim - 1]));
    int i0 = bsearch_r8(N.pt9, kPartDim, t9c);
    double t90 = N.pt9[i0 - 1], t91 = N.pt9[i0];
    double Dt9 = (t9c - t90) / (t91 - t90);
    for (int p = tid; p < N.npart; p += nt) {
      const double *pv = N.pval + (size_t)p * kPartDim;
      W.partinter[p] = pv[i0 - 1] + (pv[i0] - pv[i0 - 1]) * Dt9;
    }
  }
  GSYNC();
  // REACLIB rates (reaclib.F90:471-581)
  {
    double t = fmax(t9, 0.01), rhoye = rho * ye;
    double t9inv = 1.0 / t, t13 = pow(t, 1.0 / 3.0), t13inv = 1.0 / t13, t43 = t * t13, t53 = t13 * t43;
    double lnt9 = log(t);
    for (int r = tid; r < N.nr; r += nt) {
      double acc = 0.0;
      for (int c = N.rl_first[r]; c < N.rl_first[r + 1]; ++c) {
        const double *a = N.rl_a + (size_t)c * 7;
        double r0 = a[0] + a[1] * t9inv + a[2] * t13inv + a[3] * t13 + a[4] * t + a[5] * t53 + a[6] * lnt9;
        acc = acc + exp(r0);
      }
      int info = N.rl_info[r];
      double Gfac = 1.0;
      if (info & 0x100) {
        double g[6];
        for (int s = 0; s < 6; ++s) {
          int p = N.rl_part[r * 6 + s];
          g[s] = p < 0 ? 1.0 : W.partinter[p];
        }
        switch (info & 0xff) {
          case 1: Gfac = g[1] / g[0]; break;
          case 2: Gfac = g[1] * g[2] / g[0]; break;
          case 3: Gfac = g[1] * g[2] * g[3] / g[0]; break;
          case 4: Gfac = g[2] / (g[0] * g[1]); break;
          case 5: Gfac = g[2] * g[3] / (g[0] * g[1]); break;
          case 6: Gfac = g[2] * g[3] * g[4] / (g[0] * g[1]); break;
          case 7: Gfac = g[2] * g[3] * g[4] * g[5] / (g[0] * g[1]); break;
          case 8: Gfac = g[3] / (g[0] * g[1] * g[2]); break;
          case 9: Gfac = g[3] * g[4] / (g[0] * g[1] * g[2]); break;
          case 10: Gfac = g[4] * g[5] / (g[0] * g[1] * g[2] * g[3]); break;
          case 11: Gfac = g[1] * g[2] * g[3] * g[4] * g[5] / g[0]; break;
          default: Gfac = 1.0;
        }
      }
      double rv = acc * Gfac, out;
      switch (info >> 16) {
        case i_bm: case i_gn: case i_bn: case i_bp: case i_gp: case i_ga: out = rv; break;
        case i_ec: out = (info & 0x200) ? rv * rhoye : rv; break;
        case i_ng: case i_pg: case i_ag: case i_np: case i_na: case i_pn: case i_pa: case i_an: case i_ap:
          out = rv * rho; break;
        default: out = 1.e-99;
      }
      W.rv[r] = fmax(out, 1e-99);
    }
  }
  // NETGEN tables (netgen.F90:179-310)
  if (N.ngn > 0) {
    double t8 = t9 * 10.0, rhoye = rho * ye, ane_in = rhoye * K_AVOGADRO;
    t8 = fmin(fmax(t8, N.ngt8[0]), N.ngt8[N.ngk - 1]);
    int klo = bsearch_r8(N.ngt8, N.ngk, t8), khi = klo + 1;
    double h = N.ngl10t8[khi - 1] - N.ngl10t8[klo - 1];
    double b = (log10(t8) - N.ngl10t8[klo - 1]) / h;
    for (int i = tid; i < N.ngn; i += nt) {
      const size_t lo = ((size_t)(klo - 1) * N.ngn + i) * N.ngd, hi = ((size_t)(khi - 1) * N.ngn + i) * N.ngd;
      double v = 0.0, flg = N.ngflag[i];
      if (flg <= 0.0) {
        double l10 = N.ngl10v[lo] + b * (N.ngl10v[hi] - N.ngl10v[lo]);
        switch ((int)llrint(flg)) {
          case -14:
            v = pow(10.0, l10) * rhoye;
            if (t8 < 0.01) v = fmin(v, 1.51e-7 / rhoye);
            break;
          case -13: v = pow(10.0, l10) * rhoye; break;
          case -11: v = pow(10.0, l10); break;
          case -10: v = pow(10.0, l10) * rho; break;
          case -100: v = pow(10.0, l10) * (rho * rho); break;
          case -200: v = pow(10.0, l10) * (rho * rho * rho); break;
          default: v = 0.0;
        }
      } else {
        // every rate re-locates its electron density (the reference caches it per table shape)
        int ndt = N.ngndata[i];
        const double *ane = N.ngane + (size_t)i * N.ngd;
        double an = fmin(fmax(ane_in, flg), ane[ndt - 1]);
        int jlo = bsearch_r8(ane, ndt, an), jhi = jlo + 1;
        double anelo = ane[jlo - 1], anehi = ane[jhi - 1];
        double vlow = N.ngl10v[lo + jlo - 1] + b * (N.ngl10v[hi + jlo - 1] - N.ngl10v[lo + jlo - 1]);
        double vhigh = N.ngl10v[lo + jhi - 1] + b * (N.ngl10v[hi + jhi - 1] - N.ngl10v[lo + jhi - 1]);
        vlow = pow(10.0, vlow);
        vhigh = pow(10.0, vhigh);
        v = (vhigh - vlow) / (anehi - anelo) * (an - anelo) + vlow;
      }
      W.ngv[i] = fmax(v, 1e-99);
    }
  }
  // FFN (fuller.F90:92-122 with generic_interp_2d, utils.F90:624-666)
  if (N.ffv > 0) {
    double t90 = log10(t9), r0 = log10(rho * ye);
    t90 = fmin(fmax(t90, N.fft9[0]), N.fft9[N.fft - 1]);
    r0 = fmin(fmax(r0, N.ffrho[0]), N.ffrho[N.ffr - 1]);
    int ix1 = bsearch_r8(N.fft9, N.fft, t90), iy1 = bsearch_r8(N.ffrho, N.ffr, r0);
    double x1 = N.fft9[ix1 - 1], x2 = N.fft9[ix1], y1 = N.ffrho[iy1 - 1], y2 = N.ffrho[iy1];
    double xb = (t90 - x1) / (x2 - x1), xa = 1.0 - xb, yb = (r0 - y1) / (y2 - y1), ya = 1.0 - yb;
    for (int v = tid; v < N.ffv; v += nt) {
      const double *F = N.ffl10v + (size_t)v * N.fft * N.ffr;
      double f11 = F[(ix1 - 1) * N.ffr + iy1 - 1], f21 = F[ix1 * N.ffr + iy1 - 1];
      double f12 = F[(ix1 - 1) * N.ffr + iy1], f22 = F[ix1 * N.ffr + iy1];
      double fA = f11 * ya + f12 * yb, fC = f21 * ya + f22 * yb;
      W.ffv[v] = pow(10.0, fA * xa + fC * xb);
    }
  }
  // KADoNiS, Akima in kT (kadonis.F90:150-187, akima.F90:135-170)
  if (N.kdn > 0) {
    bool on = t9 > 0.001;  // t9_netgen_limit (netgen.F90:42)
    double E = t9 * 1e9 * (K_BOLTZMANN / K_KEV2ERG);
    E = fmin(fmax(E, N.kdE[0]), N.kdE[N.kde - 1]);
    int j = N.kde - 1;
    while (j > 1 && E < N.kdE[j - 1]) --j;
    double dx = E - N.kdE[j - 1];
    for (int i = tid; i < N.kdn; i += nt) {
      const double *c = N.kdcoef + ((size_t)i * (N.kde - 1) + (j - 1)) * 4;
      W.kdv[i] = on ? (c[0] + c[1] * dx + c[2] * powi(dx, 2) + c[3] * powi(dx, 3)) * rho : 0.0;
    }
  }
  // G of every species for detailed balance (reverse.F90:123-137)
  for (int s = tid; s < N.nsp; s += nt) {
    double g = N.gspin_nse[s];
    W.G[s] = g != 0.0 ? (N.spart[s] >= 0 ? W.partinter[N.spart[s]] : 1.0) * g : 1.0;
  }
  GSYNC();
  // gather by source (ppn_physics.F90:550-589), VITAL, constants; rate factors (evaluate_rates.F90:195)
  {
    double tv = fmin(t9, 10.0), tm13 = 1.0 / pow(tv, 1.0 / 3.0);
    for (int l = tid; l < N.nre; l += nt) {
      double v = 0.0;
      if (!N.rev_target[l]) {
        int i = N.sidx[l];
        switch (N.src[l]) {
          case NUPPN_SRC_VITAL: {
            if (N.vform[i] > 0) {
              v = vital_formula(N.vform[i], tv, rho, N.vxfac[i] >= 0 ? y[N.vxfac[i]] : 0.0);
              break;
            }
            double s = 0.0;
            for (int t = N.vfirst[i]; t < N.vfirst[i + 1]; ++t) {
              const double *c = N.vterms + (size_t)t * 5;
              s = s + c[0] * pow(tv, c[1]) * exp(c[2] * tm13 + c[3] / tv + c[4] * tv);
            }
            double f = pow(rho, N.vdpow[i]);
            if (N.vxfac[i] >= 0) f = f * (0.5 * (1.0 + y[N.vxfac[i]]));
            v = s * f;
            break;
          }
          case NUPPN_SRC_REACLIB: v = W.rv[i]; break;
          case NUPPN_SRC_NETGEN: v = W.ngv[i]; break;
          case NUPPN_SRC_FULLER: v = W.ffv[i]; break;
          case NUPPN_SRC_KADONIS: v = W.kdv[i]; break;
          case NUPPN_SRC_CONST: v = N.constr[i]; break;
          default: v = 0.0;
        }
      }
      W.v[l] = fmax(v * N.rfac[l], 1.e-99);
    }
  }
  GSYNC();
  // detailed balance (reverse.F90:107-335, Coulomb corrections off); forwards read before writes
  if (N.kn.detailed_balance) {
    double kTerg = K_BOLTZMANN * t9 * 1.e9, kTMeV = kTerg * K_ERG2MEV;
    for (int l = tid; l < N.nre; l += nt) {
      double out = -1.0;
      if (N.crea[l] && N.irev[l] >= 0 && N.rev_kind[l] > 0 && W.v[l] > 1.e-97) {
        const int *sp = N.rev_sp + (size_t)l * 4;
        double Ga1 = W.G[sp[0]], Ga2 = W.G[sp[1]], Gb1 = sp[2] >= 0 ? W.G[sp[2]] : 0.0, Gb2 = W.G[sp[3]];
        double pfac, mfac, rhofac;
        if (N.rev_kind[l] == 1) {
          pfac = Ga1 * Ga2 / Gb2;
          mfac = pow(N.rev_mc[l] * kTerg, 1.5);
          rhofac = 1.0 / rho / K_AVOGADRO;
        } else {
          pfac = Ga1 * Ga2 / Gb1 / Gb2;
          mfac = N.rev_mc[l];
          rhofac = 1.0;
        }
        double x = fmin(-N.rev_Q[l] / kTMeV, 200.0);
        double fac = mfac * exp(x) * rhofac * pfac;
        fac = fmin(fmax(fac, 1e-99), 1e99);
        out = fmax(W.v[l] * fac, 1e-99);
      }
      W.contrib[l] = out;
    }
    GSYNC();
    for (int l = tid; l < N.nre; l += nt)
      if (W.contrib[l] >= 0.0) W.v[N.irev[l]] = W.contrib[l];
  }
  // screening precalc (screening_chugunov.F90:67-134 with calculate_azbar, utils.F90:504-525)
  Screen S;
  {
    double ytot = 0.0, sa = 0.0, sz = 0.0;
    for (int s = tid; s < N.nsp; s += nt)
      if (N.ciso[s]) {
        double yy = y[s] / N.an[s];
        ytot += yy;
        sa += N.an[s] * yy;
        sz += N.zn[s] * yy;
      }
    ytot = block_sum(ytot, sred);
    sa = block_sum(sa, sred);
    sz = block_sum(sz, sred);
    double abar = sa / ytot, zbar = sz / ytot, tkin = t9 * 1.e9;
    const double fourov3pi = 4.0 / (3.0 * K_PI * K_PI), fourpiqe2 = 4.0 * K_PI * K_QE2;
    const double t1 = 0.1, t2 = 0.2, t0 = (t1 + t2) * 0.5;
    double ntot = rho / (abar * K_AMU);
    double denom = pow(3.0 / (4.0 * K_PI * zbar * ntot), 1.0 / 3.0);
    double a_av = denom * pow(zbar, 1.0 / 3.0);
    double wp = pow(fourpiqe2 * zbar * zbar * ntot / (abar * K_AMU), 0.5);
    double tp = K_HBAR_ERG * wp / K_BOLTZMANN;
    double tn = tkin / tp, tk;
    if (tn >= 2.0 * t2) tk = tkin;
    else if (tn <= 0.5 * t1) tk = t1 * tp;
    else {
      double s = 1.0 / (1.0 + exp(-(tn - t0) / 0.01));
      tn = (1.0 - s) * t1 + s * tn;
      tk = tn * tp;
    }
    S.gamfac = K_QE2 / (a_av * tk) / K_BOLTZMANN;
    S.zeta = pow(fourov3pi * tp * tp / tk / tk, 1.0 / 3.0);
  }
  // screening loop and toggles (evaluate_rates.F90:69-172)
  {
    const double zhe = N.ihe4 >= 0 ? N.zn[N.ihe4] : 0.0, zbe = N.ibe8 >= 0 ? N.zn[N.ibe8] : 0.0;
    for (int l = tid; l < N.nre; l += nt) {
      double v = W.v[l];
      int mode = N.scr_mode[l];
      if (mode != 3 && v > 1.e-99) {
        if (mode == 1) v = v * screening(N, S, zhe, zhe) * screening(N, S, zhe, zbe);
        else if (mode == 2) v = v * screening(N, S, zhe, zhe);
        else v = v * screening(N, S, N.scr_z1[l], N.scr_z2[l]);
      }
      if (N.crea[l]) {
        int t = N.ilabb[l];
        bool weak = t == i_ec || t == i_bm || t == i_bn || t == i_bp || t == i_ve || t == i_vp || t == i_vsp ||
                    t == i_vsn || t == i_vsa;
        if (!N.kn.weak_rates && weak) v = 1.e-99;
        if (!N.kn.strong_rates && !weak) v = 1.e-99;
        if (N.kn.decay && !(t == i_ec || t == i_bm || t == i_bn || t == i_bp || t == i_ba)) v = 1.e-99;
      }
      W.v[l] = fmax(v, 1.e-99);
    }
  }
  GSYNC();
}

// ---------------------------------------------------------------------------------------------
// RHS: calculate_dxdt (jac_rhs.F90:217-278)
__device__ void dev_dxdt(const DevNet &N, const Ws &W, const double *x, double *dxdt) {
  const int tid = GT, nt = GN;
  for (int s = tid; s < N.nsp; s += nt)
    W.xn[s] = s == N.ig ? 1.0 : ((N.ciso[s] && N.an[s] != 0.0) ? x[s] / N.an[s] : 0.0);
  GSYNC();
  for (int a = tid; a < N.nact; a += nt) {
    const int *k = N.act_k + (size_t)a * 8;
    W.flux[a] = c_fact[k[1]] * W.v[N.act_slot[a]] * powi(W.xn[k[0]], k[1]) * W.xn[k[2]];
  }
  GSYNC();
  for (int s = tid; s < N.nsp; s += nt) {
    int p0 = N.dg_ptr[s], p1 = N.dg_ptr[s + 1];
    if (p1 - p0 > kLongList) continue;
    double acc = 0.0;
    for (int p = p0; p < p1; ++p) acc = acc + N.dg_coef[p] * W.flux[N.dg_item[p] >> 2];
    if (N.ciso[s]) acc = acc * N.an[s];
    dxdt[s] = s == N.ig ? 0.0 : acc;
  }
  {
    const int lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    for (int q = w; q < N.ndg_long; q += nw) {
      int s = N.dg_long[q];
      int p0 = N.dg_ptr[s], p1 = N.dg_ptr[s + 1];
      double acc = 0.0;
      for (int p = p0 + lane; p < p1; p += 32) acc += N.dg_coef[p] * W.flux[N.dg_item[p] >> 2];
      acc = warp_sum(acc);
      if (lane == 0) {
        if (N.ciso[s]) acc = acc * N.an[s];
        dxdt[s] = s == N.ig ? 0.0 : acc;
      }
    }
  }
  GSYNC();
}

// ---------------------------------------------------------------------------------------------
// Jacobian values, entry set flags and dynamic-network mask: calculate_jacobian (jac_rhs.F90:282-455).
// The mask of the reference grows while its reaction loop runs; reaction a sets its entries only if
// its participants were masked by a reaction a' <= a. first_l[s] = min a' that masks s reproduces
// that exactly.
__device__ void dev_jacobian(const DevNet &N, const Ws &W, double dzeit, const double *x) {
  const int tid = GT, nt = GN, g = N.ig;
  const double dfdNmin = N.kn.cyminformal / dzeit;
  for (int s = tid; s < N.nsp; s += nt) {
    W.xn[s] = s == g ? 1.0 : ((N.ciso[s] && N.an[s] > 0.0) ? x[s] / N.an[s] : 0.0);
    W.first_l[s] = 0x7fffffff;
  }
  for (int e = tid; e < N.nnzJ; e += nt) W.eset[e] = 0;
  GSYNC();
  for (int a = tid; a < N.nact; a += nt) {
    const int *k = N.act_k + (size_t)a * 8;
    double v = W.v[N.act_slot[a]];
    double *c = W.contrib + (size_t)a * 8;
    if (!(fabs(v) / dzeit > N.kn.min_rate_ov_dt)) {
      for (int s = 0; s < 8; ++s) c[s] = 0.0;
      W.flux[a] = 0.0;
      continue;
    }
    W.flux[a] = 1.0;
    int in1 = k[0], in2 = k[2], out1 = k[4], out2 = k[6];
    int Nin1 = k[1], Nin2 = k[3], Nout1 = k[5], Nout2 = k[7];
    double ain1 = N.an[in1], ain2 = N.an[in2], aout1 = N.an[out1], aout2 = N.an[out2];
    double y1 = W.xn[in1], y2 = W.xn[in2];
    double stem = c_fact[Nin1] * c_fact[Nin2] * v;
    double dfdN = stem * powi(y1, Nin1) * y2;
    if (fabs(dfdN) > dfdNmin) {
      atomicMin(&W.first_l[in1], a); atomicMin(&W.first_l[in2], a);
      atomicMin(&W.first_l[out1], a); atomicMin(&W.first_l[out2], a);
    }
    stem = (double)Nin1 * c_fact[Nin1] * c_fact[Nin2] * powi(y2, Nin2) * powi(y1, Nin1 - 1) * v;
    double dfin1dy1 = (double)(-Nin1) * stem, dfin2dy1 = (double)(-Nin2) * stem;
    double dfout1dy1 = (double)Nout1 * stem, dfout2dy1 = (double)Nout2 * stem;
    stem = (double)Nin2 * c_fact[Nin1] * c_fact[Nin2] * powi(y1, Nin1) * powi(y2, Nin2 - 1) * v;
    double dfin1dy2 = (double)(-Nin1) * stem, dfin2dy2 = (double)(-Nin2) * stem;
    double dfout1dy2 = (double)Nout1 * stem, dfout2dy2 = (double)Nout2 * stem;
    // slot order: in1in1, in2in1, out1in1, out2in1, in1in2, in2in2, out1in2, out2in2
    c[0] = in1 != g ? dfin1dy1 * ain1 / ain1 : 0.0;
    c[1] = (in1 != g && in2 != g) ? dfin2dy1 * ain2 / ain1 : 0.0;
    c[4] = (in1 != g && in2 != g) ? dfin1dy2 * ain1 / ain2 : 0.0;
    c[2] = (in1 != g && out1 != g) ? dfout1dy1 * aout1 / ain1 : 0.0;
    c[3] = (in1 != g && out2 != g) ? dfout2dy1 * aout2 / ain1 : 0.0;
    c[5] = in2 != g ? dfin2dy2 * ain2 / ain2 : 0.0;
    c[6] = (in2 != g && out1 != g) ? dfout1dy2 * aout1 / ain2 : 0.0;
    c[7] = (in2 != g && out2 != g) ? dfout2dy2 * aout2 / ain2 : 0.0;
  }
  GSYNC();
  for (int a = tid; a < N.nact; a += nt) {
    if (W.flux[a] == 0.0) continue;
    const int *k = N.act_k + (size_t)a * 8;
    int in1 = k[0], in2 = k[2], out1 = k[4], out2 = k[6];
    if (in2 != g && W.first_l[in2] > a) continue;
    if (out1 != g && W.first_l[out1] > a) continue;
    if (W.first_l[in1] > a || W.first_l[out2] > a) continue;
    const int *ice = N.act_ice + (size_t)a * 8;
    if (in1 != g) W.eset[ice[0]] = 1;
    if (in1 != g && in2 != g) { W.eset[ice[1]] = 1; W.eset[ice[4]] = 1; }
    if (in1 != g && out1 != g) W.eset[ice[2]] = 1;
    if (in1 != g && out2 != g) W.eset[ice[3]] = 1;
    if (in2 != g) W.eset[ice[5]] = 1;
    if (in2 != g && out1 != g) W.eset[ice[6]] = 1;
    if (in2 != g && out2 != g) W.eset[ice[7]] = 1;
  }
  for (int e = tid; e < N.nnzJ; e += nt) {
    int p0 = N.jg_ptr[e], p1 = N.jg_ptr[e + 1];
    if (p1 - p0 > kLongList) continue;
    double acc = 1.e-99;
    for (int p = p0; p < p1; ++p) acc = acc + W.contrib[N.jg_item[p]];
    W.jac[e] = acc;
  }
  {
    const int lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    for (int q = w; q < N.njg_long; q += nw) {
      int e = N.jg_long[q];
      int p0 = N.jg_ptr[e], p1 = N.jg_ptr[e + 1];
      double acc = 0.0;
      for (int p = p0 + lane; p < p1; p += 32) acc += W.contrib[N.jg_item[p]];
      acc = warp_sum(acc);
      if (lane == 0) W.jac[e] = 1.e-99 + acc;
    }
  }
  for (int s = tid; s < N.nsp; s += nt) W.mask[s] = (W.first_l[s] != 0x7fffffff && s != g) ? 1 : 0;
  GSYNC();
}

// First pass of calculate_jacobian for the integrator: only the dynamic-network mask (first_l, mask)
// and each reaction's rate test (flux[a] = 1 if |v|/dt > min_rate_ov_dt). The values and entry flags
// are then built for the active subsystem only (dev_jacobian_active, active_lu.cuh).
__device__ void dev_jacobian_mask(const DevNet &N, const Ws &W, double dzeit, const double *x) {
  const int tid = GT, nt = GN, g = N.ig;
  const double dfdNmin = N.kn.cyminformal / dzeit;
  for (int s = tid; s < N.nsp; s += nt) {
    W.xn[s] = s == g ? 1.0 : ((N.ciso[s] && N.an[s] > 0.0) ? x[s] / N.an[s] : 0.0);
    W.first_l[s] = 0x7fffffff;
  }
  GSYNC();
  for (int a = tid; a < N.nact; a += nt) {
    const int *k = N.act_k + (size_t)a * 8;
    const double v = W.v[N.act_slot[a]];
    if (!(fabs(v) / dzeit > N.kn.min_rate_ov_dt)) {
      W.flux[a] = 0.0;
      continue;
    }
    W.flux[a] = 1.0;
    const double dfdN = c_fact[k[1]] * c_fact[k[3]] * v * powi(W.xn[k[0]], k[1]) * W.xn[k[2]];
    if (fabs(dfdN) > dfdNmin) {
      atomicMin(&W.first_l[k[0]], a); atomicMin(&W.first_l[k[2]], a);
      atomicMin(&W.first_l[k[4]], a); atomicMin(&W.first_l[k[6]], a);
    }
  }
  GSYNC();
  for (int s = tid; s < N.nsp; s += nt) W.mask[s] = (W.first_l[s] != 0x7fffffff && s != g) ? 1 : 0;
  GSYNC();
}
NUPPN_END

#include "active_lu.cuh"
#include "nse.cuh"
#include "integrator.cuh"

NUPPN_BEGIN

// ---------------------------------------------------------------------------------------------
// kernels: persistent groups, one zone at a time, workspace slab per group; dynamic shared memory
// holds the active-subsystem LU when it fits (act_smem bytes per group).
constexpr int kQueueSpinLimit = 1 << 24;  // polls of the serving queue per claim, whatever the queue does
#if NUPPN_GROUP_WARP
#define NUPPN_INTEGRATE_BOUNDS __launch_bounds__(256, 1)
#else
#define NUPPN_INTEGRATE_BOUNDS __launch_bounds__(256, 3)
#endif

// Next request of the serving queue for the calling thread's group, or -1 once the queue has stayed
// empty for Q.idle_polls polls (the group then leaves and the host relaunches the loop when requests
// come again) or the host has asked the loop to stop. Requests are claimed in publication order.
// Every wait is bounded.
__device__ long long queue_claim(const ServeQueue &Q) {
  unsigned ns = 128;
  int idle = 0;
  for (int it = 0; it < kQueueSpinLimit; ++it) {
    const long long p = *(const volatile long long *)Q.published;
    const unsigned long long c = *(volatile unsigned long long *)Q.claimed;
    if ((long long)c < p) {
      if (atomicCAS(Q.claimed, c, c + 1ull) == c) return (long long)c;
      continue;  // another group took request c
    }
    if (*(const volatile int *)Q.stop || ++idle > Q.idle_polls) return -1;
    __nanosleep(ns);
    if (ns < 8192) ns <<= 1;
  }
  return -1;
}

// One zone per group: a CTA of the cta variant (3 resident per SM), a warp of the warp variant (8
// per CTA, one CTA per SM: the groups' shares of shared memory set the residency). Each group owns
// workspace slab blockIdx.x * groups + GID and act_smem bytes of the dynamic shared memory.
// kTraj: tppnp's trajectory loop per zone (IntegrateArgs::npts > 0); a separate instantiation so the
// single-interval kernel keeps its own register allocation. The trajectory instantiation also runs
// the serving loop (IntegrateArgs::queue), whose requests are single intervals or trajectories.
// One zone (or one served request) for the calling group: inputs from the arrays of A indexed by
// zone zq, or from the serving queue's slot of request zq; integrate; write the outputs back.
template <bool kTraj>
__device__ __forceinline__ void run_zone(const DevNet &N, const Ws &W, const IntegrateArgs &A, bool queue,
                                         long long zq, char *smem, int act_smem, double *sred, int *sint) {
  const ServeQueue &Q = A.queue;
  // the zone's inputs: arrays indexed by zone, or a queue slot (rewritten by copies between
  // requests, so read around L1)
  int z = 0, slot = 0, kind = kTraj ? 1 : 0, npts = A.npts, st = 0;
  double t9_0 = 0, t9_1 = 0, rho_0 = 0, rho_1 = 0, ye = 0, dtwant = 0;
  const double *tt = nullptr, *tp = nullptr, *tr = nullptr;
  bool seq_ok = true;
  if (queue) {
    slot = (int)(zq % Q.nslots);
    const RingIn *in = Q.in + slot;
    for (int it = 0; __ldcg(&in->seq) != zq; ++it)
      if (it > kSpinLimit) { seq_ok = false; break; }
    kind = __ldcg(&in->kind);
    npts = __ldcg(&in->npts);
    st = __ldcg(&in->bd);
    t9_0 = __ldcg(&in->t9_0); t9_1 = __ldcg(&in->t9_1);
    rho_0 = __ldcg(&in->rho_0); rho_1 = __ldcg(&in->rho_1);
    ye = __ldcg(&in->ye); dtwant = __ldcg(&in->dtwant);
    const double *g = Q.grid + (size_t)slot * 3 * Q.npts_max;
    tt = g; tp = g + Q.npts_max; tr = g + 2 * Q.npts_max;
    const double *x = Q.x_in + (size_t)slot * N.nsp;
    for (int s = GT; s < N.nsp; s += GN) W.y[s] = __ldcg(x + s);
  } else {
    z = (int)zq;
    st = A.bd_state ? A.bd_state[z] : 0;
    ye = A.ye[z];
    if (kTraj) {
      tt = A.tr_time + (size_t)z * A.npts; tp = A.tr_t9 + (size_t)z * A.npts; tr = A.tr_rho + (size_t)z * A.npts;
    } else {
      t9_0 = A.t9_0[z]; t9_1 = A.t9_1[z]; rho_0 = A.rho_0[z]; rho_1 = A.rho_1[z]; dtwant = A.dtwant[z];
    }
    for (int s = GT; s < N.nsp; s += GN) W.y[s] = A.X[(size_t)z * A.ldx + s];
  }
  GSYNC();
  ZoneCtl C;
  memset(&C.st, 0, sizeof(C.st));
  C.kopt = (st >= 2 && st <= N.kmax) ? st : N.kopt0;
  C.reduce = false;
  C.sumerr = 0.0;
  C.smem = smem;
  C.smem_bytes = act_smem;
  C.sint = sint;
  C.rates_ver = 0;
  C.built_ver = -1;
  C.act_ok = false;
  nse_reset(C.nse);
  int ierr, fail = -1;
  if (!seq_ok) {
    ierr = NUPPN_BAD_INPUT;
  } else if (kTraj && kind == 1) {
    // the trajectory loop of tppnp (tppnp.F90:131-168) for this zone
    if (fabs(1.0 - vsum(W.y, N.nsp, sred)) > 1.e-8) dev_renorm_ksum(W.y, N.nsp, sred);
    bool frst = st <= 0;
    ierr = 0;
    for (int i = 1; i < npts; ++i) {
      ye = dev_ye(N, W.y, sred);
      ierr = dev_integrate_zone(N, W, C, __ldcg(tp + i - 1), __ldcg(tp + i), __ldcg(tr + i - 1), __ldcg(tr + i), ye,
                                __ldcg(tt + i) - __ldcg(tt + i - 1), frst, sred);
      frst = false;
      if (ierr != 0) {
        fail = i - 1;
        break;
      }
      if (fabs(1.0 - vsum(W.y, N.nsp, sred)) > 5.e-7) dev_renorm_ksum(W.y, N.nsp, sred);
    }
  } else {
    ierr = dev_integrate_zone(N, W, C, t9_0, t9_1, rho_0, rho_1, ye, dtwant, st <= 0, sred);
  }
  if (queue) {
    // results to host-mapped memory, made visible to the host before `done`
    double *xo = Q.x_out + (size_t)slot * N.nsp;
    for (int s = GT; s < N.nsp; s += GN) xo[s] = W.y[s];
    RingOut *o = Q.out + slot;
    if (GT == 0) {
      o->ierr = ierr;
      o->fail = fail;
      o->bd = C.kopt;
      o->ye = ye;
      o->st = C.st;
    }
    __threadfence_system();
    GSYNC();
    if (GT == 0) *(volatile long long *)&o->done = zq + 1;
    return;
  }
  for (int s = GT; s < N.nsp; s += GN) A.X[(size_t)z * A.ldx + s] = W.y[s];
  if (GT == 0) {
    A.ye[z] = ye;
    A.ierr[z] = ierr;
    if (A.stats) A.stats[z] = C.st;
    if (A.bd_state) A.bd_state[z] = C.kopt;
    if (A.tr_fail) A.tr_fail[z] = fail;
  }
}

// One zone per group: a CTA of the cta variant (3 resident per SM), a warp of the warp variant (8
// per CTA, one CTA per SM: the groups' shares of shared memory set the residency). Each group owns
// workspace slab blockIdx.x * groups + GID and act_smem bytes of the dynamic shared memory.
// kTraj: tppnp's trajectory loop per zone (IntegrateArgs::npts > 0); a separate instantiation so the
// single-interval kernel keeps its own register allocation. The trajectory instantiation also runs
// the serving loop (IntegrateArgs::queue), whose requests are single intervals or trajectories.
template <bool kTraj>
__global__ void NUPPN_INTEGRATE_BOUNDS k_integrate(const __grid_constant__ DevNet N, const __grid_constant__ WsLayout L,
                                                   char *ws, const __grid_constant__ IntegrateArgs A, int act_smem) {
  extern __shared__ __align__(16) char smem_dyn[];
  __shared__ double sred_g[NUPPN_MAX_GROUPS][32];
  __shared__ int sint_g[NUPPN_MAX_GROUPS][32];
  __shared__ long long zsh_g[NUPPN_MAX_GROUPS];
  double *sred = sred_g[GID];
  int *sint = sint_g[GID];
  long long &zsh = zsh_g[GID];
  const int groups = (int)blockDim.x / GN;
  const Ws W = ws_bind(ws + ((size_t)blockIdx.x * groups + GID) * L.bytes, L);
  const bool queue = kTraj && A.queue.in != nullptr;
  for (;;) {
    GSYNC();
    if (GT == 0) {
      if (queue) {
        zsh = queue_claim(A.queue);
      } else {
        const int k = atomicAdd(A.counter, 1);
        zsh = (k < A.nz && A.order) ? A.order[k] : k;
      }
    }
    GSYNC();
    const long long zq = zsh;
    if (queue ? zq < 0 : zq >= A.nz) break;
    run_zone<kTraj>(N, W, A, queue, zq, smem_dyn + (size_t)GID * act_smem, act_smem, sred, sint);
  }
}

#if !NUPPN_GROUP_WARP
// Zones of several networks in one launch (one zone per CTA): zone z uses network A.net_of[z], whose
// DevNet and workspace layout the CTA copies from A.nets / A.lays into shared memory when it takes
// the zone; every CTA's slab is A.slab bytes, the largest of the networks' slabs.
__global__ void __launch_bounds__(256, 3) k_integrate_multi(const __grid_constant__ IntegrateArgs A, char *ws,
                                                            int act_smem) {
  extern __shared__ __align__(16) char smem_dyn[];
  __shared__ double sred[32];
  __shared__ int sint[32];
  __shared__ long long zsh;
  __shared__ __align__(16) DevNet sN;
  __shared__ __align__(16) WsLayout sL;
  char *slab = ws + (size_t)blockIdx.x * A.slab;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const int k = atomicAdd(A.counter, 1);
      zsh = (k < A.nz && A.order) ? A.order[k] : k;
    }
    __syncthreads();
    const long long zq = zsh;
    if (zq >= A.nz) break;
    const int nid = A.net_of[zq];
    if (nid < 0 || nid >= A.nnets) {  // no such network: the zone is left as it is
      if (threadIdx.x == 0) A.ierr[zq] = NUPPN_BAD_INPUT;
      continue;
    }
    {  // the zone's network description (8-byte words; both structs are 8-byte aligned)
      const unsigned long long *src = (const unsigned long long *)(A.nets + nid);
      unsigned long long *dst = (unsigned long long *)&sN;
      for (int i = threadIdx.x; i < (int)(sizeof(DevNet) / 8); i += blockDim.x) dst[i] = src[i];
      const unsigned long long *srl = (const unsigned long long *)(A.lays + nid);
      unsigned long long *dl = (unsigned long long *)&sL;
      for (int i = threadIdx.x; i < (int)(sizeof(WsLayout) / 8); i += blockDim.x) dl[i] = srl[i];
    }
    __syncthreads();
    const Ws W = ws_bind(slab, sL);
    run_zone<false>(sN, W, A, false, zq, smem_dyn, act_smem, sred, sint);
  }
}
#endif

#if !NUPPN_GROUP_WARP
__global__ void __launch_bounds__(256) k_phase(const __grid_constant__ DevNet N, const __grid_constant__ WsLayout L,
                                               char *ws, const __grid_constant__ PhaseArgs A, int act_smem) {
  extern __shared__ __align__(16) char smem_dyn[];
  __shared__ double sred[32];
  __shared__ int sint[32];
  const Ws W = ws_bind(ws + (size_t)blockIdx.x * L.bytes, L);
  const int tid = GT, nt = GN;
  for (int z = blockIdx.x; z < A.nz; z += gridDim.x) {
    if (A.X)
      for (int s = tid; s < N.nsp; s += nt) W.y[s] = A.X[(size_t)z * A.ldx + s];
    if (A.v_in)
      for (int l = tid; l < N.nre; l += nt) W.v[l] = A.v_in[(size_t)z * N.nre + l];
    GSYNC();
    if (A.op == 0) {
      dev_eval_rates(N, W, A.t9[z], A.rho[z], A.ye[z], W.y, sred);
      for (int l = tid; l < N.nre; l += nt) A.out_v[(size_t)z * N.nre + l] = W.v[l];
    } else if (A.op == 1) {
      dev_dxdt(N, W, W.y, W.dxdt);
      for (int s = tid; s < N.nsp; s += nt) A.out_dxdt[(size_t)z * N.nsp + s] = W.dxdt[s];
    } else if (A.op == 2) {
      dev_jacobian(N, W, A.dt[z], W.y);
      for (int e = tid; e < N.nnzJ; e += nt) {
        A.out_jac[(size_t)z * N.nnzJ + e] = W.jac[e];
        A.out_eset[(size_t)z * N.nnzJ + e] = W.eset[e];
      }
      for (int s = tid; s < N.nsp; s += nt) A.out_mask[(size_t)z * N.nsp + s] = W.mask[s];
    } else if (A.op == 3) {
      for (int e = tid; e < N.nnzJ; e += nt) {
        W.jac[e] = A.jac_in[(size_t)z * N.nnzJ + e];
        W.eset[e] = A.eset_in[(size_t)z * N.nnzJ + e];
      }
      for (int s = tid; s < N.nsp; s += nt) {
        W.mask[s] = A.mask_in[(size_t)z * N.nsp + s];
        W.rhs[s] = A.b[(size_t)z * N.nsp + s];
      }
      GSYNC();
      Act act;
      dev_compact(N, W, act, smem_dyn, act_smem, sint);
      dev_load_active_jacobian(N, W, act);
      bool ok = dev_factor_active(N, W, act, A.dt[z]);
      ok = dev_solve_species(N, act, W.rhs, W.dxdt) && ok;
      for (int s = tid; s < N.nsp; s += nt) A.out_x[(size_t)z * N.nsp + s] = ok ? W.dxdt[s] : NAN;
    } else if (A.op == 4) {
      NseCtl S;
      nse_reset(S);
      double mu_p, mu_n;
      int it;
      const int ierr = dev_compute_nse(N, W, S, A.t9[z], A.rho[z], A.ye[z], W.nse_y1, mu_p, mu_n, it, sred);
      for (int s = tid; s < N.nsp; s += nt) A.out_x[(size_t)z * N.nsp + s] = ierr == 0 ? W.nse_y1[s] : 0.0;
      if (tid == 0) {
        A.out_mu_p[z] = mu_p;
        A.out_mu_n[z] = mu_n;
        A.out_iters[z] = it;
        A.out_ierr[z] = ierr;
      }
    }
    GSYNC();
  }
}

// Zone schedule for k_integrate: a counting sort of the zones on log2 T9 (64 bins per octave over
// 2^-12 .. 2^4), hottest first. Hot zones have the largest dynamic networks and the most rejected
// steps, and a persistent kernel ends when its last zone does: starting the costliest zones first
// keeps one of them from starting late and running alone at the end. key[z * stride] (and, if
// key_b is given, the larger of it and key_b[z * stride]) is the zone's temperature. One CTA; the
// order within a bin follows the atomics, which is harmless: a zone's result does not depend on
// which CTA integrates it or when.
constexpr int kOrderBins = 1024;
__global__ void __launch_bounds__(1024) k_zone_order(const double *key, const double *key_b, int stride, int nz,
                                                     int *order) {
  __shared__ int cnt[kOrderBins];
  for (int b = GT; b < kOrderBins; b += GN) cnt[b] = 0;
  GSYNC();
  auto bin_of = [&](int z) {
    double t = key[(size_t)z * stride];
    if (key_b) t = fmax(t, key_b[(size_t)z * stride]);
    if (!(t > 0.0) || !isfinite(t)) return kOrderBins - 1;  // rejected by the kernel at once: last
    const double u = (log2(t) + 12.0) * 64.0;
    const int b = u <= 0.0 ? 0 : (u >= kOrderBins - 1 ? kOrderBins - 1 : (int)u);
    return kOrderBins - 1 - b;  // hottest first
  };
  for (int z = GT; z < nz; z += GN) atomicAdd(&cnt[bin_of(z)], 1);
  GSYNC();
  if (GT == 0) {  // exclusive offsets (1024 bins: a serial pass is a few microseconds)
    int acc = 0;
    for (int b = 0; b < kOrderBins; ++b) {
      const int c = cnt[b];
      cnt[b] = acc;
      acc += c;
    }
  }
  GSYNC();
  for (int z = GT; z < nz; z += GN) order[atomicAdd(&cnt[bin_of(z)], 1)] = z;
}

cudaError_t launch_zone_order(const double *key, const double *key_b, int stride, int nz, int *order,
                              cudaStream_t st) {
  k_zone_order<<<1, 1024, 0, st>>>(key, key_b, stride, nz, order);
  return cudaGetLastError();
}

#endif  // !NUPPN_GROUP_WARP

// act_smem: shared-memory bytes of each group; the launch gives every group of the CTA its share.
cudaError_t launch_integrate(const DevNet &N, const WsLayout &L, char *ws, int grid, int block, int act_smem,
                             const IntegrateArgs &A, cudaStream_t st) {
  const size_t dyn = (size_t)act_smem * NUPPN_GROUPS_PER_CTA(block);
  if (A.npts > 0) k_integrate<true><<<grid, block, dyn, st>>>(N, L, ws, A, act_smem);
  else k_integrate<false><<<grid, block, dyn, st>>>(N, L, ws, A, act_smem);
  return cudaGetLastError();
}

#if !NUPPN_GROUP_WARP
cudaError_t launch_integrate_multi(const IntegrateArgs &A, char *ws, int grid, int act_smem, cudaStream_t st) {
  k_integrate_multi<<<grid, 256, act_smem, st>>>(A, ws, act_smem);
  return cudaGetLastError();
}

cudaError_t occupancy_integrate_multi(int act_smem, int *per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_integrate_multi, 256, act_smem);
}

cudaError_t launch_phase(const DevNet &N, const WsLayout &L, char *ws, int grid, int block, int act_smem,
                         const PhaseArgs &A, cudaStream_t st) {
  k_phase<<<grid, block, act_smem, st>>>(N, L, ws, A, act_smem);
  return cudaGetLastError();
}
#endif

// dyn_smem: dynamic shared memory of a whole CTA
cudaError_t configure_kernels(int dyn_smem) {
  cudaError_t e = cudaFuncSetAttribute(k_integrate<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_integrate<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
#if !NUPPN_GROUP_WARP
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_phase, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_integrate_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_smem);
#endif
  return e;
}

// CTAs of `block` threads resident per SM when every group has act_smem bytes of shared memory
cudaError_t occupancy_integrate(int block, int act_smem, int *per_sm) {
  // the smaller of the two instantiations' residencies, so that a grid sized by it is resident with
  // either (the serving loop runs the trajectory instantiation)
  const size_t dyn = (size_t)act_smem * NUPPN_GROUPS_PER_CTA(block);
  int a = 0, b = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_integrate<false>, block, dyn);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_integrate<true>, block, dyn);
  *per_sm = a < b ? a : b;
  return e;
}

NUPPN_END
