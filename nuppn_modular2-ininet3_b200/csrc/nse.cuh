// nse.cuh -- nuclear statistical equilibrium on the device (included by solver.cu).
//
// compute_nse (physics/source/nse_swj.F90:272-384) and the weak-rate coupling of Ye in NSE
// (solver/source/nse_solver.F90:33-291), per zone by one CTA. The NSE isotopes are evaluated
// block-parallel; the 2x2 Newton system in (mu_p, mu_n), the Runge-Kutta stages and the step control
// are scalar and evaluated identically by every thread. Sums over the isotopes use a fixed tree (the
// reference sorts before summing, which changes only the last bits); the Ye derivative reproduces
// the reference's sorted, position-masked sum (dev_nse_yedot), whose mask changes which terms count.
#pragma once

NUPPN_BEGIN

// state that the reference keeps in module variables of nse_swj (nse_mu, nse_mu_last, first, ...)
struct NseCtl {
  double mu[2], mu_last[2], mu_p_coul, the, phi;
  bool first;
};

__device__ __forceinline__ void nse_reset(NseCtl &S) {
  S.mu[0] = S.mu[1] = 0.0;
  S.mu_last[0] = S.mu_last[1] = -9.0;
  S.mu_p_coul = S.the = S.phi = 0.0;
  S.first = true;
}

// K block sums at once (every thread returns the same values, partials combined in a fixed order);
// needs K * warps <= 32 doubles of sred.
template <int K>
__device__ void block_sum_k(double (&v)[K], double *sred) {
  const int lane = GT & 31, w = GT >> 5, nw = GN >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  GSYNC();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sred[k * nw + w] = v[k];
  GSYNC();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double r = 0.0;
    for (int i = 0; i < nw; ++i) r += sred[k * nw + i];
    v[k] = r;
  }
}

// coulomb_corrections (nse_swj.F90:545-580)
__device__ void dev_nse_coulomb(const DevNet &N, const Ws &W, NseCtl &S, double t9, double rho, double ye) {
  const double a1 = -0.9052, a2 = 0.6322, a3 = -0.5 * sqrt(3.0) - a1 / sqrt(a2);
  const double kT_erg = K_BOLTZMANN * t9 * 1.e9, kT_mev = kT_erg * K_ERG2MEV;
  const double ae = pow(4.0 * K_PI * rho * ye * K_AVOGADRO / 3.0, -(1.0 / 3.0));
  const double Gam_e = K_QE * K_QE / kT_erg / ae;
  for (int j = GT; j < N.nse_num; j += GN) {
    const double G = Gam_e * pow(N.nse_z[j], 5.0 * (1.0 / 3.0));
    const double mc = a1 * (sqrt(G * (a2 + G)) - a2 * log(sqrt(G / a2) + sqrt(1.0 + G / a2))) +
                      2.0 * a3 * (sqrt(G) - atan(sqrt(G)));
    W.nse_mc[j] = mc * kT_mev;
  }
  GSYNC();
  S.mu_p_coul = W.nse_mc[N.nse_iprot];
}

// partition_functions (nse_swj.F90:585-597) with reaclib_interpolate_partition_functions
// (reaclib.F90:586-605): g_tot = G(T9) * (2J+1), G = 1 without a partition row.
__device__ void dev_nse_partition(const DevNet &N, const Ws &W, double t9) {
  if (N.npart > 0) {
    const double t9c = fmax(N.pt9[0], fmin(t9, N.pt9[kPartDim - 1]));
    const int i0 = bsearch_r8(N.pt9, kPartDim, t9c);
    const double t90 = N.pt9[i0 - 1], t91 = N.pt9[i0];
    const double Dt9 = (t9c - t90) / (t91 - t90);
    for (int p = GT; p < N.npart; p += GN) {
      const double *pv = N.pval + (size_t)p * kPartDim;
      W.partinter[p] = pv[i0 - 1] + (pv[i0] - pv[i0 - 1]) * Dt9;
    }
  }
  GSYNC();
  for (int j = GT; j < N.nse_num; j += GN) {
    const int p = N.nse_part[j];
    W.nse_gtot[j] = (p >= 0 ? W.partinter[p] : 1.0) * N.nse_g[j];
  }
  GSYNC();
}

// nse_distribution (nse_swj.F90:524-541) into W.nse_x
__device__ void dev_nse_dist(const DevNet &N, const Ws &W, const NseCtl &S, double mu_p, double mu_n, double t9,
                             double rho) {
  const double kT_erg = K_BOLTZMANN * t9 * 1.e9, kT_mev = kT_erg * K_ERG2MEV;
  for (int j = GT; j < N.nse_num; j += GN) {
    const double m = N.nse_m[j];
    const double lam = sqrt(K_PLANCK_ERG * K_PLANCK_ERG / (2.0 * K_PI * m * kT_erg));
    const double fac = N.nse_z[j] * (mu_p + S.mu_p_coul) + N.nse_n[j] * mu_n - W.nse_mc[j] + N.nse_q[j];
    const double pre = m / rho * W.nse_gtot[j] / (lam * lam * lam);
    W.nse_x[j] = pre * exp(fac / kT_mev);
  }
  GSYNC();
}

// calculate_rhs (nse_swj.F90:510-520): theta = sum X - 1, phi = sum (Z/A) X - Ye
__device__ void dev_nse_rhs(const DevNet &N, const Ws &W, NseCtl &S, double ye, double *sred) {
  double v[2] = {0.0, 0.0};
  for (int j = GT; j < N.nse_num; j += GN) {
    v[0] += W.nse_x[j];
    v[1] += N.nse_zoa[j] * W.nse_x[j];
  }
  block_sum_k<2>(v, sred);
  S.the = v[0] - 1.0;
  S.phi = v[1] - ye;
}

// calculate_jac (nse_swj.F90:483-506)
__device__ void dev_nse_jac(const DevNet &N, const Ws &W, double t9, double (&jac)[2][2], double *sred) {
  const double kT_mev = K_BOLTZMANN * t9 * 1.e9 * K_ERG2MEV;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = GT; j < N.nse_num; j += GN) {
    const double dp = W.nse_x[j] * N.nse_z[j] / kT_mev, dn = W.nse_x[j] * N.nse_n[j] / kT_mev;
    v[0] += dp;
    v[1] += dn;
    v[2] += N.nse_zoa[j] * dp;
    v[3] += N.nse_zoa[j] * dn;
  }
  block_sum_k<4>(v, sred);
  jac[0][0] = v[0];
  jac[0][1] = v[1];
  jac[1][0] = v[2];
  jac[1][1] = v[3];
}

// Crout LU with implicit partial pivoting and its back substitution for the 2x2 Jacobian
// (ludcmp_nse / lubksb_nse, nse_swj.F90:751-883). Returns false for a zero row.
__device__ bool nse_lu2(double (&a)[2][2], int (&indx)[2]) {
  double vv[2];
  for (int i = 0; i < 2; ++i) {
    const double aamax = fmax(fabs(a[i][0]), fabs(a[i][1]));
    if (aamax == 0.0) return false;
    vv[i] = 1.0 / aamax;
  }
  for (int j = 0; j < 2; ++j) {
    for (int i = 0; i < j; ++i) {
      double sum = a[i][j];
      for (int k = 0; k < i; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
    }
    double aamax = 0.0;
    int imax = j;
    for (int i = j; i < 2; ++i) {
      double sum = a[i][j];
      for (int k = 0; k < j; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
      const double dum = vv[i] * fabs(sum);
      if (dum >= aamax) {
        imax = i;
        aamax = dum;
      }
    }
    if (j != imax) {
      for (int k = 0; k < 2; ++k) {
        const double t = a[imax][k];
        a[imax][k] = a[j][k];
        a[j][k] = t;
      }
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (a[j][j] == 0.0) a[j][j] = 1.0e-20;
    if (j != 1) {
      const double dum = 1.0 / a[j][j];
      a[1][j] = a[1][j] * dum;
    }
  }
  return true;
}

__device__ void nse_lub2(const double (&a)[2][2], const int (&indx)[2], double (&b)[2]) {
  int ii = -1;
  for (int i = 0; i < 2; ++i) {
    const int ll = indx[i];
    double sum = b[ll];
    b[ll] = b[i];
    if (ii >= 0) {
      for (int j = ii; j < i; ++j) sum = sum - a[i][j] * b[j];
    } else if (sum != 0.0) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = 1; i >= 0; --i) {
    double sum = b[i];
    for (int j = i + 1; j < 2; ++j) sum = sum - a[i][j] * b[j];
    b[i] = sum / a[i][i];
  }
}

// solve_nse (nse_swj.F90:388-460): Newton on (theta, phi) in (mu_p, mu_n) with a x1e-2 line search,
// starting from W.nse_x and S.mu = (mu_p, mu_n).
__device__ int dev_solve_nse(const DevNet &N, const Ws &W, NseCtl &S, double t9, double rho, double ye,
                             double &mu_p, double &mu_n, int &it, int max_iter, double *sred) {
  const int lnsrchmax = 100;
  S.mu[0] = mu_p;
  S.mu[1] = mu_n;
  for (int i = 1; i <= max_iter; ++i) {
    it = i;
    const double mu_old0 = S.mu[0], mu_old1 = S.mu[1];
    dev_nse_rhs(N, W, S, ye, sred);
    const double the_old = S.the, phi_old = S.phi;
    double jac[2][2];
    dev_nse_jac(N, W, t9, jac, sred);
    int indx[2];
    if (!nse_lu2(jac, indx)) return BAD_STEP;
    double del[2] = {S.the, S.phi};
    nse_lub2(jac, indx, del);
    double gamma = 1.0;
    for (int j = 1; j <= lnsrchmax; ++j) {
      if (j == lnsrchmax) return NSE_CNVRG;
      S.mu[0] = mu_old0 - gamma * del[0];
      S.mu[1] = mu_old1 - gamma * del[1];
      dev_nse_dist(N, W, S, S.mu[0], S.mu[1], t9, rho);
      dev_nse_rhs(N, W, S, ye, sred);
      if (fabs(S.the) > 1.e10 * fabs(the_old) + 1.e-10 || fabs(S.phi) > 1.e10 * fabs(phi_old) + 1.e-10)
        gamma = gamma * 1.e-2;
      else
        break;
    }
    if (fabs(S.the) <= 1.e-9 && fabs(S.phi) <= 1.e-9) break;
    if (i == max_iter) return NSE_CNVRG;
  }
  mu_p = S.mu[0];
  mu_n = S.mu[1];
  return 0;
}

// initial_guess with ni56_initial (nse_swj.F90:466-478): X(Ni56) = 1 and mu_p = mu_n, or the last
// converged solution of this zone.
__device__ void dev_nse_initial_guess(const DevNet &N, const Ws &W, NseCtl &S, double &mu_p, double &mu_n,
                                      double t9, double rho) {
  if (!S.first) {
    S.mu[0] = S.mu_last[0];
    S.mu[1] = S.mu_last[1];
    mu_p = S.mu[0];
    mu_n = S.mu[1];
    return;
  }
  const double kT_erg = K_BOLTZMANN * t9 * 1.e9, kT_mev = kT_erg * K_ERG2MEV;
  const int j = N.nse_ini56;
  const double m = N.nse_m[j];
  const double lam = sqrt(K_PLANCK_ERG * K_PLANCK_ERG / (2.0 * K_PI * m * kT_erg));
  mu_p = kT_mev * log(1.0 * rho * powi(lam, 3) / W.nse_gtot[j] / m) - N.nse_q[j] + W.nse_mc[j] - N.nse_z[j] * S.mu_p_coul;
  mu_p = mu_p / (N.nse_z[j] + N.nse_n[j]);
  mu_n = mu_p;
}

// compute_nse (nse_swj.F90:272-384) into yps[nsp]. Where the reference stops the run after a failed
// temperature descent, the failure is returned as the outcome code.
__device__ int dev_compute_nse(const DevNet &N, const Ws &W, NseCtl &S, double t9in, double rho, double ye,
                               double *yps, double &mu_p, double &mu_n, int &iter, double *sred) {
  if (ye <= 0.0 || ye >= 1.0) return BAD_YE;
  mu_n = 0.0;
  mu_p = 0.0;
  iter = 0;
  int it = 0;
  double t9 = t9in;
  dev_nse_coulomb(N, W, S, t9, rho, ye);
  dev_nse_partition(N, W, t9);
  dev_nse_initial_guess(N, W, S, mu_p, mu_n, t9, rho);
  dev_nse_dist(N, W, S, mu_p, mu_n, t9, rho);
  int ierr = dev_solve_nse(N, W, S, t9, rho, ye, mu_p, mu_n, it, 100, sred);
  iter += it;
  if (ierr != 0) {  // temperature descent from T9 = 100 (nse_swj.F90:331-342)
    const int tsteps = 10;
    const double coeff = pow(100.0 / t9in, 1.0 / ((double)tsteps - 1.0));
    for (int i = 1; i <= tsteps; ++i) {
      t9 = t9in * powi(coeff, tsteps - i);
      dev_nse_coulomb(N, W, S, t9, rho, ye);
      dev_nse_partition(N, W, t9);
      if (i == 1) dev_nse_initial_guess(N, W, S, mu_p, mu_n, t9, rho);
      dev_nse_dist(N, W, S, mu_p, mu_n, t9, rho);
      ierr = dev_solve_nse(N, W, S, t9, rho, ye, mu_p, mu_n, it, 500, sred);
      iter += it;
    }
    if (ierr != 0) return ierr == BAD_STEP ? BAD_STEP : NSE_CNVRG;
  }
  dev_nse_dist(N, W, S, mu_p, mu_n, t9, rho);
  for (int s = GT; s < N.nsp; s += GN) yps[s] = 1.e-99;
  GSYNC();
  for (int j = GT; j < N.nse_num; j += GN) yps[N.nse_idx[j]] = fmax(W.nse_x[j], 1e-99);
  GSYNC();
  S.mu_last[0] = S.mu[0];
  S.mu_last[1] = S.mu[1];
  S.first = false;
  return 0;
}

__device__ __forceinline__ bool weak_label(int lab) {  // ilabb of the weak reactions kept in NSE
  return lab == i_bm || lab == i_ec || lab == i_ve || lab == i_vp;
}

// nse_solver_cache_lm_ov_a (nse_solver.F90:33-66): keep only the weak rates in W.v, and for each
// parent sum (lambda_beta - lambda_ec) / A over its reactions in reaction order (the k1 lists).
__device__ void dev_nse_cache_lm(const DevNet &N, const Ws &W) {
  for (int l = GT; l < N.nre; l += GN)
    if (!weak_label(N.ilabb[l])) W.v[l] = 0.0;
  GSYNC();
  for (int s = GT; s < N.nsp; s += GN) {
    double acc = 0.0;
    for (int p = N.k1_ptr[s]; p < N.k1_ptr[s + 1]; ++p) {
      const int a = N.k1_list[p];
      const double lm = W.v[N.act_slot[a]];
      if (lm == 0.0) continue;
      const int dau = N.act_k[(size_t)a * 8 + 6];
      if (N.zn[s] < N.zn[dau]) acc = acc + lm / N.an[s];
      else acc = acc - lm / N.an[s];
    }
    W.nse_lm[s] = acc;
  }
  GSYNC();
}

// yedot (nse_solver.F90:104-113): sortedsum(x * lm_ov_a, mask = considerisotope). The reference's
// sortedsum tests the mask at the sorted position (utils.F90:489-495), so the terms left out are
// those whose rank matches an unconsidered species' index; the values are sorted here (bitonic, in
// shared memory when it fits) to leave out the same terms.
__device__ double dev_nse_yedot(const DevNet &N, const Ws &W, const double *x, char *smem, size_t smem_bytes,
                                double *sred) {
  const int tid = GT, nt = GN, P = N.nse_p2;
  double *t = (size_t)P * 8 <= smem_bytes ? (double *)smem : W.nse_sort;
  for (int i = tid; i < P; i += nt) t[i] = i < N.nsp ? x[i] * W.nse_lm[i] : INFINITY;
  GSYNC();
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P; i += nt) {
        const int l = i ^ j;
        if (l > i) {
          const double a = t[i], b = t[l];
          if (((i & k) == 0) ? (a > b) : (a < b)) {
            t[i] = b;
            t[l] = a;
          }
        }
      }
      GSYNC();
    }
  double v[1] = {0.0};
  for (int i = tid; i < N.nsp; i += nt)
    if (N.ciso[i]) v[0] += t[i];
  block_sum_k<1>(v, sred);
  return v[0];
}

// rk4_nse_step (nse_solver.F90:116-238): Cash-Karp Runge-Kutta for Ye in NSE; y1 gets the NSE
// abundances at the fifth-order Ye.
__device__ int dev_rk4_nse_step(const DevNet &N, const Ws &W, NseCtl &S, double dt, double rho, double t9,
                                double &ye, double *y1, double &error, char *smem, size_t smem_bytes, double *sred) {
  const double b21 = 1.0 / 5.0, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0, b41 = 3.0 / 10.0, b42 = -9.0 / 10.0,
               b43 = 6.0 * (1.0 / 5.0), b51 = -11.0 / 54.0, b52 = 5.0 * 0.5, b53 = -70.0 / 27.0, b54 = 35.0 / 27.0,
               b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0, b63 = 575.0 / 13824.0, b64 = 44275.0 / 110592.0,
               b65 = 253.0 / 4096.0, c1 = 37.0 / 378.0, c1s = 2825.0 / 27648.0, c2 = 0.0, c2s = 0.0,
               c3 = 250.0 / 621.0, c3s = 18575.0 / 48384.0, c4 = 125.0 / 594.0, c4s = 13525.0 / 55296.0, c5 = 0.0,
               c5s = 277.0 / 14336.0, c6 = 512.0 / 1771.0, c6s = 1.0 / 4.0;
  double mu_p, mu_n;
  int iters, ierr;
  const double ye_0 = ye;
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  const double k1 = dt * dev_nse_yedot(N, W, y1, smem, smem_bytes, sred);
  ye = ye_0 + (b21 * k1);
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  const double k2 = dt * dev_nse_yedot(N, W, y1, smem, smem_bytes, sred);
  ye = ye_0 + (b31 * k1 + b32 * k2);
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  const double k3 = dt * dev_nse_yedot(N, W, y1, smem, smem_bytes, sred);
  ye = ye_0 + (b41 * k1 + b42 * k2 + b43 * k3);
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  const double k4 = dt * dev_nse_yedot(N, W, y1, smem, smem_bytes, sred);
  ye = ye_0 + (b51 * k1 + b52 * k2 + b53 * k3 + b54 * k4);
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  const double k5 = dt * dev_nse_yedot(N, W, y1, smem, smem_bytes, sred);
  ye = ye_0 + (b61 * k1 + b62 * k2 + b63 * k3 + b64 * k4 + b65 * k5);
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  const double k6 = dt * dev_nse_yedot(N, W, y1, smem, smem_bytes, sred);
  const double ye_5th = ye_0 + c1 * k1 + c2 * k2 + c3 * k3 + c4 * k4 + c5 * k5 + c6 * k6;
  const double ye_4th = ye_0 + c1s * k1 + c2s * k2 + c3s * k3 + c4s * k4 + c5s * k5 + c6s * k6;
  ye = ye_5th;
  if ((ierr = dev_compute_nse(N, W, S, t9, rho, ye, y1, mu_p, mu_n, iters, sred)) != 0) return ierr;
  error = fabs(ye_5th - ye_4th);
  return 0;
}

// nse_yedot_rk4 (nse_solver.F90:72-101); yps gets the new NSE abundances on success
__device__ int dev_nse_rk4(const DevNet &N, const Ws &W, NseCtl &S, double *yps, double t9, double rho, double &ye,
                           double dt, double &dtrcmd, char *smem, size_t smem_bytes, double *sred) {
  const double maxfac = 2.0, minfac = 0.1, ye_tol = 1.e-5;
  const double ye_old = ye;
  double error = 0.0, fac;
  int ierr = dev_rk4_nse_step(N, W, S, dt, rho, t9, ye, W.nse_y1, error, smem, smem_bytes, sred);
  if (ierr != 0) error = ye_old;
  if (ierr != 0 || ye < 0.0 || ye > 1.0) {
    ierr = BAD_YE;
    fac = 0.5 * pow(fabs(ye_tol * ye_old / fmax(error, K_SMALL)), 1.0 / 5.0);
  } else if (error / ye > ye_tol) {
    ierr = NSE_WEAK;
    fac = 0.5 * pow(fabs(ye_tol * ye / fmax(error, K_SMALL)), 1.0 / 5.0);
  } else {
    ierr = 0;
    fac = pow(fabs(ye_tol * ye / fmax(error, K_SMALL)), 1.0 / 5.0);
    for (int s = GT; s < N.nsp; s += GN) yps[s] = W.nse_y1[s];
  }
  GSYNC();
  dtrcmd = dt * fmax(fmin(fac, maxfac), minfac);
  return ierr;
}

// nse_yedot_euler (nse_solver.F90:241-289)
__device__ int dev_nse_euler(const DevNet &N, const Ws &W, NseCtl &S, double *yps, double t9, double rho, double &ye,
                             double dt, double &dtrcmd, char *smem, size_t smem_bytes, double *sred) {
  const double deltamax = 1.e-5;
  double mu_p, mu_n;
  int iters;
  int ierr = dev_compute_nse(N, W, S, t9, rho, ye, W.nse_y1, mu_p, mu_n, iters, sred);
  if (ierr != 0 || ye < 0.0 || ye > 1.0) {
    dtrcmd = 0.1 * dt;
    return BAD_STEP;
  }
  const double dyedt = dev_nse_yedot(N, W, W.nse_y1, smem, smem_bytes, sred);
  const double d_ye = dyedt * dt;
  if (d_ye > deltamax) {
    dtrcmd = deltamax / fabs(dyedt);
    return NSE_WEAK;
  }
  ye = ye + d_ye;
  ierr = dev_compute_nse(N, W, S, t9, rho, ye, W.nse_y1, mu_p, mu_n, iters, sred);
  if (ierr == 0)
    for (int s = GT; s < N.nsp; s += GN) yps[s] = W.nse_y1[s];
  else
    ierr = NSE_CNVRG;
  GSYNC();
  dtrcmd = deltamax / fabs(dyedt);
  return ierr;
}

NUPPN_END
