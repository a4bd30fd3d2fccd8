// integrator.cuh -- step control on the device (included by solver.cu after the phase kernels).
//
// backward_euler_newton / newton_iteration   solver/source/backward_euler.F90:29-176
// bader_deuflhard_integration and helpers   solver/source/bader_deuflhard.F90:139-488
// integrate_network / do_one_time_step      solver/source/solver.F90:53-274
//
// All threads of the CTA run this control flow with identical scalars. Within one step only the
// species of the dynamic network change (the reference's correction is zero elsewhere,
// ddecompac, jac_rhs.F90:584-608), so the Bader-Deuflhard vectors are kept on the active rows only;
// for frozen species the extrapolation tableau is exact (a constant column), their error terms are
// zero, and their share of the mass sum and of the negative-abundance test is a per-step constant.
#pragma once

NUPPN_BEGIN

struct ZoneCtl {
  nuppn_zone_stats st;
  int kopt;
  bool reduce;
  double sumerr;  // kept between levels like the reference's module variable
  double err[kMaxLevels + 1];
  double xhist[kMaxLevels + 1];
  char *smem;     // dynamic shared memory for the active subsystem
  int smem_bytes;
  int *sint;      // shared scan scratch (>= 32 ints)
  Act act;        // active subsystem of the current Jacobian
  NseCtl nse;     // NSE solver state of the zone (kept across its NSE calls within one call)
  // The active subsystem's structure and right-hand side items depend only on the mask, the rates
  // and the frozen species' abundances; when none changed since they were built they are kept.
  int rates_ver;  // incremented by every rate evaluation
  int built_ver;  // rates_ver when act was built; act_ok: act's shared memory still holds it
  bool act_ok;
};

__device__ void vcopy(double *dst, const double *src, int n) {
  for (int i = GT; i < n; i += GN) dst[i] = src[i];
  GSYNC();
}

__device__ double vsum(const double *a, int n, double *sred) {
  double s = 0.0;
  for (int i = GT; i < n; i += GN) s += a[i];
  return block_sum(s, sred);
}

__device__ double vmaxneg(const double *a, int n, double *sred) {
  double m = -DBL_MAX;
  for (int i = GT; i < n; i += GN) m = fmax(m, -a[i]);
  return block_max(m, sred);
}

// ypsplus (utils.F90:726-740)
__device__ void ypsplus(double *y, int n) {
  for (int i = GT; i < n; i += GN) {
    double v = y[i];
    if (v < -1.e-27) v = 1.e-99;
    if (v < 1.e-27) v = 1.e-99;
    y[i] = v;
  }
  GSYNC();
}

// renorm_1d (utils.F90:436-446): y / ksum(y), the Kahan sum (utils.F90:670-685) taken in order
__device__ void dev_renorm_ksum(double *y, int n, double *sred) {
  if (GT == 0) {
    double c = 0.0, s = 0.0;
    for (int i = 0; i < n; ++i) {
      const double yy = y[i] - c;
      const double t = s + yy;
      c = (t - s) - yy;
      s = t;
    }
    sred[0] = s;
  }
  GSYNC();
  const double s = sred[0];
  GSYNC();
  for (int i = GT; i < n; i += GN) y[i] = y[i] / s;
  GSYNC();
}

// calculate_ye (utils.F90:537-553)
__device__ double dev_ye(const DevNet &N, const double *x, double *sred) {
  double s = 0.0;
  for (int i = GT; i < N.nsp; i += GN)
    if (N.ciso[i]) s += (N.an[i] - 2.0 * N.zn[i]) * x[i] / N.an[i];
  s = block_sum(s, sred);
  return (1.0 - s) * 0.5;
}

// Jacobian pass, compaction, active Jacobian and restricted right-hand side for abundances y. The
// compaction and the right-hand side items are rebuilt only if the mask, the rates or a frozen
// species' abundance changed since the last build (about half the Jacobians of a He-shell zone keep
// all three); the Jacobian values are always new.
__device__ void dev_new_jacobian(const DevNet &N, const Ws &W, ZoneCtl &C, double dt, const double *y) {
  dev_jacobian_mask(N, W, dt, y);
  int same = C.act_ok && C.built_ver == C.rates_ver;
  if (same) {
    int diff = 0;
    for (int s = GT; s < N.nsp; s += GN)
      diff |= W.mask[s] != W.cache_mask[s] || (!W.mask[s] && W.xn[s] != W.cache_xn[s]);
    same = !g_or(diff);
  }
  if (!same) {
    dev_compact(N, W, C.act, C.smem, C.smem_bytes, C.sint);
    dev_compact_rhs(N, W, C.act, C.smem, C.smem_bytes, C.sint);
    for (int s = GT; s < N.nsp; s += GN) {
      W.cache_mask[s] = W.mask[s];
      W.cache_xn[s] = W.xn[s];
    }
    C.built_ver = C.rates_ver;
    C.act_ok = true;
  }
  dev_jacobian_active(N, W, C.act, C.sint);
  C.st.nvar1_last = C.act.na;
  C.st.nvar1_max = max(C.st.nvar1_max, C.act.na);
}

// ---------------------------------------------------------------------------------------------
__device__ int dev_backward_euler(const DevNet &N, const Ws &W, ZoneCtl &C, double *yps, double dt, double &dtrcmd,
                                  double *sred) {
  const int nsp = N.nsp, tid = GT, nt = GN;
  const double rmin = 0.2, rmax = 2.0, dgrd = N.kn.dgrd;
  const double sum_check = N.kn.grdthreshold * N.nvar * dgrd;
  double *yc = W.bd, *dxc = W.bd + N.nsys;
  for (int i = tid; i < nsp; i += nt) { W.y_new[i] = yps[i]; W.y_old[i] = yps[i]; W.y_cur[i] = yps[i]; }
  GSYNC();
  int iter = 0;
  double grd = 0.0;
  for (;;) {
    if (iter > N.kn.ittd) {
      double mneg = vmaxneg(W.y_new, nsp, sred), err, tol;
      double sumy = vsum(W.y_new, nsp, sred);
      int ierr;
      if (mneg >= sum_check) { err = mneg; tol = sum_check; ierr = NEG_ABUNDS; }
      else if (fabs(1.0 - sumy) > K_SUM_TOL) { err = fabs(1.0 - sumy); tol = K_SUM_TOL; ierr = SUM_X; }
      else { err = grd; tol = dgrd; ierr = SLV_CNVRG; }
      dtrcmd = fmax(fmin(pow(tol / fmax(err, K_SMALL), 0.5), rmax), rmin) * dt;
      return ierr;
    }
    // newton_iteration (backward_euler.F90:120-176) on the dynamic network
    dev_new_jacobian(N, W, C, dt, W.y_cur);
    Act &A = C.act;
    bool ok = dev_factor_active(N, W, A, dt);
    for (int c = tid; c < A.na; c += nt) yc[c] = W.y_cur[N.sp_of_sys[A.arow[c]]];
    GSYNC();
    dev_dxdt_active(A, yc, dxc);
    for (int c = tid; c < A.na; c += nt) {
      const int s = N.sp_of_sys[A.arow[c]];
      A.xs[c] = W.y_old[s] - W.y_cur[s] + dt * dxc[c];
    }
    GSYNC();
    ok = dev_solve_active(A) && ok;
    if (!ok) return BAD_STEP;
    C.st.nfact++; C.st.nsolve++;
    double g = 0.0;
    for (int c = tid; c < A.na; c += nt) {  // unmasked species keep y_new = y_cur (zero correction)
      const int s = N.sp_of_sys[A.arow[c]];
      const double yn = W.y_cur[s] + A.xs[c];
      W.y_new[s] = yn;
      if (W.y_cur[s] > N.kn.grdthreshold) g = fmax(g, fabs((yn - W.y_cur[s]) / W.y_cur[s]));
    }
    grd = block_max(g, sred);
    iter++;
    C.st.newton_iters++;
    double mneg = vmaxneg(W.y_new, nsp, sred);
    double sumy = vsum(W.y_new, nsp, sred);
    if (grd <= dgrd && mneg < sum_check && fabs(1.0 - sumy) <= K_SUM_TOL) {
      vcopy(yps, W.y_new, nsp);
      dtrcmd = 2.0 * fmax(fmin(pow(dgrd / fmax(grd, K_SMALL), 0.5), rmax), rmin) * dt;
      ypsplus(yps, nsp);
      return 0;
    }
    vcopy(W.y_cur, W.y_new, nsp);
  }
}

// ---------------------------------------------------------------------------------------------
// Compact Bader-Deuflhard vectors (indexed by active row c)
struct BdVec {
  double *yk, *dk, *yext, *ysc, *dxc, *Q, *E;
};

__device__ __forceinline__ BdVec bd_bind(const Ws &W, int nsys) {
  BdVec B;
  B.yk = W.bd; B.dk = W.bd + nsys; B.yext = W.bd + 2 * nsys; B.ysc = W.bd + 3 * nsys; B.dxc = W.bd + 4 * nsys;
  B.Q = W.bd + 6 * nsys;
  B.E = W.bd + (6 + kMaxLevels + 1) * (size_t)nsys;
  return B;
}

// one semi-implicit midpoint sub-step, bader_deuflhard_step (bader_deuflhard.F90:410-488)
__device__ int dev_bd_substep(const DevNet &N, const Ws &W, ZoneCtl &C, const BdVec &B, double h, int stage,
                              bool huge_frozen) {
  const int tid = GT, nt = GN;
  Act &A = C.act;
  dev_dxdt_active(A, B.yk, B.dxc);
  if (stage == 1) for (int c = tid; c < A.na; c += nt) A.xs[c] = h * B.dxc[c];
  else for (int c = tid; c < A.na; c += nt) A.xs[c] = h * B.dxc[c] - B.dk[c];
  GSYNC();
  if (!dev_solve_active(A)) return BAD_STEP;
  C.st.nsolve++;
  bool huge = false;
  for (int c = tid; c < A.na; c += nt) {
    const double d = stage == 2 ? B.dk[c] + 2.0 * A.xs[c] : A.xs[c];
    B.dk[c] = d;
    const double yk = B.yk[c] + d;
    B.yk[c] = yk;
    if (yk > 2.0) huge = true;
  }
  return (block_any(huge) || huge_frozen) ? HUGE_ABUNDS : 0;
}

// All sub-steps of one level (semi_implicit_extrapolation, bader_deuflhard.F90:276-316) for a
// tile-sized active system. Each sub-step's right-hand-side terms are computed by the whole CTA;
// the row sums, the tile solve and the update are done by warp 0, whose lane l keeps y_k and delta_k
// of active rows l + 32 i in registers. Two barriers per sub-step. Same arithmetic as
// dev_bd_substep. Leaves y_k / delta_k in B.yk / B.dk; returns 0 or HUGE_ABUNDS.
template <int R>
__device__ int bd_level_tile(const Act &A, const BdVec &B, double h, int nseq, bool huge_frozen, int &nsolve,
                             int &ir_sweeps, int *sflag) {
  const int tid = GT, nt = GN, lane = tid & 31, w = tid >> 5, na = A.na;
  double y[R], d[R], ri[R], an[R];
  int sweeps = 0;  // refinement sweeps (mixed precision), counted by warp 0
  if (w == 0) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = lane + 32 * i;
      const bool on = r < na;
      y[i] = on ? B.yk[r] : 0.0;
      d[i] = 0.0;
      ri[i] = on ? A.rinv[r] : 0.0;
      an[i] = on ? A.anc[r] : 1.0;
      if (on) A.xnc[r] = y[i] / an[i];
    }
    if (lane == 0) {
      sflag[0] = 0;  // stop: HUGE_ABUNDS
      sflag[1] = 0;  // solves done
      sflag[2] = 0;  // refinement sweeps
    }
  }
  for (int j = 0;; ++j) {
    GSYNC();  // xnc of sub-step j and the stop flag are written
    if (sflag[0] != 0 || j > nseq) break;
#pragma unroll 4
    for (int q = tid; q < A.ngi; q += nt) A.gterm[q] = rhs_term(A, q);
    GSYNC();
    if (w == 0) {
      const int stage = j == 0 ? 1 : (j < nseq ? 2 : 3);  // FIRST, MID, LAST
      double x[R];
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int r = lane + 32 * i;
        x[i] = 0.0;
        if (r < na) {
          const double dx = gather_dxdt(A, r);
          x[i] = stage == 1 ? h * dx : h * dx - d[i];
        }
      }
      if (A.mixed_now) {
        sweeps += tile_solve_mixed<R>(A, x, lane);
      } else {
        tile_permute_rhs<R>(x, A.perm, na, A.xs, lane);  // the factor is of P (I - hJ)
        tile_solve_regs<R>(A.T, A.rinv, na, x, ri, lane);
      }
      bool huge = false;
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int r = lane + 32 * i;
        d[i] = stage == 2 ? d[i] + 2.0 * x[i] : x[i];
        y[i] = y[i] + d[i];
        huge |= r < na && y[i] > 2.0;
        if (r < na) A.xnc[r] = y[i] / an[i];
      }
      huge = __any_sync(NUPPN_FULL, huge) || huge_frozen;
      if (lane == 0) {
        sflag[1] = j + 1;
        if (huge) sflag[0] = HUGE_ABUNDS;
      }
    }
  }
  if (w == 0) {
#pragma unroll
    for (int i = 0; i < R; ++i)
      if (lane + 32 * i < na) {
        B.yk[lane + 32 * i] = y[i];
        B.dk[lane + 32 * i] = d[i];
      }
    if (lane == 0) sflag[2] = sweeps;
  }
  GSYNC();
  const int err = sflag[0];
  nsolve += sflag[1];
  ir_sweeps += sflag[2];
  GSYNC();
  return err;
}

__device__ int dev_bd_level_tile(const Act &A, const BdVec &B, double h, int nseq, bool huge_frozen, int &nsolve,
                                 int &ir_sweeps, int *sflag) {
  return A.tile_rows == 32 ? bd_level_tile<1>(A, B, h, nseq, huge_frozen, nsolve, ir_sweeps, sflag)
                           : bd_level_tile<2>(A, B, h, nseq, huge_frozen, nsolve, ir_sweeps, sflag);
}

// extrapolate (bader_deuflhard.F90:371-407): Neville tableau, column k, on the active rows
__device__ void dev_extrapolate(ZoneCtl &C, const BdVec &B, int na, int k, double xest) {
  C.xhist[k] = xest;
  for (int j = GT; j < na; j += GN) {
    const double yest = B.yk[j];
    if (k == 1) {
      B.Q[(size_t)k * na + j] = yest;
      B.E[(size_t)k * na + j] = yest;
      B.yext[j] = yest;
      continue;
    }
    double yz = yest, d = yest, e = yest;
    for (int k1 = 1; k1 <= k - 1; ++k1) {
      const double delta = 1.0 / (C.xhist[k - k1] - xest);
      const double f1 = xest * delta, f2 = C.xhist[k - k1] * delta;
      const double q = B.Q[(size_t)k1 * na + j];
      B.Q[(size_t)k1 * na + j] = e;
      const double dl = d - q;
      e = f1 * dl;
      d = f2 * dl;
      yz = yz + e;
    }
    B.E[(size_t)k * na + j] = e;
    B.Q[(size_t)k * na + j] = e;
    B.yext[j] = yz;
  }
  GSYNC();
}

__device__ int dev_bader_deuflhard(const DevNet &N, const Ws &W, ZoneCtl &C, double *yps, double dt, double &dtrcmd,
                                   bool frst, double *sred) {
  const int tid = GT, nt = GN;
  const double safe1 = 0.25, safe2 = 0.7, redmin = 0.7, redmax = 1.e-5, scalmx = 0.25;
  const double thr = N.kn.grdthreshold;
  int km = -1, k;
  double scal = 1.0, red = -1.0, errmax = 0.0, abuerr = 0.0, negerr = 0.0;
  dev_new_jacobian(N, W, C, dt, yps);
  Act &A = C.act;
  const int na = A.na;
  const BdVec B = bd_bind(W, N.nsys);
  // frozen species: constant share of the mass sum, of the negative test and of the error mask
  double sum_fz = 0.0, neg_fz = -DBL_MAX;
  bool big_fz = false, huge_fz = false;
  for (int s = tid; s < N.nsp; s += nt) {
    if (W.mask[s]) continue;
    const double y = yps[s];
    sum_fz += y;
    if (y < thr) neg_fz = fmax(neg_fz, -y);
    if (y > 1e-27) big_fz = true;
    if (y > 2.0) huge_fz = true;
  }
  sum_fz = block_sum(sum_fz, sred);
  neg_fz = block_max(neg_fz, sred);
  big_fz = block_any(big_fz);
  huge_fz = block_any(huge_fz);
  for (k = 1; k <= N.kmax; ++k) {
    for (int c = tid; c < na; c += nt) B.yk[c] = yps[N.sp_of_sys[A.arow[c]]];
    GSYNC();
    // semi_implicit_extrapolation (bader_deuflhard.F90:276-316)
    const double h = dt / (double)N.nseq[k];
    const double xest = powi(h / N.nseq[k], 2);
    if (!dev_factor_active(N, W, A, h)) {
      dtrcmd = dt * 0.2;
      return BAD_STEP;
    }
    C.st.nfact++;
    int ierr;
    if (A.tile) {
      ierr = dev_bd_level_tile(A, B, h, N.nseq[k], huge_fz, C.st.nsolve, C.st.ir_sweeps, C.sint);
    } else {
      ierr = dev_bd_substep(N, W, C, B, h, 1, huge_fz);
      for (int i = 1; ierr == 0 && i <= N.nseq[k] - 1; ++i) ierr = dev_bd_substep(N, W, C, B, h, 2, huge_fz);
      if (ierr == 0) ierr = dev_bd_substep(N, W, C, B, h, 3, huge_fz);
    }
    if (ierr != 0) {
      dtrcmd = dt * 0.2;
      return ierr;
    }
    C.st.newton_iters += N.nseq[k];
    dev_extrapolate(C, B, na, k, xest);
    bool nan = false;
    for (int c = tid; c < na; c += nt) {
      const double y = B.yext[c];
      B.yk[c] = y;
      if (y != y) nan = true;
      B.ysc[c] = fmax(fabs(y), thr);
    }
    if (block_any(nan)) {
      dtrcmd = dt * 0.2;
      return GOT_NAN;
    }
    if (k != 1) {
      // compute_error (bader_deuflhard.F90:325-366)
      double am = big_fz ? 0.0 : -DBL_MAX, nm = -DBL_MAX, sy = 0.0;
      for (int c = tid; c < na; c += nt) {
        const double y = B.yk[c];
        if (y > 1e-27) am = fmax(am, fabs(B.E[(size_t)k * na + c] / B.ysc[c]));
        if (y < thr) nm = fmax(nm, -y);
        sy += y;
      }
      abuerr = block_max(am, sred) / N.kn.dgrd;
      negerr = fmax(block_max(nm, sred), neg_fz) / thr;
      sy = block_sum(sy, sred);
      if (abuerr < 1e-3) {
        errmax = abuerr;
      } else {
        C.sumerr = fabs(1.0 - (sy + sum_fz)) / K_SUM_TOL;
        errmax = fmax(abuerr, C.sumerr);
      }
      errmax = fmax(errmax, negerr);
      km = k - 1;
      C.err[km] = pow(errmax / safe1, 1.0 / (2.0 * km + 1.0));
    }
    if (k != 1 && (k >= C.kopt - 1 || frst)) {
      if (errmax <= 1.0) {
        C.reduce = false;
        break;
      } else {
        if (k == N.kmax || k == C.kopt + 1) {
          C.reduce = true; red = safe2 / C.err[km];
        } else if (k == C.kopt) {
          if (N.alf[C.kopt - 1][C.kopt] < C.err[km]) { C.reduce = true; red = safe2 / C.err[km]; }
        } else if (C.kopt == N.kmax) {
          if (N.alf[km][N.kmax - 1] < C.err[km]) { C.reduce = true; red = N.alf[km][N.kmax - 1] * safe2 / C.err[km]; }
        } else if (N.alf[km][C.kopt] < C.err[km]) {
          C.reduce = true; red = N.alf[km][C.kopt - 1] / C.err[km];
        }
      }
    }
  }
  int ierr = 0;
  if (k > N.kmax) k = N.kmax + 1;
  if (C.reduce) {
    red = fmax(redmax, fmin(red, redmin));
    dtrcmd = dt * red;
    if (negerr > C.sumerr && negerr > abuerr) ierr = NEG_ABUNDS;
    else if (C.sumerr > abuerr) ierr = SUM_X;
    else ierr = SLV_CNVRG;
  } else {
    double workmin = 1.e35;
    for (int kk = 1; kk <= km; ++kk) {
      double f = fmax(C.err[kk], scalmx), work = f * N.bd_a[kk + 1];
      if (work < workmin) { scal = f; workmin = work; C.kopt = kk + 1; }
    }
    dtrcmd = 2.0 * dt / scal;
    if (C.kopt >= k && C.kopt != N.kmax) {
      double f = fmax(scal / N.alf[C.kopt - 1][C.kopt], scalmx);
      if (N.bd_a[C.kopt + 1] * f <= workmin) {
        dtrcmd = dtrcmd * scal / f;
        C.kopt = C.kopt + 1;
      }
    }
  }
  for (int c = tid; c < na; c += nt) yps[N.sp_of_sys[A.arow[c]]] = B.yk[c];  // yps(:) = y_k(:)
  GSYNC();
  return ierr;
}

__device__ __forceinline__ double interp2(double x1, double y0, double y1, double xw) {  // interp.F90:29-50
  double xwant = fmin(fmax(xw, 0.0), x1);
  return y0 + (y1 - y0) * (xwant - 0.0) / (x1 - 0.0);
}

// integrate_network (solver.F90:53-238) for the CTA's zone; W.y holds yps on entry and exit
__device__ int dev_integrate_zone(const DevNet &N, const Ws &W, ZoneCtl &C, double t9_0, double t9_1, double rho_0,
                                  double rho_1, double &ye, double dtwant, bool frst, double *sred) {
  const int nsp = N.nsp;
  const nuppn_knobs &kn = N.kn;
  double *yps = W.y;
  if (!(t9_0 > 0.0) || !(t9_1 > 0.0) || !(rho_0 > 0.0) || !(rho_1 > 0.0) || !isfinite(t9_0 + t9_1 + rho_0 + rho_1) ||
      !(dtwant > 0.0) || !isfinite(dtwant))
    return NUPPN_BAD_INPUT;
  vcopy(W.y_old, yps, nsp);
  double ye_old = ye, dtdone = 0.0, dtrcmd = 0.0, dttry = dtwant;
  double t9_last = 0.5 * (t9_0 + t9_1), rho_last = 0.5 * (rho_0 + rho_1);
  dev_eval_rates(N, W, t9_last, rho_last, ye, yps, sred);  // the frame's evaluate_all_rates
  C.rates_ver++;
  for (int i = 1; i <= kn.max_sub_steps; ++i) {
    if (i > 1) frst = false;
    double t_0 = dtdone, t_1 = fmin(dtdone + dttry, dtwant);
    double my_t9_0 = 0, my_t9_1 = 0, my_rho_0 = 0, my_rho_1 = 0, my_t9, my_rho;
    if (kn.interpolate_temp) {
      my_t9_0 = interp2(dtwant, t9_0, t9_1, t_0);
      my_t9_1 = interp2(dtwant, t9_0, t9_1, t_1);
      my_t9 = 0.5 * (my_t9_0 + my_t9_1);
    } else {
      my_t9 = 0.5 * (t9_0 + t9_1);
    }
    if (kn.interpolate_dens) {
      my_rho_0 = interp2(dtwant, rho_0, rho_1, t_0);
      my_rho_1 = interp2(dtwant, rho_0, rho_1, t_1);
      my_rho = 0.5 * (my_rho_0 + my_rho_1);
    } else {
      my_rho = 0.5 * (rho_0 + rho_1);
    }
    double diff = fmax(fabs(my_t9_0 - my_t9_1) / my_t9_0, fabs(my_rho_0 - my_rho_1) / my_rho_0);
    if (diff > kn.delta_state_max && t9_0 > kn.min_t9_for_slv && t9_1 > kn.min_t9_for_slv) {
      dttry = 0.5 * dttry;
      continue;
    }
    if (my_t9 != t9_last || my_rho != rho_last) {
      dev_eval_rates(N, W, my_t9, my_rho, ye, yps, sred);
      C.rates_ver++;
      t9_last = my_t9; rho_last = my_rho;
    }
    // NSE above nse_min_t9 (solver.F90:153-158; do_one_time_step, solver.F90:260-266)
    const bool do_nse = kn.i_nse == 1 && my_t9 >= kn.nse_min_t9;
    if (do_nse) dev_nse_cache_lm(N, W);
    int ierr = 0;
    if (my_t9 >= kn.min_t9_for_slv) {
      if (do_nse) {
        C.act_ok = false;  // the NSE step works in the same shared memory
        if (kn.nse_weak_method == 0)
          ierr = dev_nse_euler(N, W, C.nse, yps, my_t9, my_rho, ye, dttry, dtrcmd, C.smem, C.smem_bytes, sred);
        else
          ierr = dev_nse_rk4(N, W, C.nse, yps, my_t9, my_rho, ye, dttry, dtrcmd, C.smem, C.smem_bytes, sred);
      } else {
        if (kn.integration_method == 0) ierr = dev_backward_euler(N, W, C, yps, dttry, dtrcmd, sred);
        else ierr = dev_bader_deuflhard(N, W, C, yps, dttry, dtrcmd, frst, sred);
        ye = dev_ye(N, yps, sred);
      }
      if (dttry < K_SMALL) return SMALL_DT;
    }
    if (ierr == 0) {
      dtdone = dtdone + dttry;
      for (int s = GT; s < nsp; s += GN) {
        double y = fmax(yps[s], 1.e-99);
        yps[s] = y;
        W.y_old[s] = y;
      }
      GSYNC();
      ye_old = ye;
      C.st.nsucc++;
      if (dtdone >= dtwant) break;
    } else {
      vcopy(yps, W.y_old, nsp);
      ye = ye_old;
      C.st.nfail++;
    }
    dttry = fmin(dtrcmd, dtwant - dtdone);
    if (i == kn.max_sub_steps) return MAX_SUBSTEPS;
  }
  if (kn.integration_method == 1) {
    double s = vsum(yps, nsp, sred);
    for (int q = GT; q < nsp; q += GN) yps[q] = yps[q] / s;
    GSYNC();
  }
  for (int q = GT; q < nsp; q += GN) yps[q] = fmax(yps[q], 1.e-99);
  GSYNC();
  return 0;
}

NUPPN_END
