"""Error of device results against the checker (TEST INFRASTRUCTURE: used by tests/ and by bench.py's
checker leg, never by the product).

The reference's FP64 CPU path is restated in oracle.cpp and calls the reference's own SuperLU, so
the checker's output is the yardstick. Some zones are ill-conditioned in the reference's own
algorithm: a change of one unit in the last place of the input, of one rounding in the sums of
dX/dt, or of the LU's elimination order changes their sub-step sequence or their final abundances
far beyond 1e-6. For those, `checker_spread` measures how far the checker itself moves under these
three kinds of perturbation, and a device result is judged against that spread. (The second kind is what any implementation that does
not add the reference's terms in the reference's order is free to differ by: H-burning zones at
T9 < 0.08 over 1e10 s move by 1-50 % under it while 1-ulp input changes move them far less.)
"""
from __future__ import annotations

import numpy as np

REL_TOL = 1.0e-6     # final X, relative, for X > 1e-12 (the parity bar)
ABS_TOL = 1.0e-15    # final X, absolute, for X <= 1e-12
X_SMALL = 1.0e-12


def zone_errors(X, Xr):
    """Per zone: max relative error over species with Xr > 1e-12 and max absolute error below."""
    X = np.atleast_2d(X)
    Xr = np.atleast_2d(Xr)
    big = Xr > X_SMALL
    rel = np.where(big, np.abs(X - Xr) / np.where(big, Xr, 1.0), 0.0).max(axis=1)
    ab = np.where(big, 0.0, np.abs(X - Xr)).max(axis=1)
    return rel, ab


def checker_spread(ref, zb, X0, trials=(1, 2), nthreads=1, rhs_noise=True, lu_permute=True):
    """Per zone: the largest relative change (species with X0 > 1e-12) of the checker's own final
    abundances over seeded draws of three perturbations, one draw of each per entry of `trials`:
    every initial abundance moved by -1, 0 or +1 ulp at random; with rhs_noise, every dX/dt entry of
    every evaluation scaled by 1 - 2^-52, 1 or 1 + 2^-52 at random; with lu_permute, every
    Bader-Deuflhard system factored by SuperLU in another (seeded) elimination order. X0 is the
    checker's unperturbed result for the batch zb; the checker's perturbations are off afterwards."""
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    spread = np.zeros(zb.nz)
    for t in trials:
        Xp = zb.X * (1.0 + np.random.default_rng(t).choice([-1.0, 0.0, 1.0], size=zb.X.shape) * 2.2e-16)
        X1, _, _, _, _ = ref.integrate_network(Xp, *args, nthreads=nthreads)
        spread = np.maximum(spread, zone_errors(X1, X0)[0])
    for on, setter in ((rhs_noise, ref.set_rhs_noise), (lu_permute, ref.set_lu_permute)):
        if not on:
            continue
        try:
            for t in trials:
                setter(t)
                X1, _, _, _, _ = ref.integrate_network(zb.X, *args, nthreads=nthreads)
                spread = np.maximum(spread, zone_errors(X1, X0)[0])
        finally:
            setter(None)
    return spread


def summary(X, ierr, nsucc, Xr, ierr_r, nsucc_r, spread=None):
    """Statistics of device results (X, ierr, accepted steps) against the checker's."""
    rel, ab = zone_errors(X, Xr)
    ok = (ierr == 0) & (ierr_r == 0)
    beyond = (rel > REL_TOL) | (ab > ABS_TOL)
    out = {
        "zones": int(len(rel)),
        "max_rel_err_X_gt_1e-12": float(rel[ok].max(initial=0.0)),
        "max_abs_err_X_le_1e-12": float(ab[ok].max(initial=0.0)),
        "max_abs_sum_X_minus_1": float(np.abs(np.atleast_2d(X)[ierr == 0].sum(axis=1) - 1.0).max(initial=0.0)),
        "ierr_equal": int((ierr == ierr_r).sum()),
        "accepted_steps_equal": int((np.asarray(nsucc) == np.asarray(nsucc_r)).sum()),
        "zones_within_1e-6": int((ok & ~beyond).sum()),
        "zones_beyond_1e-6": int((ok & beyond).sum()),
    }
    if spread is not None:
        out["zones_beyond_checker_spread"] = int((ok & beyond & (rel > spread)).sum())
        out["zones_beyond_2x_checker_spread"] = int((ok & beyond & (rel > 2.0 * spread)).sum())
        out["max_checker_spread"] = float(np.max(spread, initial=0.0))
    return out
