"""CPU tests: the checker against its pins and invariants, the synthetic networks, and the C ABI
library's exports (no device calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_superlu_matrixtest_pin(orc):
    """slu_f90/matrixtest.f90: the reference's own 20x20 smoke system through slu_solve; x(1) =
    0.38737081 is the value the reference prints."""
    L = C.CDLL(orc.SLU)
    n, nnz = 20, 24
    val = np.array([1., 0.66004251, 1., 1., 0.16580944, 1., 1., 1., 1., 1., 0.48754192, 1., 1., 1., 1., 1.,
                    1., 0.39321144, 1., 1., 1., 1., 1., 1.])
    colind = (np.array([0, 2, 1, 2, 15, 3, 4, 5, 6, 7, 1, 8, 9, 10, 11, 12, 13, 10, 14, 15, 16, 17, 18, 19]) + 1).astype(np.int32)
    rowptr = (np.array([0, 2, 3, 5, 6, 7, 8, 9, 10, 12, 13, 14, 15, 16, 17, 19, 20, 21, 22, 23, 24]) + 1).astype(np.int32)
    rhs = np.array([0.36505416, 0.87209716, 0.11306562, 0.15746164, 0.36074325, 0.95214683, 0.97631797,
                    0.26061262, 0.25675798, 0.75232693, 0.07135243, 0.07346062, 0.41943103, 0.48905309,
                    0.12271773, 0.88581534, 0.99626864, 0.6568508, 0.63238463, 0.65226356])
    b = rhs.copy()
    ierr = C.c_int(0)
    P = lambda a: C.c_void_p(a.ctypes.data)
    L.slu_solve(n, nnz, 1, 1, P(val), P(colind), P(rowptr), P(b), C.byref(ierr))
    assert ierr.value == 0
    assert abs(b[0] - 0.38737081) < 5e-9
    # residual of the unscaled system
    A = np.zeros((n, n))
    ci, rp = colind - 1 + 1, rowptr  # slu_solve shifted the index arrays to 0-based in place
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            A[i, ci[k]] = val[k]
    assert np.abs(A @ b - rhs).max() < 1e-12


def test_sortedsum_heapsort_order(orc):
    rng = np.random.default_rng(0)
    a = np.concatenate([10.0 ** rng.uniform(-30, 0, 500), -10.0 ** rng.uniform(-30, -5, 50)])
    s = orc.sortedsum(a)
    ref = 0.0
    for x in np.sort(a):
        ref = ref + x
    assert s == ref


@pytest.fixture(scope="module")
def small(wl):
    return wl.network(120)


def test_network_layout(small, sn):
    net = small
    assert net.zis[net.igamma] == "OOOOO" and not net.considerisotope[net.igamma]
    k = net.k[net.considerreaction == 1]
    assert (k[:, [0, 2, 4, 6]] >= 0).all() and (k[:, [0, 2, 4, 6]] < net.nsp).all()
    assert (k[:, 0] != net.igamma).all() and (k[:, 6] != net.igamma).all()
    # triple alpha in the reference's slot 43 (1-based)
    assert net.k[42, 0] == net.species_index("HE  4") and net.k[42, 1] == 3
    # baryon number conserved by every considered reaction
    A = net.anetw
    lhs = A[k[:, 0]] * k[:, 1] + A[k[:, 2]] * k[:, 3]
    rhs = A[k[:, 4]] * k[:, 5] + A[k[:, 6]] * k[:, 7]
    assert np.allclose(lhs, rhs)
    Z = net.znetw
    lz = Z[k[:, 0]] * k[:, 1] + Z[k[:, 2]] * k[:, 3]
    rz = Z[k[:, 4]] * k[:, 5] + Z[k[:, 6]] * k[:, 7]
    # charge: network reactions other than weak ones (the VITAL block labels p(p,e+nu)d as (p,g))
    idx = np.nonzero(net.considerreaction == 1)[0]
    strong = ~np.isin(net.ilabb[idx], [13, 14, 15, 16]) & (idx >= net.nrcp)
    assert np.allclose(lz[strong], rz[strong])


def test_network_deterministic(sn):
    a, b = sn.build_network(150, seed=3), sn.build_network(150, seed=3)
    assert (a.k == b.k).all() and np.array_equal(a.rl_a, b.rl_a)


def test_oracle_rhs_conserves_mass(orc, abi, small, wl):
    """sum_i dX_i/dt = 0 for mass-conserving reactions (calculate_dxdt, jac_rhs.F90:217-278)."""
    ref = orc.Oracle(small, abi.default_knobs())
    zb = wl.heshell_batch(3, net=small, seed=4)
    v = ref.evaluate_all_rates(zb.t9_0, zb.rho_0, zb.ye, zb.X)
    d = ref.calculate_dxdt(v, zb.X)
    scale = np.abs(d).max(axis=1)
    assert (np.abs(d.sum(axis=1)) <= 1e-10 * scale).all()


def test_oracle_detailed_balance_ratio(orc, abi, small, wl):
    """v_rev / v_fwd equals the reverse.F90 factor before screening: checked with screening off."""
    kn = abi.default_knobs(screen_option=0)
    ref = orc.Oracle(small, kn)
    zb = wl.heshell_batch(1, net=small, seed=4)
    v = ref.evaluate_all_rates(zb.t9_0, zb.rho_0, zb.ye, zb.X)[0]
    pairs = [(i, j) for i, j in enumerate(small.irev) if j >= 0 and small.considerreaction[i]]
    assert pairs
    kn0 = abi.default_knobs(screen_option=0, detailed_balance=0)
    v0 = orc.Oracle(small, kn0).evaluate_all_rates(zb.t9_0, zb.rho_0, zb.ye, zb.X)[0]
    # without detailed balance the 'RVRSE' slots are not gathered (clipped to 1e-99)
    assert all(v0[j] == 1e-99 for _, j in pairs)
    changed = [j for i, j in pairs if v[i] > 1e-97]
    assert any(v[j] > 1e-99 for j in changed)


def test_oracle_jacobian_is_dfdx(orc, abi, small, wl):
    """calculate_jacobian values are the derivative of dxdt (finite differences on a few columns)."""
    ref = orc.Oracle(small, abi.default_knobs())
    zb = wl.heshell_batch(1, net=small, seed=9)
    X = zb.X[0].copy()
    X[X < 1e-20] = 1e-6  # move every species off the floor so derivatives are well defined
    X /= X.sum()
    v = ref.evaluate_all_rates(zb.t9_0, zb.rho_0, zb.ye, X)
    jac, es, mk = ref.calculate_jacobian(v, X, 1.0)
    row, col, _ = ref.jac_pattern()
    J = {}
    for e in range(len(row)):
        J[(row[e], col[e])] = jac[0, e] - 1e-99
    d0 = ref.calculate_dxdt(v, X)[0]
    for j in [small.species_index(s) for s in ("HE  4", "C  12", "NE 22")]:
        h = X[j] * 1e-6
        Xp = X.copy(); Xp[j] += h
        fd = (ref.calculate_dxdt(v, Xp)[0] - d0) / h
        for i in range(small.nsp):
            if i == small.igamma:
                continue
            ana = J.get((i, j), 0.0)
            # finite-difference round-off: a few ulps of dxdt_i divided by the step
            fd_noise = 64 * np.finfo(float).eps * abs(d0[i]) / h
            assert abs(fd[i] - ana) <= 1e-4 * max(abs(ana), abs(fd[i])) + fd_noise


def test_oracle_bd_conserves_mass(orc, abi, wl):
    net = wl.network(200)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    zb = wl.heshell_batch(2, net=net, seed=5)
    X, ye, ierr, st, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    assert (ierr == 0).all()
    assert np.abs(X.sum(axis=1) - 1).max() < 1e-12
    assert all(s.nsucc >= 1 for s in st)
    # Ye from composition (calculate_ye) of the last sub-step, before the final renormalisation
    # of solver.F90:234, so equal to the Ye of the returned X only to the size of that correction
    for z in range(2):
        assert abs(ye[z] - ref.calculate_ye(X[z])) < 1e-8


def test_oracle_bd_order_on_linear_decay(orc, abi, sn, wl):
    """Bader-Deuflhard on a chain whose solution is analytic: the He-shell batch with strong rates
    switched off leaves pure beta decays; conservation and positivity must hold."""
    net = wl.network(120)
    kn = abi.default_knobs(integration_method=1, strong_rates=0)
    ref = orc.Oracle(net, kn)
    zb = wl.heshell_batch(1, net=net, seed=6)
    X, ye, ierr, st, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    assert ierr[0] == 0
    assert (X >= 1e-99).all()


def test_hburn_first_step_ill_conditioned(orc, abi, wl):
    """The first backward-Euler frame step of the H-burning zone (dt = 1e3 s from the initial
    composition) does not converge on the first Newton try in the reference's algorithm, and its
    retry sequence depends on the last bits of the input: 1-ulp changes of X give different sub-step
    counts and results that differ by far more than the step tolerance. Device parity for that one
    step is therefore checked by success and mass conservation, not by value."""
    net = wl.network(300)
    zb, dts = wl.hburn_zone(net)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=0))
    outcomes, results = set(), []
    for trial in range(4):
        X = zb.X.copy()
        if trial:
            X = X * (1.0 + np.random.default_rng(trial).choice([-1.0, 0.0, 1.0], size=X.shape) * 2.2e-16)
        Xn, _, ierr, st, _ = ref.integrate_network(X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, dts[0])
        assert ierr[0] == 0 and st[0].nfail >= 1
        outcomes.add((st[0].nsucc, st[0].nfail))
        results.append(Xn)
    assert len(outcomes) > 1
    big = results[0] > 1e-12
    spread = max((np.abs(r - results[0])[big] / results[0][big]).max() for r in results[1:])
    assert spread > 1e-3


def test_hot_heshell_zones_ill_conditioned(orc, abi, wl):
    """The hottest He-shell zones of the 1109-species network (T9 ~ 0.3) reject about half of their
    Bader-Deuflhard steps; in the reference's algorithm 1-ulp changes of the input change the accepted
    step count and move final abundances far beyond the 1e-6 tolerance. Device parity on these zones
    is therefore checked against the checker's own spread, not by step count."""
    net = wl.network(1107)
    full = wl.heshell_batch(1024, net=net, seed=2)
    zb = full.take(np.argsort(-full.t9_0)[:2])
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    X0, _, _, st0, _ = ref.integrate_network(zb.X, *args, nthreads=2)
    steps, spread = {tuple(s.nsucc for s in st0)}, 0.0
    big = X0 > 1e-12
    for trial in (1, 2, 3):
        Xp = zb.X * (1.0 + np.random.default_rng(trial).choice([-1.0, 0.0, 1.0], size=zb.X.shape) * 2.2e-16)
        X1, _, ierr, st, _ = ref.integrate_network(Xp, *args, nthreads=2)
        assert (ierr == 0).all()
        steps.add(tuple(s.nsucc for s in st))
        spread = max(spread, (np.abs(X1 - X0)[big] / X0[big]).max())
    assert len(steps) > 1
    assert spread > 1e-3


def test_oracle_nse_satisfies_constraints(orc, abi, wl):
    """compute_nse converges to theta = sum X - 1 = 0 and phi = sum (Z/A) X - Ye = 0 within the
    reference's Newton tolerance (1e-9, nse_swj.F90:104), over T9 6..10 and rho 1e6..1e8."""
    net = wl.network(1107)
    ref = orc.Oracle(net, abi.default_knobs())
    zb = wl.nse_batch(8, net=net)
    X, mu_p, mu_n, it, ierr = ref.compute_nse(zb.t9_0, zb.rho_0, zb.ye)
    assert (ierr == 0).all() and (it > 0).all()
    zoa = np.where(net.anetw > 0, net.znetw / np.where(net.anetw > 0, net.anetw, 1.0), 0.0)
    assert np.abs(X.sum(axis=1) - 1.0).max() < 2e-9
    assert np.abs((X * zoa).sum(axis=1) - zb.ye).max() < 2e-9
    assert np.isfinite(mu_p).all() and np.isfinite(mu_n).all()


def test_library_exports_header_symbols(solver_mod):
    """Every function declared in include/nuppn.h is exported by the built library."""
    hdr = open(os.path.join(ROOT, "include", "nuppn.h")).read()
    names = sorted(set(re.findall(
        r"^(?:nuppn_status|int32_t|int64_t|void|const char \*)\s*(nuppn_[a-z_]+)\(", hdr, re.M)))
    assert len(names) >= 14
    L = solver_mod.load_library()
    for n in names:
        assert hasattr(L, n), n
    assert L.nuppn_abi_version() == 3


def test_no_cpu_fallback_in_product(solver_mod):
    """The product package never loads the checker."""
    pkgdir = os.path.join(ROOT, "nuppn_modular2-ininet3_b200")
    for f in os.listdir(pkgdir):
        if f.endswith(".py"):
            src = open(os.path.join(pkgdir, f)).read()
            assert "oracle" not in src.replace("reference", ""), f


def test_oracle_rhs_noise_is_seeded_and_shows_hburn_sensitivity(orc, abi, wl):
    """The checker's dX/dt perturbation (a rounding-sized change of every entry, the freedom any
    implementation that sums the terms in another order has) and its elimination-order perturbation
    of the LU: off by default and after they are switched off, deterministic per seed and
    independent of the thread count. Cool H-burning zones
    (300 species, T9 0.02-0.05, 1e10 s) move by far more than 1e-6 under it, which is why the
    parity bar for such zones is the checker's spread under these perturbations."""
    net = wl.network(300)
    hb, _ = wl.hburn_zone(net)
    n = 6
    t9 = np.linspace(0.02, 0.05, n)
    rho = np.full(n, 100.0)
    X = np.repeat(hb.X, n, axis=0)
    ye = np.repeat(hb.ye, n)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    run = lambda nt: ref.integrate_network(X, t9, t9, rho, rho, ye, np.full(n, 1e10), nthreads=nt)
    X0, _, ie0, _, _ = run(3)
    ref.set_rhs_noise(7)
    Xa, _, iea, _, _ = run(1)
    Xb, _, ieb, _, _ = run(3)
    ref.set_rhs_noise(None)
    Xc, _, _, _, _ = run(2)
    assert np.array_equal(Xa, Xb) and np.array_equal(iea, ieb)  # per-zone generators
    assert np.array_equal(Xc, X0)  # off again
    ref.set_lu_permute(3)  # another elimination order: deterministic, off again afterwards
    Xp1, _, _, _, _ = run(1)
    Xp2, _, _, _, _ = run(3)
    ref.set_lu_permute(None)
    assert np.array_equal(Xp1, Xp2) and np.array_equal(run(2)[0], X0)
    ok = (ie0 == 0) & (iea == 0)
    assert ok.sum() >= 3
    big = X0 > 1e-12
    rel = np.where(big, np.abs(Xa - X0) / np.where(big, X0, 1.0), 0.0).max(axis=1)
    assert (rel[ok] > 1e-6).any(), rel
