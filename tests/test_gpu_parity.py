"""Device path vs the CPU checker, through the C ABI, on the same seeded inputs.

Tolerances: rates 1e-11 relative (device exp/pow vs glibc); dxdt and Jacobian entries bit-equal for
targets summed in the reference's order, 1e-12 of the summed magnitude for the long n/p/alpha lists;
entry-set flags and dynamic-network masks bit-exact; integrated mass fractions within 1e-6 relative
for X > 1e-12 and 1e-15 absolute below (the acceptance bound of the workload).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net300(wl):
    return wl.network(300)


@pytest.fixture(scope="module")
def batch(wl, net300):
    return wl.heshell_batch(6, net=net300, seed=11)


def _dev(solver_mod, net, abi, **kw):
    return solver_mod.NetworkSolver(net, abi.default_knobs(**kw), device=0)


def test_rates_match_checker(solver_mod, abi, orc, net300, batch):
    dev = _dev(solver_mod, net300, abi)
    ref = orc.Oracle(net300, abi.default_knobs())
    v = dev.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    vr = ref.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    big = vr > 1e-90
    rel = np.abs(v - vr)[big] / vr[big]
    assert rel.max() < 1e-11, rel.max()
    assert (v[~big] <= 1e-89).all()


def test_dxdt_matches_checker(solver_mod, abi, orc, net300, batch):
    dev = _dev(solver_mod, net300, abi)
    ref = orc.Oracle(net300, abi.default_knobs())
    vr = ref.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    d = dev.calculate_dxdt(vr, batch.X)
    dr = ref.calculate_dxdt(vr, batch.X)
    scale = np.abs(dr).max(axis=1, keepdims=True)
    assert (np.abs(d - dr) <= 1e-12 * scale).all()
    assert (d == dr).mean() > 0.9  # short lists are accumulated in the reference's order


def test_jacobian_matches_checker(solver_mod, abi, orc, net300, batch):
    dev = _dev(solver_mod, net300, abi)
    ref = orc.Oracle(net300, abi.default_knobs())
    vr = ref.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    for dt in (1.0e2, 1.0e8):
        j, es, mk = dev.calculate_jacobian(vr, batch.X, dt)
        jr, esr, mkr = ref.calculate_jacobian(vr, batch.X, dt)
        assert (mk == mkr).all()
        assert (es == esr).all()
        scale = np.abs(jr).max(axis=1, keepdims=True)
        assert (np.abs(j - jr) <= 1e-12 * scale).all()


def test_pattern_matches_checker(solver_mod, abi, orc, net300):
    dev = _dev(solver_mod, net300, abi)
    ref = orc.Oracle(net300, abi.default_knobs())
    r, c, m = dev.jac_pattern()
    rr, cr, mr = ref.jac_pattern()
    assert (r == rr).all() and (c == cr).all() and (m == mr).all()


def test_reduced_solve_matches_superlu(solver_mod, abi, orc, net300, batch):
    dev = _dev(solver_mod, net300, abi)
    ref = orc.Oracle(net300, abi.default_knobs())
    vr = ref.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    dt = 1.0e8
    jr, esr, mkr = ref.calculate_jacobian(vr, batch.X, dt)
    rng = np.random.default_rng(5)
    b = rng.normal(size=(batch.nz, net300.nsp)) * 1e-3
    x = dev.solve_reduced(jr, esr, mkr, dt, b)
    xr, ierr = ref.solve_reduced(jr, esr, mkr, dt, b)
    assert (ierr == 0).all()
    err = np.abs(x - xr).max(axis=1) / np.abs(xr).max(axis=1)
    assert err.max() < 1e-9, err


def _compare_X(X, Xr):
    big = Xr > 1e-12
    rel = np.abs(X - Xr)[big] / Xr[big]
    small = np.abs(X - Xr)[~big]
    return rel.max(initial=0.0), small.max(initial=0.0)


def test_integrate_bd_matches_checker(solver_mod, abi, orc, net300, batch):
    kn = abi.default_knobs(integration_method=1)
    dev = _dev(solver_mod, net300, abi, integration_method=1)
    ref = orc.Oracle(net300, kn)
    args = (batch.X, batch.t9_0, batch.t9_1, batch.rho_0, batch.rho_1, batch.ye, batch.dtwant)
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    Xr, yer, ierr_r, str_, _ = ref.integrate_network(*args)
    assert (ierr == ierr_r).all()
    assert [s.nsucc for s in st] == [s.nsucc for s in str_]
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10


def test_integrate_be_hburn_matches_checker(solver_mod, abi, orc, wl):
    net = wl.network(300)
    zb, dts = wl.hburn_zone(net)
    kn = abi.default_knobs(integration_method=0)
    dev = _dev(solver_mod, net, abi, integration_method=0)
    ref = orc.Oracle(net, kn)
    X, Xr = zb.X.copy(), zb.X.copy()
    ye, yer = zb.ye.copy(), zb.ye.copy()
    for dt in dts[:40]:
        X, ye, ierr, _, _ = dev.integrate_network(X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, ye, dt)
        Xr, yer, ierr_r, _, _ = ref.integrate_network(Xr, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, yer, dt)
        assert ierr[0] == ierr_r[0] == 0
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)
