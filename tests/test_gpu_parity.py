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


@pytest.mark.parametrize("tile", [0, -1], ids=["tile", "sparse"])
@pytest.mark.parametrize("dt", [1.0e2, 1.0e8])
def test_reduced_solve_matches_superlu(solver_mod, abi, orc, net300, batch, tile, dt):
    dev = _dev(solver_mod, net300, abi, lu_tile_max=tile)
    ref = orc.Oracle(net300, abi.default_knobs())
    vr = ref.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    jr, esr, mkr = ref.calculate_jacobian(vr, batch.X, dt)
    rng = np.random.default_rng(5)
    b = rng.normal(size=(batch.nz, net300.nsp)) * 1e-3
    x = dev.solve_reduced(jr, esr, mkr, dt, b)
    xr, ierr = ref.solve_reduced(jr, esr, mkr, dt, b)
    assert (ierr == 0).all()
    err = np.abs(x - xr).max(axis=1) / np.abs(xr).max(axis=1)
    assert err.max() < 1e-9, err


@pytest.mark.parametrize("na", [11, 60], ids=["tile32", "tile64"])
def test_tile_solve_divides_like_superlu(solver_mod, abi, net300, na):
    """SuperLU's triangular solve divides by U(c, c) (dgstrs.c:248, dmyblas2.c:139). On a diagonal
    system (only the diagonal entries set, dt = 1 so that 1 - dt J_cc is formed exactly as numpy forms
    it) the tile path must return b / (1 - J_cc) bit for bit, signed zeros included: right-hand sides
    of 0, -0 and 1e-300..1e300 with pivots over 1e-14..1e250 of either sign (inside and outside the
    range of the reciprocal-based quotient)."""
    dev = _dev(solver_mod, net300, abi)
    r, c, _ = dev.jac_pattern()
    nz, nsp = 256, net300.nsp
    rng = np.random.default_rng(na)
    diag = np.nonzero((r == c) & net300.considerisotope[r].astype(bool))[0]
    sp_diag = r[diag]  # species of each diagonal entry (considered species only)
    jac = np.zeros((nz, r.size))
    es = np.zeros((nz, r.size), np.uint8)
    es[:, diag] = 1
    d = rng.choice([-1.0, 1.0], size=(nz, diag.size)) * 10.0 ** rng.uniform(-14, 250, size=(nz, diag.size))
    jac[:, diag] = 1.0 - d
    piv = -jac[:, diag] + 1.0  # assemble_entry: J * (-dt) + 1 with dt = 1
    mk = np.zeros((nz, nsp), np.uint8)
    act = np.argsort(rng.random((nz, diag.size)), axis=1)[:, :na]
    mk[np.arange(nz)[:, None], sp_diag[act]] = 1
    b = rng.choice([-1.0, 1.0], size=(nz, nsp)) * 10.0 ** rng.uniform(-300, 300, size=(nz, nsp))
    b[:, ::7] = 0.0
    b[:, 3::11] = -0.0
    x = dev.solve_reduced(jac, es, mk, 1.0, b)
    want = np.zeros((nz, nsp))
    on = mk[:, sp_diag].astype(bool)
    want[:, sp_diag] = np.where(on, b[:, sp_diag] / piv, 0.0)
    bad = np.nonzero(x.view(np.int64) != want.view(np.int64))  # signed zeros included
    assert bad[0].size == 0, (bad[0].size, x[bad][:4], want[bad][:4])


def test_trajectory_cooling_through_min_t9_matches_checker(solver_mod, abi, orc, wl):
    """A trajectory interval where T9 falls from 0.0131 to 0.0085 (crossing min_t9_for_slv) with a
    rate near 1e109 in its active system: the dynamic network has 11 species and the Bader-Deuflhard
    error test hinges on a 1e10-scale cancellation in the back substitution (a dX/dt term against
    U(r, c) x(c), both rounded products of the same factors), so the step only succeeds when the solve
    rounds as SuperLU built without FMA does: products rounded before they are subtracted, and x(c)
    divided by U(c, c) rather than multiplied by its reciprocal. Both LU paths must take the checker's
    steps and end within 1e-6 of its abundances."""
    net = wl.network(1107)
    tr = wl.trajectory_batch(1024, net=net, npts=201)
    tt, t9, rho = tr.grids()
    z, k1 = 244, 191
    kn = abi.default_knobs(integration_method=1)
    ref = orc.Oracle(net, kn)
    X = tr.X0[[z]].copy()
    bd = np.zeros(1, np.int32)
    for k in range(k1 + 1):
        ye = np.array([ref.calculate_ye(X[0])])
        a = (X, t9[z, k], t9[z, k + 1], rho[z, k], rho[z, k + 1], ye, tt[z, k + 1] - tt[z, k])
        if k == k1:
            break
        X, _, ierr, _, bd = ref.integrate_network(*a, bd_state=bd)
        assert ierr[0] == 0, k
    Xr, _, ierr_r, st_r, _ = ref.integrate_network(*a, bd_state=bd.copy())
    assert ierr_r[0] == 0
    for tile in (0, -1):
        dev = _dev(solver_mod, net, abi, integration_method=1, lu_tile_max=tile)
        Xd, _, ierr, st, _ = dev.integrate_network(*a, bd_state=bd.copy())
        assert ierr[0] == 0, (tile, st[0].nsucc, st[0].nfail)
        assert (st[0].nsucc, st[0].nfail) == (st_r[0].nsucc, st_r[0].nfail), tile
        rel, ab = _compare_X(Xd, Xr)
        assert rel <= 1e-6 and ab <= 1e-15, (tile, rel, ab)


@pytest.mark.parametrize("dt", [1.0e2, 1.0e8])
def test_reduced_solve_mixed_matches_superlu(solver_mod, abi, orc, net300, batch, dt):
    """lu_precision = 1: FP32 factor of the equilibrated tile, FP64 iterative refinement to
    ir_rtol = 1e-14; the solution must match SuperLU's FP64 one like the FP64 tile does (1e-9)."""
    dev = _dev(solver_mod, net300, abi, lu_precision=1)
    ref = orc.Oracle(net300, abi.default_knobs())
    vr = ref.evaluate_all_rates(batch.t9_0, batch.rho_0, batch.ye, batch.X)
    jr, esr, mkr = ref.calculate_jacobian(vr, batch.X, dt)
    b = np.random.default_rng(5).normal(size=(batch.nz, net300.nsp)) * 1e-3
    x = dev.solve_reduced(jr, esr, mkr, dt, b)
    xr, ierr = ref.solve_reduced(jr, esr, mkr, dt, b)
    assert (ierr == 0).all()
    err = np.abs(x - xr).max(axis=1) / np.abs(xr).max(axis=1)
    assert err.max() < 1e-9, err


def test_integrate_bd_mixed_matches_checker(solver_mod, abi, orc, net300, batch):
    """Bader-Deuflhard with lu_precision = 1 against the FP64 checker: the workload's tolerance
    (1e-6 relative for X > 1e-12, 1e-15 absolute below), mass conserved, refinement sweeps made."""
    dev = _dev(solver_mod, net300, abi, integration_method=1, lu_precision=1)
    ref = orc.Oracle(net300, abi.default_knobs(integration_method=1))
    args = (batch.X, batch.t9_0, batch.t9_1, batch.rho_0, batch.rho_1, batch.ye, batch.dtwant)
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    Xr, yer, ierr_r, str_, _ = ref.integrate_network(*args)
    assert (ierr == 0).all() and (ierr_r == 0).all()
    assert sum(s.ir_sweeps for s in st) > 0
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10


def _compare_X(X, Xr):
    big = Xr > 1e-12
    rel = np.abs(X - Xr)[big] / Xr[big]
    small = np.abs(X - Xr)[~big]
    return rel.max(initial=0.0), small.max(initial=0.0)


@pytest.mark.parametrize("tile", [0, -1], ids=["tile", "sparse"])
def test_integrate_bd_matches_checker(solver_mod, abi, orc, net300, batch, tile):
    kn = abi.default_knobs(integration_method=1)
    dev = _dev(solver_mod, net300, abi, integration_method=1, lu_tile_max=tile)
    ref = orc.Oracle(net300, kn)
    args = (batch.X, batch.t9_0, batch.t9_1, batch.rho_0, batch.rho_1, batch.ye, batch.dtwant)
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    Xr, yer, ierr_r, str_, _ = ref.integrate_network(*args)
    assert (ierr == ierr_r).all()
    assert [s.nsucc for s in st] == [s.nsucc for s in str_]
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10


@pytest.mark.parametrize("tile", [0, -1], ids=["tile", "sparse"])
def test_integrate_be_hburn_matches_checker(solver_mod, abi, orc, wl, tile):
    """ppn frame of the H-burning zone, backward Euler. The first frame step from the initial
    composition is ill-conditioned in the reference's own algorithm (its Newton iteration does not
    converge on the first try, and 1-ulp changes of the input change its sub-step sequence; see
    test_cpu_oracle.test_hburn_first_step_ill_conditioned), so that step is checked for success and
    mass conservation only; frame steps 1..39 then run on both sides from the checker's state."""
    net = wl.network(300)
    zb, dts = wl.hburn_zone(net)
    kn = abi.default_knobs(integration_method=0)
    dev = _dev(solver_mod, net, abi, integration_method=0, lu_tile_max=tile)
    ref = orc.Oracle(net, kn)
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1)
    X0, ye0, ierr0, _, _ = dev.integrate_network(zb.X, *args, zb.ye, dts[0])
    Xr, yer, ierr_r, _, _ = ref.integrate_network(zb.X, *args, zb.ye, dts[0])
    assert ierr0[0] == ierr_r[0] == 0
    assert abs(X0.sum() - 1.0) < 1e-10
    X, ye = Xr.copy(), yer.copy()
    for dt in dts[1:40]:
        X, ye, ierr, _, _ = dev.integrate_network(X, *args, ye, dt)
        Xr, yer, ierr_r, _, _ = ref.integrate_network(Xr, *args, yer, dt)
        assert ierr[0] == ierr_r[0] == 0
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)


@pytest.fixture(scope="module")
def hot1107(wl, orc, abi):
    """The four hottest He-shell zones of the 1109-species network, advanced 1e9 s by the checker:
    their dynamic networks keep 33..64 species at dt >= 1e8 s (the 64-row tile, two rows per lane)."""
    net = wl.network(1107)
    full = wl.heshell_batch(1024, net=net, seed=2)
    zb = full.take(np.argsort(-full.t9_0)[:4])
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    X, _, ierr, _, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, np.full(4, 1e9),
                                             nthreads=4)
    assert (ierr == 0).all()
    return net, zb, X, ref


@pytest.mark.parametrize("tile", [0, -1, "mixed"], ids=["tile", "sparse", "mixed"])
@pytest.mark.parametrize("dt", [1.0e2, 1.0e8, 1.0e10])
def test_reduced_solve_wide_matches_superlu(solver_mod, abi, hot1107, tile, dt):
    net, zb, X, ref = hot1107
    v = ref.evaluate_all_rates(zb.t9_1, zb.rho_1, zb.ye, X)
    jr, esr, mkr = ref.calculate_jacobian(v, X, dt)
    na = mkr.sum(axis=1)
    if dt >= 1.0e8:
        assert ((na > 32) & (na <= 64)).all(), na
    kw = dict(lu_precision=1) if tile == "mixed" else dict(lu_tile_max=tile)
    dev = _dev(solver_mod, net, abi, **kw)
    b = np.random.default_rng(7).normal(size=(zb.nz, net.nsp)) * 1e-3
    x = dev.solve_reduced(jr, esr, mkr, dt, b)
    xr, ierr = ref.solve_reduced(jr, esr, mkr, dt, b)
    assert (ierr == 0).all()
    err = np.abs(x - xr).max(axis=1) / np.abs(xr).max(axis=1)
    assert err.max() < 1e-9, err


def test_integrate_bd_hot_zones_within_reference_spread(solver_mod, abi, orc, wl):
    """Full 1e10 s integrations of the four hottest He-shell zones. Half of their Bader-Deuflhard
    steps are rejected, and in the reference's own algorithm 1-ulp changes of the input change the
    step sequence and the final abundances by up to tens of percent (see
    test_cpu_oracle.test_hot_heshell_zones_ill_conditioned). The device result must succeed, conserve
    mass, and lie within twice the spread that the checker itself shows under 1-ulp input changes and
    rounding-sized changes of dX/dt (three draws of each)."""
    import parity

    net = wl.network(1107)
    full = wl.heshell_batch(1024, net=net, seed=2)
    zb = full.take(np.argsort(-full.t9_0)[:4])
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    X0, _, ierr_r, _, _ = ref.integrate_network(zb.X, *args, nthreads=4)
    rel = lambda X: parity.zone_errors(X, X0)[0]
    spread = parity.checker_spread(ref, zb, X0, trials=(1, 2, 3), nthreads=4)
    dev = _dev(solver_mod, net, abi, integration_method=1)
    X, ye, ierr, st, _ = dev.integrate_network(zb.X, *args)
    assert (ierr == 0).all() and (ierr_r == 0).all()
    assert max(s.nvar1_max for s in st) > 32
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10
    assert (rel(X) <= np.maximum(2.0 * spread, 1e-6)).all(), (rel(X), spread)


def _heshell_sample(zb, n):
    """The 8 hottest zones of the batch and n - 8 evenly spaced others (bench.py's checker sample)."""
    hot = np.argsort(-zb.t9_0, kind="stable")[:8]
    rest = np.setdiff1d(np.arange(zb.nz), hot)
    return np.sort(np.concatenate([hot, rest[np.linspace(0, rest.size - 1, n - 8).astype(int)]]))


def test_heshell_batch_error_vs_checker(solver_mod, abi, orc, wl):
    """64 zones of the benchmarked He-shell batch (1109 species, Bader-Deuflhard over 1e10 s): the 8
    hottest and 56 evenly spaced others. Every zone succeeds on both sides and conserves mass. A zone
    whose checker result moves by less than 1e-6 under 1-ulp input changes must be within 1e-6
    relative (X > 1e-12) and 1e-15 absolute of the checker; a zone that the checker itself cannot pin
    to 1e-6 must lie within twice that spread (on the checker's side 26 of these 64 zones, nearly all
    with T9 > 0.24, move by more than 1e-6 under 1-ulp changes, by up to 72 %)."""
    import parity

    net = wl.network(1107)
    full = wl.heshell_batch(1024, net=net, seed=2)
    zb = full.take(_heshell_sample(full, 64))
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    Xr, _, ierr_r, st_r, _ = ref.integrate_network(zb.X, *args, nthreads=8)
    dev = _dev(solver_mod, net, abi, integration_method=1)
    X, _, ierr, st, _ = dev.integrate_network(zb.X, *args)
    assert (ierr == 0).all() and (ierr_r == 0).all(), (ierr, ierr_r)
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10
    rel, ab = parity.zone_errors(X, Xr)
    off = np.nonzero((rel > 1e-6) | (ab > 1e-15))[0]
    spread = np.zeros(zb.nz)
    if off.size:
        spread[off] = parity.checker_spread(ref, zb.take(off), Xr[off], nthreads=8)
    pinned = spread < 1e-6
    assert (rel[pinned] <= 1e-6).all() and (ab[pinned] <= 1e-15).all(), (rel[pinned].max(), ab[pinned].max())
    assert (rel[~pinned] <= 2.0 * spread[~pinned]).all(), (rel[~pinned], spread[~pinned])


def test_nse_matches_checker(solver_mod, abi, orc, wl):
    """compute_nse on the device (nuppn_nse) against the checker: same outcome, X within 1e-9 relative
    for X > 1e-12 and the chemical potentials within 1e-9 (isotope sums differ in rounding order)."""
    net = wl.network(1107)
    zb = wl.nse_batch(8, net=net)
    dev = _dev(solver_mod, net, abi)
    ref = orc.Oracle(net, abi.default_knobs())
    X, mp, mn, it, ierr = dev.compute_nse(zb.t9_0, zb.rho_0, zb.ye)
    Xr, mpr, mnr, itr, ierr_r = ref.compute_nse(zb.t9_0, zb.rho_0, zb.ye)
    assert (ierr == 0).all() and (ierr_r == 0).all()
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-9 and ab <= 1e-15, (rel, ab)
    assert np.abs(mp - mpr).max() <= 1e-9 * np.abs(mpr).max()
    assert np.abs(mn - mnr).max() <= 1e-9 * np.abs(mnr).max()


@pytest.mark.parametrize("method", [1, 0], ids=["rk", "euler"])
def test_integrate_nse_matches_checker(solver_mod, abi, orc, wl, method):
    """integrate_network above nse_min_t9 with i_nse = 1: NSE abundances with Ye evolved by the weak
    rates (Cash-Karp RK or Euler, nse_solver.F90). X within 1e-6 relative; the change of Ye within
    1e-6 of the checker's change."""
    net = wl.network(1107)
    zb = wl.nse_batch(6, net=net, dtwant=100.0)
    kw = dict(integration_method=1, i_nse=1, nse_weak_method=method)
    dev = _dev(solver_mod, net, abi, **kw)
    ref = orc.Oracle(net, abi.default_knobs(**kw))
    args = (zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    Xr, yer, ierr_r, str_, _ = ref.integrate_network(*args)
    assert (ierr == 0).all() and (ierr_r == 0).all()
    assert [s.nsucc for s in st] == [s.nsucc for s in str_]
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)
    assert (np.abs((ye - zb.ye) - (yer - zb.ye)) <= 1e-6 * np.abs(yer - zb.ye) + 1e-15).all(), (ye - yer)


def test_trajectories_within_reference_spread(solver_mod, abi, orc, wl):
    """tppnp-style trajectories (T9 falling from 2..5 with rho, Si28/Fe56 seed), 35 consecutive
    integrate_network intervals from 0 to ~1.2 s on the 1109-species network, each zone carrying its
    state and Bader-Deuflhard column between calls. Some trajectories are ill-conditioned in the
    reference's own algorithm (1-ulp input changes move their abundances by up to ~1e-5 here), so each
    must lie within 2x the checker's spread under such changes, or within 1e-6."""
    net = wl.network(1107)
    tr = wl.trajectory_batch(4, net=net, npts=41)
    kn = abi.default_knobs(integration_method=1)
    dev = _dev(solver_mod, net, abi, integration_method=1)
    ref = orc.Oracle(net, kn)

    def run(integrate, X, ye, **kw):
        bd = np.zeros(tr.nz, np.int32)
        for k in range(35):
            zb = tr.interval(k, X, ye)
            X, ye, ierr, _, bd = integrate(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant,
                                           bd_state=bd, **kw)
            assert (ierr == 0).all(), (k, ierr)
        return X

    Xd = run(dev.integrate_network, tr.X0, tr.ye0)
    Xr = run(ref.integrate_network, tr.X0, tr.ye0, nthreads=4)
    big = Xr > 1e-12
    rel = lambda X: (np.abs(X - Xr) * big / np.where(big, Xr, 1.0)).max(axis=1)
    spread = np.zeros(tr.nz)
    for trial in (1, 2):
        Xp = tr.X0 * (1.0 + np.random.default_rng(trial).choice([-1.0, 0.0, 1.0], size=tr.X0.shape) * 2.2e-16)
        spread = np.maximum(spread, rel(run(ref.integrate_network, Xp, tr.ye0, nthreads=4)))
    assert (rel(Xd) <= np.maximum(2.0 * spread, 1e-6)).all(), (rel(Xd), spread)
    assert np.abs(Xd.sum(axis=1) - 1.0).max() < 1e-10


def test_trajectory_from_nse_within_reference_spread(solver_mod, abi, orc, wl):
    """Explosive trajectories that start in NSE (T9_0 in [6.2, 8], X_0 from the NSE solve, i_nse = 1)
    and cool through nse_min_t9 = 6 into network integration, 21 points to 1 s, through
    nuppn_integrate_trajectories. While the trajectories are in NSE (the first 16 points) device and
    checker agree to 1e-9. After the exit the network integration starts from an NSE composition at
    T9 just below 6, where the reference's own result is not determined to better than O(1): 1-ulp
    changes of the T9 grid move its final abundances by up to ~4x. (Changes of X_0 do not probe this:
    NSE sub-steps recompute X from T, rho and Ye.) So for the whole trajectory every one must succeed,
    conserve mass, and lie (X and Ye) within 4x the largest deviation of three 1-ulp T9 perturbations
    of the checker, or 1e-6 (X) / 1e-8 (Ye)."""
    net = wl.network(1107)
    tr = wl.trajectory_batch(4, net=net, npts=21, t9_range=(6.2, 8.0), t_end=1.0)
    tt, t9, rho = tr.grids()
    kn = abi.default_knobs(integration_method=1, i_nse=1)
    dev = _dev(solver_mod, net, abi, integration_method=1, i_nse=1)
    ref = orc.Oracle(net, kn)
    X0, _, _, _, ierr0 = ref.compute_nse(t9[:, 0], rho[:, 0], np.linspace(0.48, 0.495, tr.nz))
    assert (ierr0 == 0).all()
    assert (t9[:, 15] >= 6.0).all() and (t9[:, -1] < 6.0).all()
    nse = slice(0, 16)
    Xd16 = dev.integrate_trajectories(X0, tt[:, nse], t9[:, nse], rho[:, nse])[0]
    Xr16 = ref.integrate_trajectories(X0, tt[:, nse], t9[:, nse], rho[:, nse], nthreads=4)[0]
    rel16, ab16 = _compare_X(Xd16, Xr16)
    assert rel16 <= 1e-9 and ab16 <= 1e-15, (rel16, ab16)
    Xd, yed, ierr, fail, st = dev.integrate_trajectories(X0, tt, t9, rho)
    Xr, yer, ierr_r, fail_r, _ = ref.integrate_trajectories(X0, tt, t9, rho, nthreads=4)
    assert (ierr == 0).all() and (ierr_r == 0).all() and (fail == -1).all()
    assert np.abs(Xd.sum(axis=1) - 1.0).max() < 1e-10
    big = Xr > 1e-12
    rel = lambda X: (np.abs(X - Xr) * big / np.where(big, Xr, 1.0)).max(axis=1)
    spread, ye_spread = np.zeros(tr.nz), np.zeros(tr.nz)
    for trial in (1, 2, 3):
        t9p = t9 * (1.0 + np.random.default_rng(trial).choice([-1.0, 1.0], size=t9.shape) * 2.2e-16)
        Xp, yep = ref.integrate_trajectories(X0, tt, t9p, rho, nthreads=4)[:2]
        spread = np.maximum(spread, rel(Xp))
        ye_spread = np.maximum(ye_spread, np.abs(yep - yer))
    assert (rel(Xd) <= np.maximum(4.0 * spread, 1e-6)).all(), (rel(Xd), spread)
    assert (np.abs(yed - yer) <= np.maximum(4.0 * ye_spread, 1e-8)).all(), (yed - yer, ye_spread)


def test_trajectory_entry_within_reference_spread(solver_mod, abi, orc, wl):
    """nuppn_integrate_trajectories (tppnp's trajectory loop for all zones in one launch) against the
    checker's restatement of the same loop, 4 trajectories of 36 points (0 to ~1.2 s): every
    trajectory succeeds, and each lies within 2x the checker's spread under 1-ulp input changes, or
    within 1e-6."""
    net = wl.network(1107)
    tr = wl.trajectory_batch(4, net=net, npts=41)
    tt, t9, rho = (g[:, :36] for g in tr.grids())
    kn = abi.default_knobs(integration_method=1)
    dev = _dev(solver_mod, net, abi, integration_method=1)
    ref = orc.Oracle(net, kn)
    Xd, yed, ierr, fail, st = dev.integrate_trajectories(tr.X0, tt, t9, rho)
    Xr, yer, ierr_r, fail_r, _ = ref.integrate_trajectories(tr.X0, tt, t9, rho, nthreads=4)
    assert (ierr == 0).all() and (ierr_r == 0).all() and (fail == -1).all()
    assert min(s.nsucc for s in st) >= 35
    big = Xr > 1e-12
    rel = lambda X: (np.abs(X - Xr) * big / np.where(big, Xr, 1.0)).max(axis=1)
    spread = np.zeros(tr.nz)
    for trial in (1, 2):
        Xp = tr.X0 * (1.0 + np.random.default_rng(trial).choice([-1.0, 0.0, 1.0], size=tr.X0.shape) * 2.2e-16)
        spread = np.maximum(spread, rel(ref.integrate_trajectories(Xp, tt, t9, rho, nthreads=4)[0]))
    assert (rel(Xd) <= np.maximum(2.0 * spread, 1e-6)).all(), (rel(Xd), spread)
    assert np.abs(yed - yer).max() < 1e-9
