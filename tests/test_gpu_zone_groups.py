"""The one-zone-per-warp integration kernel (knob threads_per_zone = 32) against the CPU checker,
through the C ABI, on the same cases as the one-zone-per-CTA kernel's parity tests.

Each warp integrates its own zone end to end (rates, dynamic-network Jacobian, compaction, LU, step
control), so a CTA carries up to eight zones. The arithmetic of every per-zone sum in the reference's
order is the same as in the CTA kernel; group-wide reductions (sums of X, error maxima) are taken over
one warp instead of eight, which changes rounding only. Tolerances are those of test_gpu_parity.py:
1e-6 relative for X > 1e-12 and 1e-15 absolute below, or the checker's own spread under 1-ulp input
changes for zones that are ill-conditioned in the reference's algorithm.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WARP = dict(threads_per_zone=32)
SHAPES = {"warp8": dict(threads_per_zone=32),
          "warp4_global": dict(threads_per_zone=32, zones_per_cta=4, zone_smem=4096)}


def _dev(solver_mod, net, abi, **kw):
    return solver_mod.NetworkSolver(net, abi.default_knobs(**kw), device=0)


def _compare_X(X, Xr):
    big = Xr > 1e-12
    rel = np.abs(X - Xr)[big] / Xr[big]
    small = np.abs(X - Xr)[~big]
    return rel.max(initial=0.0), small.max(initial=0.0)


@pytest.mark.parametrize("shape", list(SHAPES), ids=list(SHAPES))
@pytest.mark.parametrize("tile", [0, -1], ids=["tile", "sparse"])
def test_warp_zones_bd_matches_checker(solver_mod, abi, orc, wl, tile, shape):
    """Bader-Deuflhard, 6 zones of the 300-species network, tile and sparse LU; with zone_smem = 4 KB
    every active subsystem lives in the zone's global workspace instead of shared memory."""
    net = wl.network(300)
    zb = wl.heshell_batch(6, net=net, seed=11)
    dev = _dev(solver_mod, net, abi, integration_method=1, lu_tile_max=tile, **SHAPES[shape])
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    args = (zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    Xr, yer, ierr_r, str_, _ = ref.integrate_network(*args)
    assert (ierr == ierr_r).all()
    assert [s.nsucc for s in st] == [s.nsucc for s in str_]
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10


@pytest.mark.parametrize("tile", [0, -1], ids=["tile", "sparse"])
def test_warp_zones_be_hburn_matches_checker(solver_mod, abi, orc, wl, tile):
    """Backward Euler, the ppn H-burning frame (300 species), frame steps 1..39 from the checker's
    state after the first (ill-conditioned) one, as in test_gpu_parity."""
    net = wl.network(300)
    zb, dts = wl.hburn_zone(net)
    dev = _dev(solver_mod, net, abi, integration_method=0, lu_tile_max=tile, **WARP)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=0))
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1)
    X0, _, ierr0, _, _ = dev.integrate_network(zb.X, *args, zb.ye, dts[0])
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


def test_warp_zones_heshell_error_vs_checker(solver_mod, abi, orc, wl):
    """64 zones of the benchmarked He-shell batch (1109 species, 1e10 s): the 8 hottest and 56 evenly
    spaced others, judged as in test_gpu_parity.test_heshell_batch_error_vs_checker."""
    import parity

    net = wl.network(1107)
    full = wl.heshell_batch(1024, net=net, seed=2)
    hot = np.argsort(-full.t9_0, kind="stable")[:8]
    rest = np.setdiff1d(np.arange(full.nz), hot)
    zb = full.take(np.sort(np.concatenate([hot, rest[np.linspace(0, rest.size - 1, 56).astype(int)]])))
    args = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    Xr, _, ierr_r, _, _ = ref.integrate_network(zb.X, *args, nthreads=8)
    dev = _dev(solver_mod, net, abi, integration_method=1, **WARP)
    X, _, ierr, st, _ = dev.integrate_network(zb.X, *args)
    assert (ierr == 0).all() and (ierr_r == 0).all(), (ierr, ierr_r)
    assert max(s.nvar1_max for s in st) > 32  # 64-row tiles are exercised
    assert np.abs(X.sum(axis=1) - 1.0).max() < 1e-10
    rel, ab = parity.zone_errors(X, Xr)
    off = np.nonzero((rel > 1e-6) | (ab > 1e-15))[0]
    spread = np.zeros(zb.nz)
    if off.size:
        spread[off] = parity.checker_spread(ref, zb.take(off), Xr[off], nthreads=8)
    pinned = spread < 1e-6
    assert (rel[pinned] <= 1e-6).all() and (ab[pinned] <= 1e-15).all(), (rel[pinned].max(), ab[pinned].max())
    assert (rel[~pinned] <= 2.0 * spread[~pinned]).all(), (rel[~pinned], spread[~pinned])


def test_warp_zones_trajectories_within_reference_spread(solver_mod, abi, orc, wl):
    """nuppn_integrate_trajectories with one trajectory per warp: 4 trajectories of 36 points (0 to
    ~1.2 s, 1109 species), each within 2x the checker's 1-ulp spread or 1e-6."""
    net = wl.network(1107)
    tr = wl.trajectory_batch(4, net=net, npts=41)
    tt, t9, rho = (g[:, :36] for g in tr.grids())
    dev = _dev(solver_mod, net, abi, integration_method=1, **WARP)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    Xd, yed, ierr, fail, st = dev.integrate_trajectories(tr.X0, tt, t9, rho)
    Xr, yer, ierr_r, fail_r, _ = ref.integrate_trajectories(tr.X0, tt, t9, rho, nthreads=4)
    assert (ierr == 0).all() and (ierr_r == 0).all() and (fail == -1).all()
    big = Xr > 1e-12
    rel = lambda X: (np.abs(X - Xr) * big / np.where(big, Xr, 1.0)).max(axis=1)
    spread = np.zeros(tr.nz)
    for trial in (1, 2):
        Xp = tr.X0 * (1.0 + np.random.default_rng(trial).choice([-1.0, 0.0, 1.0], size=tr.X0.shape) * 2.2e-16)
        spread = np.maximum(spread, rel(ref.integrate_trajectories(Xp, tt, t9, rho, nthreads=4)[0]))
    assert (rel(Xd) <= np.maximum(2.0 * spread, 1e-6)).all(), (rel(Xd), spread)
    assert np.abs(yed - yer).max() < 1e-9


def test_warp_zones_nse_matches_checker(solver_mod, abi, orc, wl):
    """integrate_network above nse_min_t9 with i_nse = 1 (Cash-Karp Ye coupling): X within 1e-6."""
    net = wl.network(1107)
    zb = wl.nse_batch(6, net=net, dtwant=100.0)
    kw = dict(integration_method=1, i_nse=1, nse_weak_method=1)
    dev = _dev(solver_mod, net, abi, **kw, **WARP)
    ref = orc.Oracle(net, abi.default_knobs(**kw))
    args = (zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    Xr, yer, ierr_r, str_, _ = ref.integrate_network(*args)
    assert (ierr == 0).all() and (ierr_r == 0).all()
    rel, ab = _compare_X(X, Xr)
    assert rel <= 1e-6 and ab <= 1e-15, (rel, ab)


def test_shape_knobs_are_checked(solver_mod, abi, wl):
    """Kernel-shape knobs outside their ranges are refused at creation and by set_knobs."""
    net = wl.network(300)
    for bad in (dict(threads_per_zone=48), dict(threads_per_zone=512), dict(zones_per_cta=9),
                dict(threads_per_zone=32, zone_smem=300 * 1024)):
        with pytest.raises(solver_mod.NuppnError):
            _dev(solver_mod, net, abi, **bad)
    dev = _dev(solver_mod, net, abi, integration_method=1)
    with pytest.raises(solver_mod.NuppnError):
        dev.set_knobs(abi.default_knobs(integration_method=1, zones_per_cta=-1))
    dev.set_knobs(abi.default_knobs(integration_method=1, **WARP))  # a valid shape change is taken


def test_autotune_picks_a_shape_and_keeps_results(solver_mod, abi, orc, wl):
    """nuppn_autotune times every candidate shape on the batch, marks the fastest as chosen and applies
    it; the tuned handle then integrates the batch to the checker's results (1e-6, or twice the
    checker's own spread on zones it cannot pin to 1e-6)."""
    net = wl.network(300)
    zb = wl.heshell_batch(48, net=net, seed=17)
    dev = _dev(solver_mod, net, abi, integration_method=1)
    args = (zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    rep = dev.autotune(*args)
    assert len(rep) >= 2 and sum(r["chosen"] for r in rep) == 1
    best = max((r for r in rep if r["zone_steps_per_s"] > 0), key=lambda r: r["zone_steps_per_s"])
    assert best["chosen"] == 1 and best["ms"] > 0 and best["zones_per_sm"] >= 1
    assert {0, 64, 128, 32} <= {r["threads_per_zone"] for r in rep}
    X, ye, ierr, st, _ = dev.integrate_network(*args)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    Xr, _, ierr_r, str_, _ = ref.integrate_network(*args, nthreads=8)
    assert (ierr == 0).all() and (ierr_r == 0).all()
    import parity

    rel, ab = parity.zone_errors(X, Xr)
    off = np.nonzero((rel > 1e-6) | (ab > 1e-15))[0]
    spread = np.zeros(zb.nz)
    if off.size:
        spread[off] = parity.checker_spread(ref, zb.take(off), Xr[off], nthreads=8)
    pinned = spread < 1e-6
    assert (rel[pinned] <= 1e-6).all() and (ab[pinned] <= 1e-15).all(), (rel, ab)
    assert (rel[~pinned] <= 2.0 * spread[~pinned]).all(), (rel, spread)
