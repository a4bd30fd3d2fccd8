"""nuppn_serve_*: the device-resident request loop (config 5's serving path).

A request is one zone (integrate_network's arguments) or one tppnp trajectory. A persistent launch
takes requests from a device queue as they are submitted, one per zone group, and hands each result
back as soon as that zone is done, so requests that arrive while others run share the GPU with them.
A request's result must not depend on what it shares the GPU with: the same zone or trajectory gives
the same result alone, in a mix of zones and trajectories, and through the batched entry points,
within the parity tests' tolerance (1e-6 relative for X > 1e-12, 1e-15 absolute below).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(a, b):
    big = b > 1e-12
    rel = (np.abs(a - b)[big] / b[big]).max(initial=0.0)
    ab = np.abs(a - b)[~big].max(initial=0.0)
    return rel <= 1e-6 and ab <= 1e-15, (rel, ab)


@pytest.mark.parametrize("shape", [{}, {"threads_per_zone": 32}], ids=["cta", "warp"])
def test_serve_alone_and_in_mix(solver_mod, abi, wl, shape):
    """24 He-shell zones and 2 trajectories of the 1109-species network, each alone, then all of them
    interleaved through a queue smaller than the request count (queue slots are reused), against the
    batched entry points."""
    net = wl.network(1107)
    zb = wl.heshell_batch(24, net=net, seed=5)
    tr = wl.trajectory_batch(2, net=net, npts=11)
    tt, t9, rho = tr.grids()
    dev = solver_mod.NetworkSolver(net, abi.default_knobs(integration_method=1, **shape), device=0)
    Xb, yeb, ierrb, stb, _ = dev.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    Xt, yet, ierrt, failt, _ = dev.integrate_trajectories(tr.X0, tt, t9, rho)
    assert (ierrb == 0).all() and (ierrt == 0).all()

    srv = solver_mod.Server(dev, slots=16, queue=16)
    try:
        zone = lambda z: srv.submit(zb.X[z], zb.t9_0[z], zb.t9_1[z], zb.rho_0[z], zb.rho_1[z], zb.ye[z], zb.dtwant[z])
        traj = lambda i: srv.submit_trajectory(tr.X0[i], tt[i], t9[i], rho[i])
        alone_z = srv.wait(zone(7))
        alone_t = srv.wait(traj(1))
        ids = []
        for z in range(zb.nz):
            ids.append(("z", z, zone(z)))
            if z in (5, 17):
                i = 0 if z == 5 else 1
                ids.append(("t", i, traj(i)))
        res = [(k, i, srv.wait(rid)) for k, i, rid in ids]
        info = srv.info()
        assert info.slots >= 1 and info.queue >= info.slots and info.ctas >= 1
        assert info.published == 2 + len(ids) and info.completed == info.published
        assert info.pending == 0 and info.in_flight == 0 and info.launches >= 1
    finally:
        srv.close()

    for kind, i, (X, ye, ierr, st, bd, fail) in res:
        assert ierr == 0, (kind, i, ierr)
        ref = Xb[i] if kind == "z" else Xt[i]
        ok, err = _close(X, ref)
        assert ok, (kind, i, err)
        if kind == "z":
            assert st.nsucc == stb[i].nsucc and abs(ye - yeb[i]) <= 1e-12
        else:
            assert fail == -1 and abs(ye - yet[i]) <= 1e-12
    mix_z = next(r for k, i, r in res if k == "z" and i == 7)
    mix_t = next(r for k, i, r in res if k == "t" and i == 1)
    assert _close(alone_z[0], mix_z[0])[0] and _close(alone_t[0], mix_t[0])[0]
    assert alone_z[3].nsucc == mix_z[3].nsucc and alone_t[3].nsucc == mix_t[3].nsucc


def test_serve_overlaps_requests_and_relaunches(solver_mod, abi, wl):
    """Continuous batching: short zone requests submitted after a long trajectory finish before it
    (no batch waits for its slowest member); after the loop has left on its own (idle), a new request
    relaunches it and still matches the batched entry point."""
    net = wl.network(1107)
    zb = wl.heshell_batch(8, net=net, seed=9)
    zb.t9_0[:] = 0.11  # cool zones: few sub-steps each
    zb.t9_1[:] = 0.11
    tr = wl.trajectory_batch(1, net=net, npts=201)
    tt, t9, rho = tr.grids()
    dev = solver_mod.NetworkSolver(net, abi.default_knobs(integration_method=1), device=0)
    Xb, _, ierrb, _, _ = dev.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    assert (ierrb == 0).all()
    srv = solver_mod.Server(dev, slots=32)
    try:
        t_id = srv.submit_trajectory(tr.X0[0], tt[0], t9[0], rho[0])
        z_ids = [srv.submit(zb.X[z], zb.t9_0[z], zb.t9_1[z], zb.rho_0[z], zb.rho_1[z], zb.ye[z], zb.dtwant[z])
                 for z in range(zb.nz)]
        done_at = {}
        t_end = time.monotonic() + 300.0
        while len(done_at) < 1 + zb.nz and time.monotonic() < t_end:
            for rid in [t_id] + z_ids:
                if rid not in done_at and srv.poll(rid) is not None:
                    done_at[rid] = time.monotonic()
            time.sleep(1e-4)
        assert len(done_at) == 1 + zb.nz
        assert max(done_at[r] for r in z_ids) < done_at[t_id]
        launches = srv.info().launches
        time.sleep(0.5)  # the loop leaves after a few tens of ms without requests
        X, ye, ierr, st, bd, fail = srv.wait(srv.submit(zb.X[3], zb.t9_0[3], zb.t9_1[3], zb.rho_0[3], zb.rho_1[3],
                                                        zb.ye[3], zb.dtwant[3]))
        assert srv.info().launches == launches + 1
        assert ierr == 0 and _close(X, Xb[3])[0]
    finally:
        srv.close()


def test_serve_rejects_bad_arguments(solver_mod, abi, wl):
    net = wl.network(300)
    dev = solver_mod.NetworkSolver(net, abi.default_knobs(), device=0)
    srv = solver_mod.Server(dev, slots=1)
    try:
        with pytest.raises(solver_mod.NuppnError):
            srv.poll(12345)  # unknown id
        with pytest.raises(solver_mod.NuppnError):
            srv.submit_trajectory(np.zeros(net.nsp), [0.0], [1.0], [1.0])  # one point
        n = 600  # more points than a served trajectory may have
        with pytest.raises(solver_mod.NuppnError):
            srv.submit_trajectory(np.zeros(net.nsp), np.linspace(0, 1, n), np.ones(n), np.ones(n))
    finally:
        srv.close()


def test_serve_small_dt_outcomes_match_checker(solver_mod, abi, orc, wl):
    """48 H-burning zones of the serving stream (300 species, T9 U[0.015, 0.08], rho log-U[1, 1e3],
    1e10 s, Bader-Deuflhard) through the server: each zone's outcome (success or SMALL_DT, the step
    falling below 1e-30 s) equals the checker's on every zone whose checker outcome stays the same
    under two draws of 1-ulp input changes (on the others the reference's own outcome is not
    determined by its input), and successful zones meet the parity bar. These zones move by 1-50 %
    under rounding-sized changes of dX/dt in the reference's own algorithm, so their bar is twice the
    checker's spread over four draws of each perturbation (with two draws, the checker itself under
    another draw falls outside twice the spread on 2 of 32 zones; with four, on none)."""
    import parity

    net = wl.network(300)
    hb, _ = wl.hburn_zone(net)
    rng = np.random.default_rng(11)
    n = 48
    t9 = rng.uniform(0.015, 0.08, n)
    rho = 10.0 ** rng.uniform(0.0, 3.0, n)
    X = np.repeat(hb.X, n, axis=0)
    ye = np.repeat(hb.ye, n)
    kn = abi.default_knobs(integration_method=1)
    ref = orc.Oracle(net, kn)
    Xr, _, ierr_r, _, _ = ref.integrate_network(X, t9, t9, rho, rho, ye, np.full(n, 1e10), nthreads=8)
    stable = np.ones(n, bool)
    for trial in (1, 2):
        Xp = X * (1.0 + np.random.default_rng(trial).choice([-1.0, 0.0, 1.0], size=X.shape) * 2.2e-16)
        ie = ref.integrate_network(Xp, t9, t9, rho, rho, ye, np.full(n, 1e10), nthreads=8)[2]
        stable &= ie == ierr_r
    assert (ierr_r == 11).sum() >= 5 and stable.sum() >= 32
    dev = solver_mod.NetworkSolver(net, kn, device=0)
    srv = solver_mod.Server(dev)
    try:
        ids = [srv.submit(X[z], t9[z], t9[z], rho[z], rho[z], ye[z], 1.0e10) for z in range(n)]
        res = [srv.wait(i) for i in ids]
    finally:
        srv.close()
    ierr = np.array([r[2] for r in res])
    Xd = np.array([r[0] for r in res])
    assert (ierr[stable] == ierr_r[stable]).all(), (ierr[stable], ierr_r[stable])
    assert set(np.unique(ierr)) <= {0, 11}
    ok = stable & (ierr == 0)
    rel, ab = parity.zone_errors(Xd[ok], Xr[ok])
    off = (rel > 1e-6) | (ab > 1e-15)
    if off.any():  # only zones the checker itself cannot pin to 1e-6
        sub = np.nonzero(ok)[0][off]
        spread = parity.checker_spread(ref, wl.ZoneBatch(X=X[sub], t9_0=t9[sub], t9_1=t9[sub], rho_0=rho[sub],
                                                        rho_1=rho[sub], ye=ye[sub], dtwant=np.full(sub.size, 1e10)),
                                       Xr[sub], trials=(1, 2, 3, 4), nthreads=8)
        assert (rel[off] <= 2.0 * spread).all(), (rel[off], spread)
