"""nuppn_serve_*: continuous batching of independent requests (config 5's serving loop).

A request is one zone (integrate_network's arguments) or one tppnp trajectory. The server admits
pending requests on any idle lane while other lanes' batches run, so a request may share a launch
with any others. Its result must not depend on that: the same zone or trajectory gives the same
result alone, in a mix of zones and trajectories spread over several lanes in small batches, and
through the batched entry points, within the parity tests' tolerance (1e-6 relative for X > 1e-12,
1e-15 absolute below).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(a, b):
    big = b > 1e-12
    rel = (np.abs(a - b)[big] / b[big]).max(initial=0.0)
    ab = np.abs(a - b)[~big].max(initial=0.0)
    return rel <= 1e-6 and ab <= 1e-15, (rel, ab)


def test_serve_alone_and_in_mix(solver_mod, abi, wl):
    net = wl.network(1107)
    zb = wl.heshell_batch(24, net=net, seed=5)
    tr = wl.trajectory_batch(2, net=net, npts=11)
    tt, t9, rho = tr.grids()
    dev = solver_mod.NetworkSolver(net, abi.default_knobs(integration_method=1), device=0)
    Xb, yeb, ierrb, stb, _ = dev.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    Xt, yet, ierrt, failt, _ = dev.integrate_trajectories(tr.X0, tt, t9, rho)
    assert (ierrb == 0).all() and (ierrt == 0).all()

    srv = solver_mod.Server(dev, lanes=3, max_batch=4)
    try:
        zone = lambda z: srv.submit(zb.X[z], zb.t9_0[z], zb.t9_1[z], zb.rho_0[z], zb.rho_1[z], zb.ye[z], zb.dtwant[z])
        traj = lambda i: srv.submit_trajectory(tr.X0[i], tt[i], t9[i], rho[i])
        alone_z = srv.wait(zone(7))
        alone_t = srv.wait(traj(1))
        ids = []
        for z in range(zb.nz):  # zones and trajectories interleaved: batches of one kind, several lanes
            ids.append(("z", z, zone(z)))
            if z in (5, 17):
                i = 0 if z == 5 else 1
                ids.append(("t", i, traj(i)))
        res = [(k, i, srv.wait(rid)) for k, i, rid in ids]
        info = srv.info()
        assert info.lanes == 3 and info.batches >= 2 + 24 // 4 + 1, (info.lanes, info.batches)
        assert info.pending == 0 and info.in_flight == 0
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


def test_serve_rejects_bad_arguments(solver_mod, abi, wl):
    net = wl.network(300)
    dev = solver_mod.NetworkSolver(net, abi.default_knobs(), device=0)
    srv = solver_mod.Server(dev, lanes=1)
    try:
        with pytest.raises(solver_mod.NuppnError):
            srv.poll(12345)  # unknown id
        with pytest.raises(solver_mod.NuppnError):
            srv.submit_trajectory(np.zeros(net.nsp), [0.0], [1.0], [1.0])  # one point
    finally:
        srv.close()
