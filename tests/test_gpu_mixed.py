"""Zones of three networks in one launch (nuppn_integrate_multi), the uneven-size batch: H-burning
zones on the ~200-species network (the Z <= 30 part of the reference's isotopedatabase.txt),
He-shell zones on the ~1100-species network and hot zones on the ~2500-species network (the first
2500 lines of isotopedatabase_all.txt), interleaved in one batch.

Every zone's result must equal, bit for bit, what nuppn_integrate gives for it on its own network
(the launch only chooses which network description a CTA reads), and lie within the parity bar of
the checker: 1e-6 relative for X > 1e-12, 1e-15 absolute below, or twice the checker's own spread
(four draws each of 1-ulp input changes and of rounding-sized dX/dt changes) for zones that the
checker itself cannot pin to 1e-6 (the H-burning zones of the ~200-species network move by up to
tens of percent under the latter).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mixed_networks_one_launch(solver_mod, abi, orc, wl):
    import parity

    nets, parts, _ = wl.mixed_batch(40)
    kn = abi.default_knobs(integration_method=1)
    devs = [solver_mod.NetworkSolver(n, kn, device=0) for n in nets]
    take = 4
    subs = [(i, zb.take(np.arange(take))) for i, zb in parts]
    ldx = max(n.nsp for n in nets)
    # interleave the three networks' zones: z = 3 k + i
    nz = 3 * take
    X = np.full((nz, ldx), 1e-99)
    net_of = np.zeros(nz, np.int32)
    cols = {f: np.zeros(nz) for f in ("t9_0", "t9_1", "rho_0", "rho_1", "ye", "dtwant")}
    for i, zb in subs:
        for k in range(take):
            z = 3 * k + i
            X[z, :nets[i].nsp] = zb.X[k]
            net_of[z] = i
            for f in cols:
                cols[f][z] = getattr(zb, f)[k]
    args = [cols[f] for f in ("t9_0", "t9_1", "rho_0", "rho_1", "ye", "dtwant")]
    Xm, yem, ierrm, stm, bdm = solver_mod.integrate_multi(devs, net_of, X, *args)
    assert (ierrm == 0).all(), ierrm
    for i, zb in subs:
        rows = np.nonzero(net_of == i)[0]
        nsp = nets[i].nsp
        zargs = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
        Xs, yes, ierrs, sts, _ = devs[i].integrate_network(zb.X, *zargs)
        assert (ierrs == 0).all()
        assert np.array_equal(Xm[rows, :nsp], Xs), nets[i].name  # same kernel arithmetic, one launch
        assert np.array_equal(yem[rows], yes)
        assert [stm[r].nsucc for r in rows] == [s.nsucc for s in sts]
        assert (Xm[rows, nsp:] == 1e-99).all()  # columns beyond the zone's network untouched
        ref = orc.Oracle(nets[i], kn)
        Xr, _, ierr_r, _, _ = ref.integrate_network(zb.X, *zargs, nthreads=8)
        assert (ierr_r == 0).all()
        assert np.abs(Xs.sum(axis=1) - 1.0).max() < 1e-10
        rel, ab = parity.zone_errors(Xs, Xr)
        off = np.nonzero((rel > 1e-6) | (ab > 1e-15))[0]
        spread = np.zeros(zb.nz)
        if off.size:
            spread[off] = parity.checker_spread(ref, zb.take(off), Xr[off], trials=(1, 2, 3, 4), nthreads=8)
        pinned = spread < 1e-6
        assert (rel[pinned] <= 1e-6).all() and (ab[pinned] <= 1e-15).all(), (nets[i].name, rel, ab)
        assert (rel[~pinned] <= 2.0 * spread[~pinned]).all(), (nets[i].name, rel, spread)
    big = np.nonzero(net_of == 2)[0]
    assert max(stm[r].nvar1_max for r in big) > 64  # the large network reaches the sparse LU
