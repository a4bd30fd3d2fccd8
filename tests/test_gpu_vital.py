"""The reference's own VITAL formulas on the device (physics/source/vital.F90:339-571, slots 1-9, 14-17
and 73) against the oracle's restatement, through the C ABI, on a network built with
``vital="reference"``: every rate within 1e-11 relative (device exp/pow vs glibc) with screening on,
the formula slots equal to the restated formulas with screening off, dX/dt from those rates as the
rates parity tests bound it, and a descriptor naming a slot without a formula refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vnet(sn):
    return sn.build_network(300, vital="reference")


def _conditions(net, n=12, seed=5):
    rng = np.random.default_rng(seed)
    t9 = np.concatenate([[0.0011, 0.004, 0.008, 0.015, 0.03], 10.0 ** rng.uniform(-1.5, 0.7, n - 5)])
    rho = 10.0 ** rng.uniform(1.0, 5.0, n)
    X = np.full((n, net.nsp), 1e-99)
    for i in range(n):
        X[i, net.species_index("PROT ")] = rng.uniform(0.3, 0.75)
        X[i, net.species_index("HE  4")] = 0.98 - X[i, net.species_index("PROT ")]
        for name in ("C  12", "N  14", "O  16", "BE  7", "LI  7", "N  13"):
            X[i, net.species_index(name)] = 10.0 ** rng.uniform(-8, -2.5)
        X[i] /= X[i].sum()
    return t9, rho, np.full(n, 0.85), X


def test_vital_rates_match_checker(solver_mod, abi, orc, vnet):
    t9, rho, ye, X = _conditions(vnet)
    dev = solver_mod.NetworkSolver(vnet, abi.default_knobs(), device=0)
    ref = orc.Oracle(vnet, abi.default_knobs())
    v = dev.evaluate_all_rates(t9, rho, ye, X)
    vr = ref.evaluate_all_rates(t9, rho, ye, X)
    big = vr > 1e-90
    rel = np.abs(v - vr)[big] / vr[big]
    assert rel.max() < 1e-11, rel.max()
    assert (v[~big] <= 1e-89).all()
    d = dev.calculate_dxdt(vr, X)
    dr = ref.calculate_dxdt(vr, X)
    assert (np.abs(d - dr) <= 1e-12 * np.abs(dr).max(axis=1, keepdims=True)).all()


def test_vital_slots_are_the_formulas(solver_mod, abi, orc, sn, vnet):
    t9, rho, ye, X = _conditions(vnet, seed=6)
    kn = abi.default_knobs()
    kn.screen_option = 0
    v = solver_mod.NetworkSolver(vnet, kn, device=0).evaluate_all_rates(t9, rho, ye, X)
    form = np.asarray(vnet.vt_form)
    rows = np.nonzero(np.asarray(vnet.src) == sn.SRC_VITAL)[0]
    ip = vnet.species_index("PROT ")
    seen = set()
    for f, r in zip(form, rows):
        if f <= 0:
            continue
        for z in range(len(t9)):
            want = max(orc.vital_reference(int(f), t9[z], rho[z], X[z, ip]) * vnet.rfac[r], 1e-99)
            assert abs(v[z, r] - want) <= 1e-11 * want, (int(f), t9[z], v[z, r], want)
            seen.add(int(f))
    assert {1, 2, 3, 4, 5, 6, 7, 8, 9, 14, 15, 73} <= seen


def test_descriptor_without_formula_refused(solver_mod, abi, sn):
    net = sn.build_network(300, vital="reference")
    form = np.asarray(net.vt_form).copy()
    form[np.argmax(form == 8)] = 10  # V(10) is off in the reference (IPPIV = 0): no formula here
    net.vt_form = form
    with pytest.raises(solver_mod.NuppnError, match="vt_form"):
        solver_mod.NetworkSolver(net, abi.default_knobs(), device=0)
