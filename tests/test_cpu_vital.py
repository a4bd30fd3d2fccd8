"""The reference's own VITAL formulas (physics/source/vital.F90:339-571: the pp chains, slots 1-9, and
the first CNO reactions, slots 14-17 and 73) on the CPU.

The oracle's restatement is checked against a second, independent transcription of the same Fortran
lines written below in numpy-free Python, over a T9 sweep that crosses every threshold of the routine
(T9 = 1e-3, 1.2e-3, 5e-3, the T9PPMAX clip at 10). A network built with ``vital="reference"`` carries
those slots' reactions with the formulas as their rates (the network loop leaves the reactions to
VITAL); the oracle's rate evaluation (screening off) returns the formulas through the descriptor, and
an H-burning zone integrates on it.
"""
import math

import numpy as np
import pytest

SLOTS = (1, 2, 3, 4, 5, 6, 7, 8, 9, 14, 15, 16, 17, 73)


def _exv(x):  # vital.F90:2583-2593
    if x > 200.0:
        return (x - 200.0) * math.exp(200.0)
    if x < -200.0:
        return -math.exp(-200.0) / (x + 200.0)
    return math.exp(x)


def _vital(slot, T9, rho, xp):
    T9 = min(T9, 10.0)  # vital.F90:230
    t13, t14 = T9 ** (1.0 / 3.0), T9 ** 0.25
    t12 = t14 * t14
    t23, t32, t43 = t13 * t13, T9 * t12, T9 * t13
    t53 = T9 * t23
    m13, m23, m32 = 1.0 / t13, 1.0 / t23, 1.0 / t32
    V = {5: 1.34e-10 / t12 * (1 - 0.537 * t13 + 3.86 * t23 + 0.0027 / T9 * _exv(2.515e-3 / T9)) * rho * 0.5 * (1 + xp)}
    if T9 < 1e-3 or T9 > 10.0:
        V[5] = min(V[5], 1.51e-7)
    if T9 >= 1e-3 and 1.2e-3 < T9 < 10.0:
        V[1] = 4.01e-15 * m23 * _exv(-3.38 * m13) * (1 + 0.123 * t13 + 1.09 * t23 + 0.938 * T9) * rho
        V[2] = 2.24e3 * m23 * _exv(-3.72 * m13) * (1 + 0.112 * t13 + 3.38 * t23 + 2.65 * T9) * rho
        V[3] = 6.04e10 * m23 * _exv(-12.276 * m13) * (1 + 0.034 * t13 - 0.522 * t23 - 0.124 * T9 + 0.353 * t43
                                                       + 0.213 * t53) * rho
        tt = T9 / (1 + 0.0495 * T9)
        V[4] = 5.61e6 * tt ** (5.0 / 6.0) / t32 * _exv(-12.826 / tt ** (1.0 / 3.0)) * rho
        ta = T9 / (1 + 0.759 * T9)
        V[6] = (1.096e9 / t23 * _exv(-8.472 / t13) - 4.83e8 * ta ** (5.0 / 6.0) / t32 * _exv(-8.472 / ta ** (1.0 / 3.0))
                + 1.06e10 / t32 * _exv(-30.442 / T9)) * rho
        V[7] = (3.11e5 / t23 * _exv(-10.262 / t13) + 2.53e3 / t32 * _exv(-7.306 / T9)) * rho
        V[9] = 1.30e10 * t32 * _exv(-1.595 / T9) / rho * V[7]
        V[8] = 0.896
    if T9 > 5e-3:
        V[14] = (2e7 * m23 * _exv(-13.692 * m13 - (T9 / 0.46) ** 2) * (1 + 9.89 * T9 - 59.8 * T9 ** 2 + 266 * T9 ** 3)
                 + 1e5 * m32 * _exv(-4.913 / T9) + 4.24e5 * m32 * _exv(-21.62 / T9)) * rho
        V[73] = V[14] / rho * 8.84e9 * t32 * _exv(-22.553 / T9)
        V[15] = (9.57e7 * m23 * _exv(-13.72 * m13 - T9 * T9) * (1 + 3.56 * T9) + 1.5e6 * m32 * _exv(-5.93 / T9)
                 + math.exp(-12.057 / T9) * 6.83e5 / T9 ** 0.864) * rho
        # the reference multiplies only the second term by RHO*PROTOFAK
        V[16] = (4.04e7 * m23 * _exv(-15.202 * m13 - (T9 / 1.191) ** 2) * (1 + 0.027 * t13 - 0.803 * t23 - 0.154 * T9
                                                                          + 5.0 * t43 + 2.44 * t53)
                 + 2.43e5 * m32 * _exv(-6.348 / T9) * rho)
        V[17] = (4.9e7 / t23 * _exv(-15.228 / t13 - (T9 / 3.294) ** 2) * (1 + 0.027 * t13 - 0.778 * t23 - 0.149 * T9
                                                                          + 0.261 * t43 + 0.127 * t53)
                 + 2.37e3 / t32 * _exv(-3.011 / T9) + 2.19e4 * _exv(-12.53 / T9)) * rho
    return V.get(slot, 0.0)


T9S = (5e-4, 1e-3, 1.1e-3, 1.3e-3, 4e-3, 6e-3, 0.01, 0.02, 0.05, 0.1, 0.3, 1.0, 3.0, 9.9, 10.0, 12.0)


def test_oracle_vital_formulas_against_a_second_transcription(orc):
    worst = 0.0
    for slot in SLOTS + (10, 11, 18, 44):  # 10-13 are off (IPPIV = 0); others have no formula here
        for T9 in T9S:
            for rho in (1.0, 1e2, 1e5):
                a, b = orc.vital_reference(slot, T9, rho, 0.7), _vital(slot, T9, rho, 0.7)
                if b == 0.0:
                    assert a == 0.0, (slot, T9)
                    continue
                worst = max(worst, abs(a - b) / abs(b))
    assert worst < 1e-13, worst
    # thresholds: nothing below T9 = 1e-3 but v(5), clamped; pp rates off at the T9PPMAX clip
    assert orc.vital_reference(1, 9e-4, 1e2, 0.7) == 0.0 and orc.vital_reference(5, 9e-4, 1e2, 0.7) <= 1.51e-7
    assert orc.vital_reference(1, 12.0, 1e2, 0.7) == 0.0 and orc.vital_reference(14, 12.0, 1e2, 0.7) > 0.0
    assert orc.vital_reference(14, 5e-3, 1e2, 0.7) == 0.0 and orc.vital_reference(14, 5.1e-3, 1e2, 0.7) > 0.0


def test_reference_vital_network(orc, abi, sn):
    net = sn.build_network(300, vital="reference")
    tmpl = sn.build_network(300)
    assert not np.asarray(tmpl.vt_form).any()  # the default keeps the templates
    form = np.asarray(net.vt_form)
    vital_rows = np.nonzero(np.asarray(net.src) == sn.SRC_VITAL)[0]
    assert len(vital_rows) == len(form)
    slots = {int(f): int(r) for f, r in zip(form, vital_rows) if f > 0}
    assert set(slots) <= set(SLOTS) and {1, 2, 3, 4, 5, 6, 7, 8, 9, 14, 15, 73} <= set(slots)
    # the network loop leaves C12(p,g)N13 to VITAL slot 14: one reaction of that kind only
    ic12, ip, in13 = (net.species_index(n) for n in ("C  12", "PROT ", "N  13"))
    k = np.asarray(net.k)
    same = np.nonzero((k[:, 0] == ic12) & (k[:, 2] == ip) & (k[:, 6] == in13))[0]
    assert same.tolist() == [slots[14]]
    kn = abi.default_knobs()
    kn.screen_option = 0  # screening (evaluate_rates.F90:58-121) would scale the charged-particle slots
    ref = orc.Oracle(net, kn)
    X = np.full(net.nsp, 1e-99)
    X[net.species_index("PROT ")], X[net.species_index("HE  4")], X[ic12] = 0.7, 0.28, 0.02
    rfac = np.asarray(net.rfac)
    for T9, rho in ((0.015, 100.0), (0.03, 50.0), (0.2, 1e3), (2.0, 1e5)):
        v = ref.evaluate_all_rates(T9, rho, 0.85, X)[0]
        for slot, r in slots.items():
            want = max(orc.vital_reference(slot, T9, rho, 0.7) * rfac[r], 1e-99)
            assert abs(v[r] - want) <= 1e-14 * want, (slot, T9, v[r], want)


def test_hburning_zone_on_reference_vital_network(orc, abi, sn, wl):
    """An H-burning zone integrates with the reference's pp and CNO formulas: BD succeeds, the mass
    stays 1 and hydrogen burns."""
    net = sn.build_network(300, vital="reference")
    zb, _ = wl.hburn_zone(net)
    ref = orc.Oracle(net, abi.default_knobs())
    zb.dtwant[:] = 1e15
    X, _, ierr, _, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    assert (ierr == 0).all()
    assert abs(X.sum() - 1.0) < 1e-10
    ip = net.species_index("PROT ")
    assert X[0, ip] < zb.X[0, ip]
