"""Seeded synthetic reaction networks in NuPPN's slot layout.

The reference builds its network at start-up from the REACLIB library, NETGEN/FFN/KADoNiS tables and
``isotopedatabase.txt`` (``physics/source/ppn_physics.F90:624-1021`` rnetw2007, ``:40-414`` networkI).
The REACLIB coefficient files are not available, so this module produces networks of the same shape
from a fixed seed: the same slot layout and index order, the same reaction types, physically-shaped
but synthetic rate data. Every array it returns is what a frame would hand to ``nuppn_net_create``
after running its own network set-up.

Index order (0-based here; the reference is 1-based):

* species ``0 .. nvcp-1`` are the light "VITAL" species (``ppn_physics.input`` block, read by
  ``vital.F90:read_physics_input_data``), including the gamma slot ``OOOOO`` with
  ``considerisotope = False``;
* then the network isotopes in Z-then-A order (``isotopedatabase.txt`` order, first ``nnn`` entries);
* reactions ``0 .. nrcp-1`` are the VITAL slots (triple-alpha sits at slot 43 in the reference's
  1-based numbering, which the screening special case of ``evaluate_rates.F90:86-93`` keys on);
* then, for every network isotope in order and every reaction type 1..16 whose product is in the
  network, one reaction (``ppn_physics.F90:708-774``), with the identical-particle merges of
  ``:785-797``; then alpha decays (``:800-822``);
* a network reaction that duplicates a considered VITAL reaction is switched off (``:878-887``).

Rate sources per reaction slot (``src``): VITAL analytic templates, REACLIB (seven-coefficient
contributions summed per rate, ``reaclib.F90:431-582``), NETGEN-style beta tables
(``netgen.F90:179-310``), FFN-style 2-D weak tables (``fuller.F90:92-122``), KADoNiS-style (n,g)
tables with Akima interpolation (``kadonis.F90:150-187``) and constant alpha-decay rates.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# reaction types, reaction_info.F90:8-34
I_NG, I_GN, I_NP, I_NA, I_PG, I_GP, I_PN, I_PA, I_AG, I_GA, I_AN, I_AP = range(1, 13)
I_BM, I_EC, I_BN, I_BP, I_BA = 13, 14, 15, 16, 17
RLABELS = {1: "(n,g)", 2: "(g,n)", 3: "(n,p)", 4: "(n,a)", 5: "(p,g)", 6: "(g,p)", 7: "(p,n)",
           8: "(p,a)", 9: "(a,g)", 10: "(g,a)", 11: "(a,n)", 12: "(a,p)", 13: "(-,g)",
           14: "(+,g)", 15: "(b,n)", 16: "(b,p)", 17: "(b,a)"}

# rate sources (must match include/nuppn.h NUPPN_SRC_*)
SRC_NONE, SRC_VITAL, SRC_REACLIB, SRC_NETGEN, SRC_FULLER, SRC_KADONIS, SRC_CONST = range(7)

# physical constants, utils/source/constants.F90
EV2ERG = 1.602177e-12
MEV2ERG = EV2ERG * 1.0e6
CLIGHT = 2.99792458e10
AMU = 1.6605402e-24
ME_G = 9.10938356e-28
MP_MEV = 938.27231
MN_MEV = 939.56563

# REACLIB partition-function temperature grid (24 points, the grid of the winvn tables)
PART_T9 = np.array([0.1, 0.15, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.0, 1.5, 2.0, 2.5, 3.0,
                    3.5, 4.0, 4.5, 5.0, 6.0, 7.0, 8.0, 9.0, 10.0])

ELEMENTS = ["nn", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si",
            "P", "S", "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu",
            "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc",
            "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La",
            "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu",
            "Hf", "Ta", "W", "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po"]


def zis_name(z: int, a: int) -> str:
    """Five-character species name in the reference's style (``'FE 56'``, ``'PB206'``)."""
    if z == 0 and a == 1:
        return "NEUT "
    if z == 1 and a == 1:
        return "PROT "
    el = ELEMENTS[z].upper()
    s = f"{el:<2}{a:>3}"
    return s[:5]


_BTABLE: dict = {}


def binding_energy(z: int, a: int) -> float:
    """Binding energy (MeV): liquid-drop value, raised where needed so that every nucleus is bound
    against n, p and alpha emission by at least 0.5-1 MeV (Be8 excepted). Memoised; the recursion
    only looks at lighter nuclei, so the table is the same whatever the call order."""
    key = (z, a)
    if key not in _BTABLE:
        b = _semf(z, a)
        if a > 4 and (z, a) != (4, 8):
            if a - 1 > z or (z == 0 and a > 1):
                b = max(b, binding_energy(z, a - 1) + 1.0)
            if z >= 1 and a - 1 >= z - 1 and a > 1:
                b = max(b, binding_energy(z - 1, a - 1) + 1.0)
            if z >= 2 and a >= 8:
                b = max(b, binding_energy(z - 2, a - 4) + 28.296 + 0.5)
        _BTABLE[key] = b
    return _BTABLE[key]


def _semf(z: int, a: int) -> float:
    """Semi-empirical (Weizsaecker) binding energy in MeV; textbook coefficients."""
    if a <= 1:
        return 0.0
    n = a - z
    av, as_, ac, aa, ap = 15.75, 17.8, 0.711, 23.7, 11.18
    b = av * a - as_ * a ** (2.0 / 3.0) - ac * z * (z - 1) / a ** (1.0 / 3.0) - aa * (n - z) ** 2 / a
    if z % 2 == 0 and n % 2 == 0:
        b += ap / math.sqrt(a)
    elif z % 2 == 1 and n % 2 == 1:
        b -= ap / math.sqrt(a)
    # light nuclei are far off the liquid-drop line; keep them sensible and bound
    light = {(1, 2): 2.2246, (2, 3): 7.718, (2, 4): 28.296, (4, 8): 56.50, (6, 12): 92.16,
             (8, 16): 127.62, (3, 7): 39.24, (4, 7): 37.60, (5, 8): 37.74}
    if (z, a) in light:
        return light[(z, a)]
    return max(b, 1.0 * a)


def mass_excess(z: int, a: int) -> float:
    """Mass excess (MeV) consistent with ``binding_energy``: the inverse of nse_swj.F90:190-194."""
    n = a - z
    # atomic mass energy = Z mp + N mn - B + Z me; mass excess = that - A * amu c^2
    amu_mev = AMU * CLIGHT ** 2 / MEV2ERG
    me_mev = ME_G * CLIGHT ** 2 / MEV2ERG
    return z * MP_MEV + n * MN_MEV - binding_energy(z, a) + z * me_mev - a * amu_mev


def n_center(z: int) -> float:
    return z + 0.0059 * z * z


@dataclasses.dataclass
class Network:
    """All arrays of one network description (0-based indices, reference slot order)."""
    name: str
    zis: list
    anetw: np.ndarray
    znetw: np.ndarray
    considerisotope: np.ndarray
    exmass: np.ndarray
    gspin: np.ndarray
    spec_part: np.ndarray
    k: np.ndarray              # [nre, 8] int32: k1..k8 (species indices 0-based; counts)
    ilabb: np.ndarray
    considerreaction: np.ndarray
    rfac: np.ndarray
    src: np.ndarray
    src_idx: np.ndarray
    irev: np.ndarray
    nvcp: int
    nrcp: int
    igamma: int
    # REACLIB
    rl_a: np.ndarray           # [nc, 7]
    rl_rate: np.ndarray        # [nc] -> rate index
    rl_chapter: np.ndarray     # [nr]
    rl_vflag: np.ndarray       # [nr] uint8 ('v' reverse flag)
    rl_ecflag: np.ndarray      # [nr] uint8 ('  ec' label)
    rl_nireac: np.ndarray      # [nr] reaction type used for density factors
    rl_part: np.ndarray        # [nr, 6] partition-function rows, -1 -> empty species (g = 1)
    part_t9: np.ndarray
    part_val: np.ndarray       # [npart, 24]
    # VITAL templates: terms of c * T9^p * exp(d*T9^(-1/3) + f/T9 + g*T9)
    vt_first: np.ndarray       # [nv+1]
    vt_terms: np.ndarray       # [nt, 5]
    vt_dpow: np.ndarray        # [nv] density power
    vt_xfac: np.ndarray        # [nv] species index for a 0.5*(1+X) composition factor, or -1
    # NETGEN beta table
    ng_t8: np.ndarray          # [kgrid]
    ng_flag: np.ndarray        # [nreac]
    ng_ndata: np.ndarray       # [nreac]
    ng_ane: np.ndarray         # [nreac, ndmax]
    ng_l10v: np.ndarray        # [kgrid, nreac, ndmax]
    # FFN table
    ff_t9coo: np.ndarray       # log10 T9 grid
    ff_rhocoo: np.ndarray      # log10 rho*Ye grid
    ff_l10v: np.ndarray        # [nv, nt, nr]
    # KADoNiS
    kd_e: np.ndarray           # [ne] keV
    kd_rate: np.ndarray        # [nkad, ne]
    # constant rates
    const_rate: np.ndarray
    # per VITAL rate: 0 = the template above, k = the reference's own formula for VITAL slot k
    vt_form: np.ndarray | None = None

    @property
    def nsp(self):
        return len(self.anetw)

    @property
    def nre(self):
        return len(self.ilabb)

    def species_index(self, name: str) -> int:
        return self.zis.index(name)


# ---------------------------------------------------------------------------------------------
def _isotope_list(nnn: int):
    """Z-then-A sorted isotope band around the valley of stability; first nnn entries."""
    out = [(0, 1), (1, 1), (1, 2), (2, 3), (2, 4)]
    for z in range(3, 85):
        c = n_center(z)
        hw = 2.0 + z / 9.0
        nlo, nhi = int(math.ceil(c - hw)), int(math.floor(c + hw))
        if z < 6:
            nlo, nhi = max(nlo, z - 1), min(nhi, z + 2)
        for n in range(max(nlo, 1), nhi + 1):
            out.append((z, z + n))
    return out[:nnn]


_VITAL_SPECIES = [(0, 1), (1, 1), (1, 2), (2, 3), (2, 4), (4, 7), (5, 8), (3, 7), (6, 12),
                  (6, 13), (7, 13), (7, 14), (7, 15), (8, 16), (8, 17), (8, 18), (9, 19),
                  (10, 20), (10, 21), (10, 22), (11, 23), (12, 24), (12, 25), (12, 26),
                  (4, 8), (-1, 0)]          # (-1, 0) marks the gamma slot OOOOO


def database_isotopes(database: str, nnn: int):
    """(Z, A) of the network isotopes that networkI (``ppn_physics.F90:40-130``) takes from the first
    ``nnn`` lines of the reference's isotope database ``database`` (``"isotopedatabase"``, 1107
    entries, or ``"isotopedatabase_all"``, 5234): the entries flagged T, in file order. (networkI also
    drops isotopes whose NETGEN beta or EC rate at the set-up T9/rho beats ln 2 / tbetamin; that
    needs the real NETGEN tables and is not applied here.) The tables come from
    data/isotope_databases.npz, written by data/make_isotope_tables.py with the library's reader."""
    import os
    t = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "isotope_databases.npz"))
    z, a, f = t[database + "_z"], t[database + "_a"], t[database + "_flag"]
    if nnn > z.size:
        raise ValueError(f"{database} has {z.size} entries, fewer than nnn = {nnn}")
    return [(int(z[i]), int(a[i])) for i in range(nnn) if f[i]]


# VITAL slots whose rate the library evaluates by the reference's own formula
# (physics/source/vital.F90:339-569): the pp chains and the first CNO reactions
VITAL_FORMULA_SLOTS = (1, 2, 3, 4, 5, 6, 7, 8, 9, 14, 15, 16, 17, 73)


def build_network(nnn: int = 1107, seed: int = 20240611, name: str | None = None,
                  database: str | None = None, vital: str = "template") -> Network:
    """Build a synthetic network with ``nnn`` isotope-database entries (the reference's NNN). With
    ``database`` the isotopes are the reference database's (database_isotopes), else a synthetic band
    around the valley of stability in the same Z-then-A order. ``vital="reference"`` puts the
    reactions of VITAL_FORMULA_SLOTS in their slots with the reference's formulas as their rates (the
    network loop then leaves those reactions to VITAL); the default keeps analytic templates."""
    if vital not in ("template", "reference"):
        raise ValueError("vital must be 'template' or 'reference'")
    vital_ref = vital == "reference"  # the name vital is rebound to a helper below
    rng = np.random.default_rng(seed)
    isos = database_isotopes(database, nnn) if database else _isotope_list(nnn)

    # ---- species -------------------------------------------------------------------------
    zis, A, Z = [], [], []
    for (z, a) in _VITAL_SPECIES:
        if z < 0:
            zis.append("OOOOO"); A.append(0.0); Z.append(0.0)
        else:
            zis.append(zis_name(z, a)); A.append(float(a)); Z.append(float(z))
    nvcp = len(zis)
    pos = {(int(Z[i]), int(A[i])): i for i in range(nvcp) if zis[i] != "OOOOO"}
    for (z, a) in isos:
        if (z, a) in pos:
            continue
        pos[(z, a)] = len(zis)
        zis.append(zis_name(z, a)); A.append(float(a)); Z.append(float(z))
    nsp = len(zis)
    A = np.array(A); Z = np.array(Z)
    igamma = zis.index("OOOOO")
    considerisotope = np.ones(nsp, np.uint8)
    considerisotope[igamma] = 0
    ineut, iprot, ih2, ihe3, ihe4 = (pos[(0, 1)], pos[(1, 1)], pos[(1, 2)], pos[(2, 3)], pos[(2, 4)])
    ibe8 = pos[(4, 8)]

    exmass = np.zeros(nsp)
    gspin = np.ones(nsp)
    spec_part = np.full(nsp, -1, np.int32)
    part_rows = []
    for i in range(nsp):
        if i == igamma:
            continue
        z, a = int(Z[i]), int(A[i])
        exmass[i] = mass_excess(z, a)
        n = a - z
        if a % 2 == 1:
            gspin[i] = 2.0 * (0.5 + rng.integers(0, 4)) + 1.0
        elif z % 2 == 1:
            gspin[i] = 2.0 * rng.integers(0, 5) + 1.0
        else:
            gspin[i] = 1.0
        # partition function: 1 at low T, rising with T for heavier/odd nuclei
        amp = 0.02 * (a / 50.0) * (1.0 + (z % 2) + (n % 2)) * rng.uniform(0.5, 1.5)
        part_rows.append(1.0 + amp * PART_T9 ** 2 * np.exp(PART_T9 / 10.0))
        spec_part[i] = len(part_rows) - 1
    part_val = np.array(part_rows)

    # ---- reactions -----------------------------------------------------------------------
    K, ILABB, CONS, SRC, SIDX = [], [], [], [], []
    vt_first, vt_terms, vt_dpow, vt_xfac = [0], [], [], []
    nrcp = 117

    def add_reaction(k, ilab, src, sidx, cons=1):
        K.append(list(k)); ILABB.append(ilab); CONS.append(cons); SRC.append(src); SIDX.append(sidx)

    def vital(k, ilab, terms, dpow, xfac=-1):
        vt_terms.extend(terms); vt_first.append(len(vt_terms)); vt_dpow.append(dpow)
        vt_xfac.append(xfac)
        add_reaction(k, ilab, SRC_VITAL, len(vt_dpow) - 1)

    g = igamma
    ic12, io16 = pos[(6, 12)], pos[(8, 16)]
    vital_defs = {
        1: ((iprot, 2, g, 0, g, 0, ih2, 1), I_PG, [(4.0e-15, -2 / 3, -3.38, 0.0, 0.0)], 1.0, -1),
        2: ((ih2, 1, iprot, 1, g, 0, ihe3, 1), I_PG, [(2.2e3, -2 / 3, -3.72, 0.0, 0.0)], 1.0, -1),
        3: ((ihe3, 2, g, 0, iprot, 2, ihe4, 1), 99, [(6.0e10, -2 / 3, -12.28, 0.0, 0.0)], 1.0, -1),
        4: ((ihe4, 1, ihe3, 1, g, 0, pos[(4, 7)], 1), 99, [(5.6e6, -2 / 3, -12.83, 0.0, 0.0)], 1.0, -1),
        5: ((pos[(4, 7)], 1, g, 0, g, 0, pos[(3, 7)], 1), I_EC,
            [(1.3e-10, -0.5, 0.0, 0.0, 0.0)], 1.0, iprot),
        6: ((pos[(3, 7)], 1, iprot, 1, g, 0, ihe4, 2), I_PG, [(1.1e10, -2 / 3, -8.47, 0.0, 0.0)], 1.0, -1),
        43: ((ihe4, 3, g, 0, g, 0, ic12, 1), 99,
             [(2.8e-8, -3.0, 0.0, -4.4027, 0.0), (1.35e-7, -1.5, 0.0, -24.811, 0.0)], 2.0, -1),
        44: ((ic12, 1, ihe4, 1, g, 0, io16, 1), I_AG,
             [(1.04e8, -2.0, -32.12, 0.0, 0.0), (1.76e8, -2.0, -32.12, 0.0, 0.0),
              (1.25e3, -1.5, 0.0, -27.499, 0.0)], 1.0, -1),
        45: ((io16, 1, ihe4, 1, g, 0, pos[(10, 20)], 1), I_AG,
             [(9.37e9, -2 / 3, -39.757, 0.0, 0.0), (62.1, -1.5, 0.0, -10.297, 0.0)], 1.0, -1),
        46: ((ic12, 2, g, 0, ihe4, 1, pos[(10, 20)], 1), 99,
             [(4.27e26, -1.5, -84.165, 0.0, 0.0)], 1.0, -1),
        47: ((ibe8, 1, g, 0, g, 0, ihe4, 2), 99, [(1.0e16, 0.0, 0.0, 0.0, 0.0)], 0.0, -1),
    }
    vt_form = []
    covered = set()  # (target Z, A, reaction type) that a formula slot carries
    if vital_ref:
        ib7, ib8, ili7 = pos[(4, 7)], pos[(5, 8)], pos[(3, 7)]
        in13, ic13, in14 = pos[(7, 13)], pos[(6, 13)], pos[(7, 14)]
        ref_defs = {
            7: ((ib7, 1, iprot, 1, g, 0, ib8, 1), I_PG, (4, 7, I_PG)),
            8: ((ib8, 1, g, 0, g, 0, ihe4, 2), 99, (5, 8, I_BP)),
            9: ((ib8, 1, g, 0, iprot, 1, ib7, 1), I_GP, (5, 8, I_GP)),
            14: ((ic12, 1, iprot, 1, g, 0, in13, 1), I_PG, (6, 12, I_PG)),
            15: ((ic13, 1, iprot, 1, g, 0, in14, 1), I_PG, (6, 13, I_PG)),
            73: ((in13, 1, g, 0, iprot, 1, ic12, 1), I_GP, (7, 13, I_GP)),
        }
        if (8, 14) in pos:
            ref_defs[16] = ((in13, 1, iprot, 1, g, 0, pos[(8, 14)], 1), I_PG, (7, 13, I_PG))
        if (8, 15) in pos:
            ref_defs[17] = ((in14, 1, iprot, 1, g, 0, pos[(8, 15)], 1), I_PG, (7, 14, I_PG))
        covered.add((3, 7, I_PA))  # Li7(p,a)He4 is slot 6
        for slot, (k, ilab, cov) in ref_defs.items():
            vital_defs[slot] = (k, ilab, [], 0.0, -1)
            covered.add(cov)
    for slot in range(1, nrcp + 1):
        if slot in vital_defs:
            k, ilab, terms, dpow, xfac = vital_defs[slot]
            if vital_ref and slot in VITAL_FORMULA_SLOTS:
                terms, dpow = [], 0.0
                xfac = iprot if slot == 5 else -1  # XII(IPROT) of FABE7
            vital(k, ilab, terms, dpow, xfac)
            vt_form.append(slot if vital_ref and slot in VITAL_FORMULA_SLOTS else 0)
        else:
            add_reaction((g, 0, g, 0, g, 0, g, 0), 99, SRC_NONE, -1, cons=0)

    # network reactions: one per (isotope, type) with product in network
    prod_shift = {I_NG: (0, 1), I_GN: (0, -1), I_NP: (-1, 0), I_NA: (-2, -3), I_PG: (1, 1),
                  I_GP: (-1, -1), I_PN: (1, 0), I_PA: (-1, -3), I_AG: (2, 4), I_GA: (-2, -4),
                  I_AN: (2, 3), I_AP: (1, 3), I_BM: (1, 0), I_EC: (-1, 0), I_BN: (1, -1),
                  I_BP: (-2, -1)}
    light_in = {I_NG: (ineut, 1, g, 0), I_GN: (g, 0, ineut, 1), I_NP: (ineut, 1, iprot, 1),
                I_NA: (ineut, 1, ihe4, 1), I_PG: (iprot, 1, g, 0), I_GP: (g, 0, iprot, 1),
                I_PN: (iprot, 1, ineut, 1), I_PA: (iprot, 1, ihe4, 1), I_AG: (ihe4, 1, g, 0),
                I_GA: (g, 0, ihe4, 1), I_AN: (ihe4, 1, ineut, 1), I_AP: (ihe4, 1, iprot, 1),
                I_BM: (g, 0, g, 0), I_EC: (g, 0, g, 0), I_BN: (g, 0, ineut, 1),
                I_BP: (g, 0, iprot, 1)}

    def stable(z, a):
        n = a - z
        return abs(n - n_center(z)) <= 1.0 + z / 40.0 or a <= 4

    # rate data accumulators
    rl_a, rl_rate, rl_chapter, rl_vflag, rl_ecflag, rl_nireac, rl_part = [], [], [], [], [], [], []
    ng_rows, ff_rows, kd_rows, const_rate = [], [], [], []

    amu_mev = 931.494
    kdE = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 8.0, 10.0, 15.0, 20.0, 25.0, 30.0, 40.0, 50.0, 60.0,
                    80.0, 100.0, 150.0, 200.0, 300.0, 400.0, 500.0, 600.0, 800.0, 1000.0])
    ng_t8 = np.logspace(-2.0, 2.0, 30)

    def part_of(idx):
        return int(spec_part[idx]) if idx != igamma and idx >= 0 else -1

    def reaclib_rate(z, a, rtype, target_idx, prod_idx, lin, lout):
        """Synthetic REACLIB contributions for one reaction; returns the rate index."""
        zp = {I_NG: 0, I_NP: 0, I_NA: 0, I_PG: 1, I_PN: 1, I_PA: 1, I_AG: 2, I_AN: 2, I_AP: 2}
        ap = {I_NG: 1, I_NP: 1, I_NA: 1, I_PG: 1, I_PN: 1, I_PA: 1, I_AG: 4, I_AN: 4, I_AP: 4}
        zo, ao = int(Z[prod_idx]), int(A[prod_idx])
        # Q = B(products) - B(reactants)
        q = binding_energy(zo, ao) - binding_energy(z, a)
        if lout != g:
            q += binding_energy(int(Z[lout]), int(A[lout]))
        if lin != g:
            q -= binding_energy(int(Z[lin]), int(A[lin]))
        rev = rtype in (I_GN, I_GP, I_GA)
        contribs = []
        if rtype in zp:
            z2, a2 = zp[rtype], ap[rtype]
            mu = a * a2 / (a + a2)
            if z2 == 0:                    # neutron induced: roughly 1/v, flat N_A<sv>
                lo = math.log(10.0 ** rng.uniform(4.3, 7.3) * (1.0 if a > 20 else 1e-2))
                nmag = a - z
                if nmag in (50, 82, 126):
                    lo -= math.log(100.0)
                c = [lo, 0.0, 0.0, 0.0, rng.normal(0, 0.05), 0.0, rng.normal(0, 0.1)]
                if q < 0:
                    c[1] = 11.6045 * q
                contribs.append(c)
            else:                          # charged particle: Gamow peak
                tau = 4.2487 * (z * z * z2 * z2 * mu) ** (1.0 / 3.0)
                c = [rng.uniform(18.0, 26.0) + math.log(max(mu, 0.5)), 0.0, -tau,
                     rng.normal(0, 0.3), rng.normal(0, 0.05), 0.0, -2.0 / 3.0]
                if q < 0:
                    c[1] = 11.6045 * q
                contribs.append(c)
                if rng.uniform() < 0.4:    # a resonance contribution
                    er = rng.uniform(0.2, 1.5) + max(-q, 0.0)
                    contribs.append([rng.uniform(2.0, 10.0), -11.6045 * er, 0.0, 0.0, 0.0, 0.0, -1.5])
            chapter = 4 if lout == g else 5
            pr = [part_of(target_idx), part_of(lin), part_of(prod_idx), part_of(lout), -1, -1]
            if lout == g:
                pr = [part_of(target_idx), part_of(lin), part_of(prod_idx), -1, -1, -1]
            vflag = 1 if (q < 0 and lout != g) else 0
        else:                              # photodisintegration (the reverse of a capture)
            sep = -q
            aa = float(A[lout])
            mu = (a - aa) * aa / a
            base = math.log(10.0 ** rng.uniform(4.3, 7.3)) if lout == ineut else \
                rng.uniform(18.0, 26.0) + math.log(max(mu, 0.5))
            zz = 0 if lout == ineut else int(Z[lout])
            tau = 4.2487 * (max(z - zz, 0) ** 2 * zz * zz * mu) ** (1.0 / 3.0) if zz else 0.0
            c = [base + 23.0 + 1.5 * math.log(mu), -11.6045 * sep, -tau, 0.0, 0.0, 0.0,
                 1.5 + (-2.0 / 3.0 if zz else 0.0)]
            contribs.append(c)
            chapter = 2
            pr = [part_of(target_idx), part_of(lout), part_of(prod_idx), -1, -1, -1]
            vflag = 1
        r = len(rl_chapter)
        for c in contribs:
            rl_a.append(c); rl_rate.append(r)
        rl_chapter.append(chapter); rl_vflag.append(vflag); rl_ecflag.append(0)
        rl_nireac.append(rtype); rl_part.append(pr)
        return r

    def weak_rate(z, a, rtype):
        """Half-life from the distance to stability; returns (src, idx) or None."""
        n = a - z
        d = n - n_center(z)
        if rtype == I_BM and d <= 1.0 + z / 40.0:
            return None
        if rtype == I_EC and d >= -(1.0 + z / 40.0):
            return None
        dist = abs(d) - (1.0 + z / 40.0)
        l10lam = -15.0 + 3.5 * dist + rng.normal(0, 0.7)     # log10 decay rate (1/s)
        l10lam = min(l10lam, 0.5)
        if rtype == I_EC and 21 <= z <= 32:                  # FFN-style 2-D table
            t = np.linspace(-2.0, 1.0, 13)[:, None]
            rr = np.linspace(1.0, 11.0, 11)[None, :]
            tab = l10lam + 0.3 * np.tanh(t + 1.0) + 0.08 * np.maximum(rr - 6.0, 0.0)
            ff_rows.append(tab)
            return SRC_FULLER, len(ff_rows) - 1
        lt = np.log10(ng_t8)
        base = l10lam + 0.15 * np.tanh(lt) + rng.normal(0, 0.05, size=lt.shape) * 0.2
        if rtype == I_EC and rng.uniform() < 0.3:             # electron-density-tabulated
            ane = np.logspace(20.0, 30.0, 6)
            tab = base[:, None] + np.linspace(0.0, 0.6, 6)[None, :]
            ng_rows.append((float(ane[0]), 6, ane, tab))
        else:
            ng_rows.append((-11.0, 1, np.ones(1), base[:, None]))
        return SRC_NETGEN, len(ng_rows) - 1

    reaction_of = {}
    for (z, a) in isos:
        kk = pos[(z, a)]
        if a <= 4:          # n, p, d, 3He, 4He react through the VITAL block only
            continue
        for rtype in range(1, 17):
            if (z, a, rtype) in covered:
                continue
            dz, da = prod_shift[rtype]
            prod = (z + dz, a + da)
            if prod not in pos or prod[1] <= 0 or prod == (z, a):
                continue
            pidx = pos[prod]
            if pidx in (ineut, iprot):
                continue
            lin, nin, lout, nout = light_in[rtype]
            k = [kk, 1, lin, nin, lout, nout, pidx, 1]
            src, sidx = SRC_NONE, -1
            if rtype in (I_BM, I_EC):
                w = weak_rate(z, a, rtype)
                if w is None:
                    continue
                src, sidx = w
            elif rtype in (I_BN, I_BP):
                if z < 30 or stable(z, a) or rng.uniform() > 0.15:
                    continue
                ng_rows.append((-11.0, 1, np.ones(1),
                                (-9.0 + rng.normal(0, 1.0) + 0 * ng_t8)[:, None]))
                src, sidx = SRC_NETGEN, len(ng_rows) - 1
            else:
                if rtype == I_NG and z >= 26 and stable(z, a) and rng.uniform() < 0.7:
                    # KADoNiS-style MACS table: rate(E) rising slowly with kT
                    r30 = 10.0 ** rng.uniform(6.0, 8.3) * (0.01 if (a - z) in (50, 82, 126) else 1.0)
                    kd_rows.append(r30 * (kdE / 30.0) ** rng.uniform(0.05, 0.25))
                    src, sidx = SRC_KADONIS, len(kd_rows) - 1
                else:
                    src, sidx = SRC_REACLIB, reaclib_rate(z, a, rtype, kk, pidx, lin, lout)
            # identical-particle merges, ppn_physics.F90:785-797
            if k[0] == k[2]:
                k[1] += k[3]; k[3] = 0; k[2] = g
            if k[4] == k[6]:
                k[7] += k[5]; k[5] = 0; k[4] = g
            add_reaction(k, rtype, src, sidx)
            reaction_of[(kk, rtype)] = len(K) - 1

    # alpha decays of the heaviest isotopes (constant rates), ppn_physics.F90:800-822
    for (z, a) in isos:
        if z >= 84 and (z - 2, a - 4) in pos:
            const_rate.append(10.0 ** rng.uniform(-9.0, -6.5))
            add_reaction((pos[(z, a)], 1, g, 0, ihe4, 1, pos[(z - 2, a - 4)], 1), I_BA,
                         SRC_CONST, len(const_rate) - 1)

    K = np.array(K, np.int32)
    ILABB = np.array(ILABB, np.int32)
    CONS = np.array(CONS, np.uint8)
    nre = len(K)

    # switch off network reactions duplicating considered VITAL ones (ppn_physics.F90:878-887)
    for i in range(nrcp):
        if not CONS[i]:
            continue
        for j in range(nrcp, nre):
            if (zis[K[i, 0]] == zis[K[j, 0]] and K[i, 1] == K[j, 1] and K[i, 2] == K[j, 2]
                    and K[i, 3] == K[j, 3] and K[i, 7] == K[j, 7] and K[i, 5] == K[j, 5]
                    and zis[K[i, 4]] == zis[K[j, 4]]):
                CONS[j] = 0

    # reverse pairs (restating reverse.F90:26-104 on the synthetic REACLIB flags)
    irev = np.full(nre, -1, np.int32)
    SRC = np.array(SRC, np.int32)
    SIDX = np.array(SIDX, np.int32)
    is_rev = np.zeros(nre, bool)
    for i in range(nre):
        if CONS[i] and SRC[i] == SRC_REACLIB and ILABB[i] <= 16:
            is_rev[i] = bool(rl_vflag[SIDX[i]])
    keymap = {}
    for j in range(nre):
        if CONS[j]:
            keymap.setdefault(tuple(int(x) for x in (K[j, 6], K[j, 7], K[j, 4], K[j, 5],
                                                     K[j, 2], K[j, 3], K[j, 0], K[j, 1])), j)
    for i in range(nre):
        if not CONS[i] or ILABB[i] in (I_EC, I_BM, I_BN, I_BP) or ILABB[i] > 22:
            continue
        if K[i, 7] > 1 or is_rev[i]:
            continue
        j = keymap.get(tuple(int(x) for x in K[i]))
        if j is not None and is_rev[j]:
            irev[i] = j

    def pad(rows, width):
        return np.array(rows if rows else np.zeros((0, width)))

    nd = max([r[1] for r in ng_rows] + [1])
    ng_flag = np.array([r[0] for r in ng_rows])
    ng_ndata = np.array([r[1] for r in ng_rows], np.int32)
    ng_ane = np.ones((len(ng_rows), nd))
    ng_l10v = np.zeros((len(ng_t8), len(ng_rows), nd))
    for i, (fl, ndat, ane, tab) in enumerate(ng_rows):
        ng_ane[i, :ndat] = ane
        ng_l10v[:, i, :ndat] = tab

    return Network(
        name=name or (f"{database}{nnn}" if database else f"synth{nnn}"), zis=zis, anetw=A, znetw=Z, considerisotope=considerisotope,
        exmass=exmass, gspin=gspin, spec_part=spec_part, k=K, ilabb=ILABB,
        considerreaction=CONS, rfac=np.ones(nre), src=SRC, src_idx=SIDX, irev=irev,
        nvcp=nvcp, nrcp=nrcp, igamma=igamma,
        rl_a=pad(rl_a, 7), rl_rate=np.array(rl_rate, np.int32),
        rl_chapter=np.array(rl_chapter, np.int32), rl_vflag=np.array(rl_vflag, np.uint8),
        rl_ecflag=np.array(rl_ecflag, np.uint8), rl_nireac=np.array(rl_nireac, np.int32),
        rl_part=np.array(rl_part, np.int32).reshape(-1, 6), part_t9=PART_T9.copy(),
        part_val=part_val,
        vt_first=np.array(vt_first, np.int32), vt_terms=pad(vt_terms, 5),
        vt_dpow=np.array(vt_dpow), vt_xfac=np.array(vt_xfac, np.int32),
        ng_t8=ng_t8, ng_flag=ng_flag, ng_ndata=ng_ndata, ng_ane=ng_ane, ng_l10v=ng_l10v,
        ff_t9coo=np.linspace(-2.0, 1.0, 13), ff_rhocoo=np.linspace(1.0, 11.0, 11),
        ff_l10v=np.array(ff_rows).reshape(-1, 13, 11),
        kd_e=kdE, kd_rate=pad(kd_rows, len(kdE)), const_rate=np.array(const_rate),
        vt_form=np.array(vt_form, np.int32),
    )
