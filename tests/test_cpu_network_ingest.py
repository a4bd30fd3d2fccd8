"""Network ingest from the reference's isotope databases and networksetup.txt, on the CPU.

read_isotopedatabase (physics/source/nuc_data.F90:50-95) skips three header lines and reads Z, A, the
element symbol, a reference mass number and a T/F flag per line; networkI (ppn_physics.F90:40-130)
keeps the entries flagged T, in file order, as the network's isotopes after the VITAL species. The
library's reader (nuppn_isotopedatabase_read, host only) is checked on small files written here and,
where the reference tree is mounted, on its two databases against a plain Python parse; the species
tables that network construction uses (data/isotope_databases.npz) must equal the reader's output.
"""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("NUPPN_REFERENCE", "/root/reference")
DB = os.path.join(REF, "physics", "run_template")


def _reader(solver_mod):
    L = solver_mod.load_library()
    L.nuppn_isotopedatabase_read.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p]
    L.nuppn_isotopedatabase_read.restype = C.c_int32

    def read(path, n):
        z, a = np.zeros(n, np.int32), np.zeros(n, np.int32)
        flag = np.zeros(n, np.uint8)
        el = C.create_string_buffer(3 * max(n, 1))
        st = L.nuppn_isotopedatabase_read(str(path).encode(), n, z.ctypes.data, a.ctypes.data, flag.ctypes.data, el)
        names = [el.raw[3 * i:3 * i + 3].rstrip(b"\0").decode() for i in range(n)]
        return st, z, a, flag, names
    return read


def _python_parse(path, n):
    rows = []
    with open(path) as f:
        lines = f.read().splitlines()[3:]
    for line in lines[:n]:
        z, a, el, amin, fl = line.split()
        rows.append((int(z), int(a), el, fl.upper().startswith("T")))
    return rows


def test_reader_on_small_files(solver_mod, tmp_path):
    read = _reader(solver_mod)
    p = tmp_path / "isotopedatabase.txt"
    p.write_text("# header\n# header\n# header\n  0  1  nn  1  T\n  1  1   H  1  T \n 26 56 Fe\t56\tF\n")
    st, z, a, flag, el = read(p, 3)
    assert st == 0
    assert z.tolist() == [0, 1, 26] and a.tolist() == [1, 1, 56] and flag.tolist() == [1, 1, 0]
    assert el == ["nn", "H", "Fe"]
    assert read(p, 4)[0] == -5  # NUPPN_ERR_LIMIT: fewer entries than asked for (the reference stops)
    bad = tmp_path / "bad.txt"
    bad.write_text("h\nh\nh\n  1  1  H  1  X\n")
    assert read(bad, 1)[0] == -1  # NUPPN_ERR_ARG: a flag that is not T or F
    assert read(tmp_path / "missing.txt", 1)[0] == -1


@pytest.mark.skipif(not os.path.isdir(DB), reason="reference tree not mounted")
@pytest.mark.parametrize("name,n", [("isotopedatabase", 1107), ("isotopedatabase_all", 5234)])
def test_reader_on_reference_databases(solver_mod, name, n):
    read = _reader(solver_mod)
    st, z, a, flag, el = read(os.path.join(DB, name + ".txt"), n)
    assert st == 0
    rows = _python_parse(os.path.join(DB, name + ".txt"), n)
    assert [(r[0], r[1], r[2], r[3]) for r in rows] == list(zip(z.tolist(), a.tolist(), el, flag.astype(bool).tolist()))
    t = np.load(os.path.join(ROOT, "nuppn_modular2-ininet3_b200", "data", "isotope_databases.npz"))
    assert np.array_equal(t[name + "_z"], z) and np.array_equal(t[name + "_a"], a)
    assert np.array_equal(t[name + "_flag"], flag) and list(t[name + "_elem"]) == el


def test_database_networks_keep_the_reference_order(sn):
    """Species of a database network: the VITAL block, then the T-flagged database entries in file
    order (those already in the VITAL block keep their VITAL slot)."""
    t = np.load(os.path.join(ROOT, "nuppn_modular2-ininet3_b200", "data", "isotope_databases.npz"))
    for name, nnn in (("isotopedatabase", 201), ("isotopedatabase_all", 2500)):
        net = sn.build_network(nnn, database=name)
        keep = [(int(z), int(a)) for z, a, f in zip(t[name + "_z"][:nnn], t[name + "_a"][:nnn],
                                                   t[name + "_flag"][:nnn]) if f]
        za = [(int(z), int(a)) for z, a in zip(net.znetw, net.anetw)]
        nv = len(sn._VITAL_SPECIES)
        vital = set(za[:nv])
        assert za[nv:] == [p for p in keep if p not in vital]
        assert set(keep) <= set(za)


def _cols(line, spec):
    """Fields of a fixed-column line: spec = [(first column, width), ...], 1-based."""
    return [line[c - 1:c - 1 + w] for c, w in spec]


def test_networksetup_round_trip_and_columns(solver_mod, wl, tmp_path):
    """write_networksetup / read_networksetup (networksetup.F90:55-260) for the 300-species network:
    the lines sit in the columns of the reference's read formats, and reading the file back gives the
    species, switches, A, Z, k1..k8, reaction types, rate factors, labels and header."""
    net = wl.network(300)
    v = np.geomspace(1e-99, 1e12, net.nre)
    p = tmp_path / "networksetup.txt"
    solver_mod.networksetup_write(p, net, 0.02, 100.0, v=v)
    lines = p.read_text().splitlines()
    assert lines[0] == "*" * 72 and lines[1][:25] == "        TABLE OF ISOTOPES"
    assert float(lines[1][25:36]) == 0.02 and float(lines[1][36:47]) == 100.0  # '(a25,2(e11.3))'
    assert int(lines[4][7:12]) == net.nsp  # '(7x,I5,16x,I5)'
    sp = _cols(lines[5 + 4], [(8, 5), (16, 5), (22, 5), (29, 4), (36, 4), (43, 1)])  # fmtspecies, species 5
    assert int(sp[0]) == 5 and sp[1] == net.zis[4] and sp[2].strip() == "T"
    assert float(sp[3]) == net.anetw[4] and float(sp[4]) == net.znetw[4] and sp[5] == "1"
    r0 = 5 + net.nsp + 4
    assert int(lines[r0][7:12]) == net.nre
    l = int(np.nonzero(net.considerreaction)[0][-1])  # a network reaction: fmtreactionread columns
    f = _cols(lines[r0 + 1 + l], [(3, 5), (9, 1), (11, 2), (15, 5), (24, 2), (28, 5), (38, 2), (42, 5), (51, 2),
                                 (55, 5), (63, 9), (88, 2), (92, 10)])
    k = net.k[l]
    assert int(f[0]) == l + 1 and f[1] == "T"
    assert (int(f[2]), f[3], int(f[4]), f[5]) == (k[1], net.zis[k[0]], k[3], net.zis[k[2]])
    assert (int(f[6]), f[7], int(f[8]), f[9]) == (k[7], net.zis[k[6]], k[5], net.zis[k[4]])
    assert abs(float(f[10]) - v[l]) <= 5e-4 * v[l] and int(f[11]) == net.ilabb[l] and float(f[12]) == net.rfac[l]
    d = solver_mod.networksetup_read(p)
    assert (d["t9"], d["rho"]) == (0.02, 100.0) and d["zis"] == [z[:5].ljust(5) for z in net.zis]
    assert np.array_equal(d["k"], net.k) and np.array_equal(d["considerreaction"], net.considerreaction)
    assert np.array_equal(d["considerisotope"], net.considerisotope)
    assert np.array_equal(d["anetw"], net.anetw) and np.array_equal(d["znetw"], net.znetw)
    assert np.array_equal(d["ilabb"], net.ilabb) and np.array_equal(d["rfac"], net.rfac)
    assert np.allclose(d["v"], v, rtol=5e-4, atol=0)


def test_networksetup_switched_off_species_drop_their_reactions(solver_mod, wl, tmp_path):
    """A species marked F in the file switches off every reaction it takes part in
    (networksetup.F90:226-240); a three-digit exponent written without its E reads back."""
    net = wl.network(300)
    p = tmp_path / "networksetup.txt"
    solver_mod.networksetup_write(p, net)
    i = net.species_index("FE 56")
    lines = p.read_text().splitlines()
    row = lines[5 + i]
    lines[5 + i] = row[:21] + "    F" + row[26:]
    r0 = 5 + net.nsp + 4
    row = lines[r0 + 1]
    lines[r0 + 1] = row[:62] + "1.500-100" + row[71:]  # ES9.3 of 1.5e-100
    p.write_text("\n".join(lines) + "\n")
    d = solver_mod.networksetup_read(p)
    assert d["considerisotope"][i] == 0
    uses = (net.k[:, [0, 2, 4, 6]] == i).any(axis=1)
    assert uses.sum() > 0 and (d["considerreaction"][uses] == 0).all()
    assert np.array_equal(d["considerreaction"][~uses], net.considerreaction[~uses])
    assert d["v"][0] == 1.5e-100
