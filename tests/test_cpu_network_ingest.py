"""Network ingest from the reference's isotope databases, on the CPU.

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
