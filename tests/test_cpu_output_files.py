"""ppn's per-cycle output files (printonecycle, frames/ppn/source/ppn.F90:431-539) written by the
library's host writers, on the CPU.

Where the reference tree is mounted, its own output files pin the format byte for byte: each
iso_massf file of the examples' master results that carries the current header is parsed and written
again from the parsed values, and must come out identical. The one flux file in the tree
(examples/ppn_Hburn_simple/Notebook) was written before the time-scale column was clamped to at least
1e99 (ppn.F90:509); its other columns must come out identical, and the time scale as the clamp prints
it. Without the tree, a file written for a synthetic network must read back in the reference's
fixed columns.
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

REF = os.environ.get("NUPPN_REFERENCE", "/root/reference")
HEADER = "H NUM     Z    A ISOM  ABUNDANCE_MF  ISOTP"


def _lib(solver_mod):
    return solver_mod.load_library()


def _iso_files():
    files = sorted(glob.glob(os.path.join(REF, "examples", "*", "master_results", "**", "iso_massf*.DAT"),
                             recursive=True))
    return [f for f in files if open(f).readline().rstrip("\n") == HEADER]


def _parse_iso(path):
    lines = open(path).read().splitlines()
    t = lines[1].split()
    head = {"model": int(t[2]), "dzeit": float(t[4]), "agej": float(t[6])}
    t = lines[2].split()
    head.update(t9=float(t[3]), rho=float(t[6]))
    head.update(densn=float(lines[3].split()[2]), densp=float(lines[4].split()[2]),
                densa=float(lines[5].split()[2]), energy=float(lines[6].split()[2]))
    rows = []
    for ln in lines[7:]:  # '(I5,2x,2(1X,F4.0),2x,I2,2x,ES12.5,2x,A5)'
        rows.append((int(ln[0:5]), float(ln[8:12]), float(ln[13:17]), int(ln[19:21]), float(ln[23:35]), ln[37:42]))
    return head, rows


@pytest.mark.skipif(not _iso_files(), reason="reference tree not mounted")
def test_iso_massf_byte_for_byte_against_the_reference(solver_mod, tmp_path):
    L = _lib(solver_mod)
    files = _iso_files()
    assert len(files) >= 10
    for path in files:
        head, rows = _parse_iso(path)
        nsp = max(r[0] for r in rows)
        z, a, x = np.zeros(nsp), np.zeros(nsp), np.zeros(nsp)
        iso = np.ones(nsp, np.int32)
        cons = np.zeros(nsp, np.uint8)
        names = bytearray(b" " * (5 * nsp))
        for i, zz, aa, st, xx, nm in rows:
            z[i - 1], a[i - 1], iso[i - 1], x[i - 1], cons[i - 1] = zz, aa, st, xx, 1
            names[5 * (i - 1):5 * i] = nm.encode().ljust(5)
        nb = C.create_string_buffer(bytes(names), len(names))
        out = tmp_path / "iso.DAT"
        st = L.nuppn_write_iso_massf(str(out).encode(), head["model"], head["dzeit"], head["agej"], head["t9"],
                                     head["rho"], head["densn"], head["densp"], head["densa"], head["energy"], nsp,
                                     z.ctypes.data, a.ctypes.data, iso.ctypes.data, x.ctypes.data,
                                     C.cast(nb, C.c_void_p), cons.ctypes.data)
        assert st == 0
        assert out.read_bytes() == open(path, "rb").read(), path


FLUX = os.path.join(REF, "examples", "ppn_Hburn_simple", "Notebook", "flux_00031.DAT")


@pytest.mark.skipif(not os.path.exists(FLUX), reason="reference tree not mounted")
def test_flux_file_columns_against_the_reference(solver_mod, tmp_path):
    L = _lib(solver_mod)
    lines = open(FLUX).read().splitlines()
    rows = [ln.split() for ln in lines[1:]]
    pairs = sorted({(int(r[c]), int(r[c + 1])) for r in rows for c in (1, 3, 5, 7)})
    sp = {p: i for i, p in enumerate(pairs)}
    z = np.array([p[0] for p in pairs], float)
    a = np.array([p[1] for p in pairs], float)
    n = len(rows)
    k = np.zeros((n, 8), np.int32)
    for i, r in enumerate(rows):
        for s, c in zip((0, 2, 4, 6), (1, 3, 5, 7)):
            k[i, s] = sp[(int(r[c]), int(r[c + 1]))]
    flux = np.array([float(r[9]) for r in rows])
    energy = np.array([float(r[10]) for r in rows])
    ts = np.array([float(r[11]) for r in rows])
    out = tmp_path / "flux.DAT"
    st = L.nuppn_write_flux(str(out).encode(), n, k.ctypes.data, z.ctypes.data, a.ctypes.data, flux.ctypes.data,
                            energy.ctypes.data, ts.ctypes.data)
    assert st == 0
    got = out.read_text().splitlines()
    assert got[0] == lines[0] and len(got) == len(lines)
    for g, ln, t in zip(got[1:], lines[1:], ts):
        assert g[:93] == ln[:93]  # index, Z and A of k1, k3, k5, k7, flux and energy
        assert g[93:] == "        " + ("%.5E" % max(1e99, t)).rjust(12)


def test_iso_massf_of_a_network_reads_back(solver_mod, wl, tmp_path):
    """Without the reference tree: the file written for the 300-species network reads back in the
    reference's fixed columns, with its number densities computed as printonecycle computes them."""
    net = wl.network(300)
    rng = np.random.default_rng(3)
    X = 10.0 ** rng.uniform(-110, 0, net.nsp)
    X /= X.sum()
    out = tmp_path / "iso_massf00042.DAT"
    solver_mod.write_iso_massf(out, net, X, 42, 1.5e7, 3.25e3, 0.195, 2.5e3, total_energy_flux=1.25e6)
    head, rows = _parse_iso(out)
    assert open(out).readline().rstrip("\n") == HEADER
    assert head["model"] == 42 and head["dzeit"] == 1.5e7 and head["agej"] == 3.25e3
    assert head["t9"] == 0.195 and head["rho"] == 2.5e3 and head["energy"] == 1.25e6
    na = solver_mod.AVOGADRO
    for key, name, f in (("densn", "NEUT ", 1.0), ("densp", "PROT ", 1.0), ("densa", "HE  4", 0.25)):
        want = X[net.species_index(name)] * f * 2.5e3 * na
        assert abs(head[key] - want) <= 5e-6 * want
    cons = np.nonzero(np.asarray(net.considerisotope))[0]
    assert [r[0] for r in rows] == (cons + 1).tolist()
    for i, zz, aa, st, xx, nm in rows:
        s = i - 1
        assert (zz, aa, st) == (net.znetw[s], net.anetw[s], 1) and nm == net.zis[s][:5].ljust(5)
        assert abs(xx - max(X[s], 1e-99)) <= 5e-6 * max(X[s], 1e-99)
