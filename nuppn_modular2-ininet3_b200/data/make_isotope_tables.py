"""Regenerate isotope_databases.npz from the reference's isotope database files.

The reference selects its network isotopes from ``physics/run_template/isotopedatabase.txt`` (1107
entries) or, for larger networks, ``isotopedatabase_all.txt`` (5234 entries), read by
read_isotopedatabase (``physics/source/nuc_data.F90:50-95``). This script reads both files with the
library's own reader (``nuppn_isotopedatabase_read``, host only) and stores Z, A, the T/F flag and the
element symbol of every entry, so that network construction needs no access to the reference tree.

    NUPPN_REFERENCE=/path/to/reference python make_isotope_tables.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {"isotopedatabase": 1107, "isotopedatabase_all": 5234}


def read(L, path, n):
    z, a = np.zeros(n, np.int32), np.zeros(n, np.int32)
    flag = np.zeros(n, np.uint8)
    elem = C.create_string_buffer(3 * n)
    st = L.nuppn_isotopedatabase_read(path.encode(), n, z.ctypes.data, a.ctypes.data, flag.ctypes.data, elem)
    if st != 0:
        raise RuntimeError(f"{path}: {L.nuppn_last_error().decode()}")
    el = np.array([elem.raw[3 * i:3 * i + 3].rstrip(b"\0").decode() for i in range(n)])
    return z, a, flag, el


def main():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import importlib
    solver = importlib.import_module("nuppn_modular2-ininet3_b200.solver")
    L = solver.load_library()
    L.nuppn_isotopedatabase_read.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p]
    ref = os.environ.get("NUPPN_REFERENCE", "/root/reference")
    out = {}
    for name, n in FILES.items():
        z, a, flag, el = read(L, os.path.join(ref, "physics", "run_template", name + ".txt"), n)
        out.update({f"{name}_z": z, f"{name}_a": a, f"{name}_flag": flag, f"{name}_elem": el})
    np.savez_compressed(os.path.join(HERE, "isotope_databases.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
