"""tppnp's binary trajectory input (traj_data.F90:73-168) read by the library's host reader, on the
CPU: a file written here in the same layout reads back exactly, malformed files are refused, and,
where the reference tree is mounted, its run template's tp.lsb reads as four whole tracers that end
exactly at the end of the file."""
import os
import struct

import numpy as np
import pytest

REF = os.environ.get("NUPPN_REFERENCE", "/root/reference")
TP = os.path.join(REF, "frames", "tppnp", "run_template", "input_data", "tp.lsb")


def _write(path, tracers):
    nts = [len(t["time"]) for t in tracers]
    with open(path, "wb") as f:
        f.write(struct.pack("<3i", len(tracers), min(nts), max(nts)))
        for t in tracers:
            nt, ni = len(t["time"]), len(t["x"])
            f.write(struct.pack("<2i", t["pnum"], nt))
            f.write(struct.pack("<d", t["mass"]) + struct.pack("<3d", *t["posini"]) + struct.pack("<3d", *t["posfin"]))
            for k in ("time", "temp", "dens"):
                f.write(np.asarray(t[k], "<f8").tobytes())
            f.write(struct.pack("<2i", t["pnum"], ni))
            f.write(np.asarray(t["a"], "<i4").tobytes() + np.asarray(t["z"], "<i4").tobytes())
            f.write("".join(n.ljust(5)[:5] for n in t["zis"]).encode())
            f.write(np.asarray(t["x"], "<f8").tobytes())


def test_written_file_reads_back(solver_mod, tmp_path):
    rng = np.random.default_rng(5)
    tracers = []
    for p, nt, ni in ((7, 5, 3), (9, 11, 4)):
        tracers.append({"pnum": p, "mass": rng.uniform(), "posini": rng.uniform(size=3), "posfin": rng.uniform(size=3),
                        "time": np.sort(rng.uniform(0, 10, nt)), "temp": rng.uniform(1e8, 9e9, nt),
                        "dens": rng.uniform(1, 1e8, nt), "a": rng.integers(1, 60, ni), "z": rng.integers(0, 28, ni),
                        "zis": ["NEUT", "PROT", "HE  4", "C  12"][:ni], "x": rng.uniform(size=ni)})
    path = tmp_path / "tp.lsb"
    _write(path, tracers)
    got, hdr = solver_mod.tppnp_read(path)
    assert hdr == {"num_tracers": 2, "nsteps_min": 5, "nsteps_max": 11}
    for g, t in zip(got, tracers):
        assert g["pnum"] == t["pnum"] and g["mass"] == t["mass"]
        assert np.array_equal(g["posini"], t["posini"]) and np.array_equal(g["posfin"], t["posfin"])
        assert np.array_equal(g["time"], t["time"]) and np.array_equal(g["rho"], t["dens"])
        assert np.array_equal(g["t9"], np.asarray(t["temp"]) / 1e9)
        assert np.array_equal(g["a"], t["a"]) and np.array_equal(g["z"], t["z"]) and np.array_equal(g["x"], t["x"])
        assert g["zis"] == [n.ljust(5)[:5] for n in t["zis"]]
    short = tmp_path / "short.lsb"
    short.write_bytes(path.read_bytes()[:-9])  # the last tracer's abundances cut short
    with pytest.raises(solver_mod.NuppnError):
        solver_mod.tppnp_read(short)
    with pytest.raises(solver_mod.NuppnError):
        solver_mod.tppnp_read(tmp_path / "missing.lsb")


@pytest.mark.skipif(not os.path.exists(TP), reason="reference tree not mounted")
def test_reference_run_template_trajectories(solver_mod, wl):
    got, hdr = solver_mod.tppnp_read(TP)
    assert hdr["num_tracers"] == len(got) == 4
    nts = [len(t["time"]) for t in got]
    assert min(nts) == hdr["nsteps_min"] and max(nts) == hdr["nsteps_max"]
    size = 12 + sum(8 + 56 + 24 * len(t["time"]) + 8 + 21 * len(t["x"]) for t in got)
    assert size == os.path.getsize(TP)  # the tracers end exactly at the end of the file
    for t in got:
        assert np.all(np.diff(t["time"]) > 0) and np.all(t["t9"] > 0) and np.all(t["rho"] > 0)
        assert abs(t["x"].sum() - 1.0) < 1e-6 and t["zis"][:2] == ["NEUT ", "PROT "]
    net = wl.network(1107)
    X, lost = solver_mod.tppnp_initial_abundances(net, got[0])
    assert X.shape == (net.nsp,) and X.min() >= 1e-99
    assert X[net.species_index("HE  4")] == got[0]["x"][got[0]["zis"].index("HE  4")]
    assert 0.0 <= lost < 1.0
