"""bench.py's host-side pieces that the reported line depends on, on the CPU: the DRAM traffic per
zone read from the committed ncu summary, and the clock sampler's summary, which must use only the
nvidia-smi rows that arrived inside the timed region."""
import importlib.util
import os
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_per_zone_from_profile():
    b = _bench()
    v = b.measured_traffic_per_zone()
    with open(os.path.join(ROOT, "profiles", "k_integrate_heshell1107_256_memory.md")) as f:
        line = next(l for l in f if l.startswith("traffic_bytes_per_zone"))
    assert v == int(line.split("=")[1]) and v > 0


def test_clock_summary_uses_timed_rows_only():
    b = _bench()
    c = b.ClockSampler(0)
    now = time.time()
    row = lambda mhz, thermal="Not Active": [str(mhz), "1965", "500", "Not Active", thermal, "Not Active", "Not Active"]
    c.rows = [(now - 10.0, row(800, "Active")),  # before the timed region: ignored
              (now + 1.0, row(1965)), (now + 1.1, row(1950)), (now + 1.2, row(1965)),
              (now + 10.0, row(700, "Active"))]  # after it: ignored
    c.t0, c.t1 = now, now + 5.0
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == []
    c.t0, c.t1 = now + 20.0, now + 30.0
    assert c.summary()["reasons"] == ["unsampled"]


def test_roofline_model_is_below_measured_traffic():
    """The roofline's algorithmic bytes are the compulsory HBM traffic of the integration (abundances in
    and out, scalars, the network arena once): they cannot exceed what ncu measured the kernel moving,
    so at any launch time the model's fraction of HBM peak stays below the measured DRAM fraction and
    below 1."""
    b = _bench()
    nz, nsp, arena = 1024, 1109, 8 << 20
    tpz = b.measured_traffic_per_zone()
    assert b.model_bytes(nz, nsp, arena) <= tpz * nz
    for per_launch_s in (1e-4, 1e-3, 0.034):
        r = b.roofline(nz, nsp, arena, per_launch_s, 6542.0, "measured", 1965.0)
        assert r["bound"] == "hbm" and r["unit"] == "GB/s"
        assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
        assert r["frac"] <= r["dram_frac"] and r["frac"] <= 1.0
