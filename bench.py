"""Benchmark: zone-timesteps/s of batched Bader-Deuflhard integration on the ~1100-species network.

Workload (one GPU): 1024 independent He-burning shell zones on the 1109-slot synthetic network
(NNN = 1107), T9 ~ U[0.10, 0.30], rho log-U[1e2, 1e4], X(He4)=0.97, X(C12)=0.01, X(Ne22)=0.02,
Fe56=1e-3 (renormalised) x lognormal(0.05) per species, one integrate_network call of 1e10 s per zone
with adaptive Bader-Deuflhard steps, FP64. A "step" is one call over the whole batch, restarted from
the same initial state. The metric counts accepted sub-steps (zone-timesteps) per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--nz Z]

--impl reference times the reference's own algorithm on the host cores (the CPU restatement of
NuPPN's FP64 path, calling the reference's SuperLU) on a bounded sample of the same workload.
For N > 1 (torchrun) the zones are sharded across ranks, balanced by peak temperature (snake order);
there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "nuppn_modular2-ininet3_b200"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region. The sampler is started before
    the warm-up (nvidia-smi takes a few hundred ms to start) and samples every 50 ms; only the rows
    that arrive between mark() and the end of the `with` block are summarised."""

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None
        self.t0 = None
        self.t1 = None

    def mark(self):
        self.t0 = time.time()

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append((time.time(), parts))

    def __exit__(self, *a):
        self.t1 = time.time()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        t0 = self.t0 if self.t0 is not None else 0.0
        t1 = self.t1 if self.t1 is not None else time.time()
        rows = [r for t, r in self.rows if t0 <= t <= t1]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def profile_value(name, key):
    """A `key = value` line of a committed ncu summary under profiles/ (None if absent)."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith(key + " ="):
                return float(line.split("=")[1])
    except OSError:
        pass
    return None


HESHELL_PROFILE = "k_integrate_heshell1107_256_memory.md"


def measured_traffic_per_zone():
    """DRAM bytes per zone of k_integrate from the committed ncu summary (None if absent)."""
    v = profile_value(HESHELL_PROFILE, "traffic_bytes_per_zone")
    return int(v) if v is not None else None


def model_bytes(nz, nsp, arena_bytes):
    """Bytes the integration must move between HBM and the SMs per launch, at minimum: each zone's
    abundances in and out (2 * nsp doubles), its six input scalars (T9 and rho at both ends, Ye,
    dtwant), its outputs (Ye, ierr, 8 counters, the Bader-Deuflhard state) and the zone-shared network
    arena once. Everything else a zone touches (rates, Jacobian, LU, extrapolation tableau) is
    per-zone working state that an ideal kernel keeps on chip."""
    per_zone = 2 * nsp * 8 + 6 * 8 + 8 + 4 + 8 * 4 + 2 * 4
    return nz * per_zone + arena_bytes


def roofline(nz, nsp, arena_bytes, per_launch_s, peak_gbs, peak_kind, sm_mhz, n_sm=148):
    """The `roofline` object of the bench line. bound "hbm": achieved = model bytes per launch /
    launch time, against the measured HBM copy bandwidth. traffic = ncu DRAM bytes per zone (a 256-zone
    capture) times the zones. The kernel is bound by per-zone dependency chains, not by either
    peak; fp64_pipe_frac = FP64-pipe warp instructions (ncu, per zone, times the zones) / (SMs x the
    pipe's peak per SM cycle x SM clock x launch time) shows how much of the FP64 pipe it uses."""
    model = model_bytes(nz, nsp, arena_bytes)
    achieved = model / per_launch_s / 1e9
    tpz = measured_traffic_per_zone()
    traffic = tpz * nz if tpz else None
    out = {"bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s", "frac": achieved / peak_gbs,
           "traffic": traffic, "peak_source": peak_kind, "kernel": "k_integrate",
           "algorithmic_bytes_per_launch": model,
           "model": "per zone 2*nsp*8 (X in, out) + 100 B of scalars; network arena once per launch",
           "dram_achieved_gbs": (traffic / per_launch_s / 1e9) if traffic else None,
           "dram_frac": (traffic / per_launch_s / 1e9 / peak_gbs) if traffic else None,
           "traffic_source": "ncu dram__bytes_read+write per zone at 256 zones, x zones"}
    fp64 = profile_value(HESHELL_PROFILE, "fp64_inst_per_zone")
    fp64_peak = profile_value(HESHELL_PROFILE, "fp64_inst_peak_per_sm_cycle")
    if fp64 and fp64_peak and sm_mhz:
        out["fp64_pipe_frac"] = fp64 * nz / (n_sm * fp64_peak * sm_mhz * 1e6 * per_launch_s)
        out["fp64_source"] = "ncu sm__inst_executed_pipe_fp64 per zone at 256 zones, x zones"
    return out


def heshell_config(nz_total, nsp):
    """The workload both arms print in `config` (the same dict, so the arms are the same config)."""
    return {"workload": "heshell-1107 BD 1e10 s", "zones": int(nz_total), "network_species": int(nsp),
            "integrator": "bader-deuflhard", "arithmetic": "fp64"}


def parity_sample(zb, n):
    """A fixed sample of n zones for the checker: the 8 hottest (the costliest and least well-conditioned
    zones) and the rest evenly spaced over the batch, in batch order."""
    n = min(n, zb.nz)
    hot = np.argsort(-np.maximum(zb.t9_0, zb.t9_1), kind="stable")[:min(8, n)]
    rest = np.setdiff1d(np.arange(zb.nz), hot)
    pick = rest[np.linspace(0, rest.size - 1, max(n - hot.size, 0)).astype(int)] if n > hot.size else rest[:0]
    return np.sort(np.concatenate([hot, pick]))


# The reference arm integrates the whole batch every step when it has at most this many zones (about
# 4 s a step on 16 host cores for the 1024-zone batch), else this many zones of it.
REF_MAX_ZONES = 1024


def run_reference(args, rank, world):
    """CPU reference arm: the checker (restated FP64 path + reference SuperLU), all host threads, on the
    same batch as the GPU arm (the whole batch up to REF_MAX_ZONES zones per step)."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    wl = importlib.import_module(PKG + ".workloads")
    abi = importlib.import_module(PKG + ".abi")
    net = wl.network(1107)
    nz_total = args.nz * world
    zb = wl.heshell_batch(nz_total, net=net, seed=2)
    cores = os.cpu_count() or 1
    sample = min(nz_total, REF_MAX_ZONES)
    idx = np.arange(nz_total) if sample == nz_total else parity_sample(zb, sample)
    # hottest first: the checker's threads take zones from a shared counter, so the costliest start first
    idx = idx[np.argsort(-zb.t9_0[idx], kind="stable")]
    sub = zb.take(idx)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    times, steps = [], []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        X, ye, ierr, st, _ = ref.integrate_network(sub.X, sub.t9_0, sub.t9_1, sub.rho_0, sub.rho_1, sub.ye,
                                                   sub.dtwant, nthreads=cores)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
            steps.append(sum(s.nsucc for s in st))
    v = sum(steps) / sum(times)
    what = "all" if sample == nz_total else f"{sample} (the 8 hottest and evenly spaced others) of"
    line = {"impl": "reference", "metric": "zone-timesteps/s", "value": v, "unit": "zone-timesteps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": heshell_config(nz_total, net.nsp),
            "cpu_baseline": {"value": v, "unit": "zone-timesteps/s", "cores": cores, "kind": "port",
                             "sample": f"{what} {nz_total} zones per step, restated FP64 path + "
                                       f"reference SuperLU 5.0, one zone per thread"},
            "e2e": {"value": v, "unit": "zone-timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_traj(args, rank, world, local):
    """Explosive-burning trajectories: args.nz per GPU, 201 points from 0 to 10 s (T9_0 in [2, 5],
    rho_0 in [1e6, 1e8], tau in [0.1, 1] s, Si28/Fe56 seed), tppnp's trajectory loop for all of them
    in one launch. A step integrates every trajectory over the whole grid."""
    wl = importlib.import_module(PKG + ".workloads")
    abi = importlib.import_module(PKG + ".abi")
    net = wl.network(1107)
    tr_all = wl.trajectory_batch(args.nz * world, net=net, npts=201)
    grids = tr_all.grids()
    sel = importlib.import_module(PKG + ".sharding").snake_shards(grids[1].max(axis=1), world)[rank]
    tt, t9, rho = (g[sel] for g in grids)
    X0, ye0 = tr_all.X0[sel], tr_all.ye0[sel]
    cfg = {"workload": "tppnp-traj-1107 201 points to 10 s", "trajectories": args.nz * world,
           "trajectories_per_gpu": args.nz, "network_species": net.nsp, "integrator": "bader-deuflhard",
           "lu": "fp64", "launches_per_step": 2}
    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        cores = os.cpu_count() or 1
        n = min(args.nz, max(cores, 16))
        ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
        times, steps = [], []
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            _, _, _, _, st = ref.integrate_trajectories(X0[:n], tt[:n], t9[:n], rho[:n], nthreads=cores)
            dt = time.perf_counter() - t0
            if it >= args.warmup:
                times.append(dt)
                steps.append(sum(s.nsucc for s in st))
        v = sum(steps) / sum(times)
        print(json.dumps({"impl": "reference", "metric": "zone-timesteps/s", "value": v, "unit": "zone-timesteps/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": v, "unit": "zone-timesteps/s", "cores": cores, "kind": "port",
                                           "sample": f"{n} of {args.nz} trajectories per step"},
                          "e2e": {"value": v, "unit": "zone-timesteps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    solver = importlib.import_module(PKG + ".solver")
    S = solver.NetworkSolver(net, abi.default_knobs(integration_method=1), device=torch.cuda.current_device())
    nz = args.nz
    cu = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    X0d, ye0d, ttd, t9d, rhod = cu(X0), cu(ye0), cu(tt), cu(t9), cu(rho)
    X, ye = X0d.clone(), ye0d.clone()
    ierr, fail = (torch.zeros(nz, dtype=torch.int32, device="cuda") for _ in range(2))
    stats = torch.zeros((nz, 8), dtype=torch.int32, device="cuda")
    bd = torch.zeros(nz, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def one_step():
        X.copy_(X0d); ye.copy_(ye0d); bd.zero_()
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        S.integrate_trajectories_device(X, ttd, t9d, rhod, ye, ierr, fail, stats, bd, stream=stream)
        e1.record()
        return e0, e1

    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(args.warmup):
            one_step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = S.launches()
        clk.mark()
        ev = [one_step() for _ in range(args.steps)]
        torch.cuda.synchronize()
    st_np = stats.cpu().numpy()
    steps_done = int(st_np[:, 0].sum()) * args.steps
    t_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    gpu_launches = S.launches() - launches0
    t0 = time.perf_counter()
    _, _, _, _, st_h = S.integrate_trajectories(X0, tt, t9, rho)
    e2e_t, e2e_steps = time.perf_counter() - t0, sum(s.nsucc for s in st_h)
    sharding = importlib.import_module(PKG + ".sharding")
    t_ms, steps_done = sharding.reduce_time_and_steps(t_ms, steps_done, "cuda", dist if world > 1 else None)
    e2e_t, e2e_steps = sharding.reduce_time_and_steps(e2e_t, e2e_steps, "cuda", dist if world > 1 else None)
    if rank == 0:
        cfg.update({"accepted_steps_per_call": int(st_np[:, 0].sum()), "rejected_steps_per_call": int(st_np[:, 1].sum()),
                    "failed_trajectories": int((fail.cpu().numpy() >= 0).sum()),
                    "l2": "flushed: 256 MiB written before each timed call"})
        line = {"metric": "zone-timesteps/s", "value": steps_done / (t_ms * 1e-3), "unit": "zone-timesteps/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": cfg, "gpu_launches": int(gpu_launches),
                "e2e": {"value": e2e_steps / e2e_t, "unit": "zone-timesteps/s",
                        "h2d_bytes_per_step": int(X0.nbytes + 3 * tt.nbytes + 8 * nz),
                        "d2h_bytes_per_step": int(X0.nbytes + 8 * nz + 8 * nz + 32 * nz)},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_hburn(args, rank, world):
    """The ppn frame of one H-burning zone (300-species network, T9 = 0.020, rho = 100, X(H) = 0.70,
    X(He4) = 0.28, Z = 0.02 solar-scaled): 200 backward-Euler frame steps, dt log-spaced 1e3 .. 1e13 s,
    each one integrate_network call carrying X, Ye and bd_state. A step is the whole frame; value =
    accepted sub-steps / time. One zone is one CTA: this measures latency, not throughput."""
    if rank != 0:
        return
    wl = importlib.import_module(PKG + ".workloads")
    abi = importlib.import_module(PKG + ".abi")
    net = wl.network(300)
    zb, dts = wl.hburn_zone(net)
    kn = abi.default_knobs(integration_method=0)
    cfg = {"workload": "ppn hburn-300 BE frame: 200 steps, dt 1e3..1e13 s", "zones": 1, "network_species": net.nsp,
           "integrator": "backward-euler", "lu": "fp64", "launches_per_step": 2 * len(dts)}
    args_zone = (zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1)
    if args.impl == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        ref = orc.Oracle(net, kn)
        times, steps = [], []
        for it in range(args.warmup + args.steps):
            X, ye, n = zb.X.copy(), zb.ye.copy(), 0
            t0 = time.perf_counter()
            for dt in dts:
                X, ye, ierr, st, _ = ref.integrate_network(X, *args_zone, ye, dt)
                n += st[0].nsucc
            if it >= args.warmup:
                times.append(time.perf_counter() - t0)
                steps.append(n)
        v = sum(steps) / sum(times)
        print(json.dumps({"impl": "reference", "metric": "zone-timesteps/s", "value": v, "unit": "zone-timesteps/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": v, "unit": "zone-timesteps/s", "cores": 1, "kind": "port",
                                           "sample": "the whole frame (one zone: one core)"},
                          "e2e": {"value": v, "unit": "zone-timesteps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    solver = importlib.import_module(PKG + ".solver")
    S = solver.NetworkSolver(net, kn, device=torch.cuda.current_device())
    cu = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    X0d, ye0d = cu(zb.X), cu(zb.ye)
    zone_d = [cu(a) for a in args_zone]
    dts_d = cu(dts)
    X, ye = X0d.clone(), ye0d.clone()
    n = len(dts)
    ierr = torch.zeros(n, dtype=torch.int32, device="cuda")
    stats = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    bd = torch.zeros(1, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def one_step():
        X.copy_(X0d); ye.copy_(ye0d); bd.zero_()
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(n):
            S.integrate_device(X, *zone_d, ye, dts_d[i:i + 1], ierr[i:i + 1], stats[i], bd, stream=stream)
        e1.record()
        return e0, e1

    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(args.warmup):
            one_step()
        torch.cuda.synchronize()
        launches0 = S.launches()
        clk.mark()
        ev = [one_step() for _ in range(args.steps)]
        torch.cuda.synchronize()
    gpu_launches = S.launches() - launches0
    st_np = stats.cpu().numpy()
    steps_done = int(st_np[:, 0].sum()) * args.steps
    t_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    failed = int(np.count_nonzero(ierr.cpu().numpy()))
    # end to end: the same frame through nuppn_integrate with host buffers
    e2e_t, e2e_steps = 0.0, 0
    for it in range(1 + args.steps):
        Xh, yeh, m = zb.X.copy(), zb.ye.copy(), 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for dt in dts:
            Xh, yeh, ie, st, _ = S.integrate_network(Xh, *args_zone, yeh, dt)
            m += st[0].nsucc
        if it >= 1:
            e2e_t += time.perf_counter() - t0
            e2e_steps += m
    print(json.dumps({"metric": "zone-timesteps/s", "value": steps_done / (t_ms * 1e-3), "unit": "zone-timesteps/s",
                      "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": dict(cfg, frame_steps_failed=failed,
                                                          accepted_steps_per_frame=int(st_np[:, 0].sum()),
                                                          l2="flushed: 256 MiB written before each timed frame"),
                      "e2e": {"value": e2e_steps / e2e_t, "unit": "zone-timesteps/s",
                              "h2d_bytes_per_step": int(n * (zb.X.nbytes + 7 * 8)),
                              "d2h_bytes_per_step": int(n * (zb.X.nbytes + 8 + 4 + 32 + 4))},
                      "gpu_launches": int(gpu_launches), "clocks": clk.summary()}), flush=True)


def run_serve(args, rank, world):
    """Serving: a seeded Poisson stream (args.rate requests/s over args.serve_seconds) of one-zone and
    one-trajectory requests, 40 % He-shell zones (1109 species, BD over 1e10 s), 40 % H-burning zones
    on the 300-species network (T9 U[0.015, 0.08], rho log-U[1, 1e3], BD over 1e10 s), 20 % tppnp
    trajectories (1109 species, 21 points to 10 s), submitted as they arrive to two servers (one per
    network, 2/3 and 1/3 of the GPU's zone slots) and polled from this thread. The same stream is
    served by the plain form (one zone per CTA) and then by the batched form (one zone per warp),
    as --serve-shapes lists them. A stream cut at --serve-limit is reported as it stood then.
    value = accepted zone sub-steps of all requests / (last completion - first arrival); latency =
    completion - arrival, from the polling loop."""
    if rank != 0:
        return
    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "unavailable": "the serving workload has no reference counterpart "
                          "(the reference integrates one zone per call on the host)"}), flush=True)
        return
    import torch
    wl = importlib.import_module(PKG + ".workloads")
    abi = importlib.import_module(PKG + ".abi")
    solver = importlib.import_module(PKG + ".solver")
    n1107, n300 = wl.network(1107), wl.network(300)
    he = wl.heshell_batch(1024, net=n1107, seed=2)
    hb0, _ = wl.hburn_zone(n300)
    tr = wl.trajectory_batch(256, net=n1107, npts=21)
    tt, t9g, rhog = tr.grids()
    rng = np.random.default_rng(11)
    gaps = rng.exponential(1.0 / args.rate, size=int(args.rate * args.serve_seconds * 1.5) + 16)
    arrive = np.cumsum(gaps)
    arrive = arrive[arrive < args.serve_seconds]
    kinds = rng.choice(3, size=arrive.size, p=[0.4, 0.4, 0.2])
    pick = rng.integers(0, 1 << 30, size=arrive.size)
    hb_t9 = rng.uniform(0.015, 0.08, size=arrive.size)
    hb_rho = 10.0 ** rng.uniform(0.0, 3.0, size=arrive.size)
    dev = torch.cuda.current_device()

    def serve_stream(shape):
        kn = abi.default_knobs(integration_method=1, **shape)
        d1107 = solver.NetworkSolver(n1107, kn, device=dev)
        d300 = solver.NetworkSolver(n300, kn, device=dev)
        probe = solver.Server(d1107)  # every zone slot of this kernel shape, to split between the servers
        total = probe.info().slots
        probe.close()
        s1107 = solver.Server(d1107, slots=max(1, (2 * total) // 3))
        s300 = solver.Server(d300, slots=max(1, total - (2 * total) // 3))

        def submit(i):
            k = kinds[i]
            if k == 0:
                z = pick[i] % he.nz
                return s1107, s1107.submit(he.X[z], he.t9_0[z], he.t9_1[z], he.rho_0[z], he.rho_1[z], he.ye[z],
                                           he.dtwant[z])
            if k == 1:
                return s300, s300.submit(hb0.X[0], hb_t9[i], hb_t9[i], hb_rho[i], hb_rho[i], hb0.ye[0], 1.0e10)
            j = pick[i] % tr.nz
            return s1107, s1107.submit_trajectory(tr.X0[j], tt[j], t9g[j], rhog[j])

        for i in range(min(args.warmup, arrive.size) * 8):  # warm-up: a few requests of each kind, waited for
            srv, rid = submit(i % arrive.size)
            srv.wait(rid)
        lat = [[], [], []]
        steps = 0
        fails = [{}, {}, {}]  # per kind: ierr code -> count
        out = {}
        t0 = time.perf_counter()
        nxt = 0
        last_done = t0
        cut = False
        with ClockSampler(dev) as clk:
            clk.mark()
            while nxt < arrive.size or out:
                now = time.perf_counter() - t0
                if now > args.serve_limit:  # stop waiting: report what completed by then
                    cut = True
                    break
                while nxt < arrive.size and arrive[nxt] <= now:
                    out[nxt] = submit(nxt)
                    nxt += 1
                for i in list(out):
                    srv, rid = out[i]
                    r = srv.poll(rid)
                    if r is None:
                        continue
                    tdone = time.perf_counter()
                    last_done = tdone
                    lat[kinds[i]].append((tdone - t0 - arrive[i]) * 1e3)
                    steps += r[3].nsucc
                    if r[2] != 0:
                        fails[kinds[i]][str(r[2])] = fails[kinds[i]].get(str(r[2]), 0) + 1
                    del out[i]
                time.sleep(1e-4)
        elapsed = max(last_done - t0 - (arrive[0] if arrive.size else 0.0), 1e-9)
        info = (s1107.info(), s300.info())
        done_n = sum(len(v) for v in lat)
        allv = np.concatenate([np.array(v) for v in lat if v]) if done_n else np.zeros(1)
        pct = lambda v: {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99))} if len(v) else None
        res = {"value": steps / elapsed, "latency_ms": {"all": pct(allv), "heshell_zone": pct(lat[0]),
                                                        "hburn_zone": pct(lat[1]), "trajectory": pct(lat[2])},
               "requests_failed": {"heshell_zone": fails[0], "hburn_zone": fails[1], "trajectory": fails[2]},
               "drain_s": float(elapsed - args.serve_seconds),
               "requests": {"arrived": int(nxt), "completed": int(done_n), "unfinished_at_limit": int(len(out)),
                            "limit_s": float(args.serve_limit), "cut_at_limit": bool(cut)},
               "zone_slots": {"1107": info[0].slots, "300": info[1].slots},
               "in_flight_at_end": {"1107": int(info[0].in_flight), "300": int(info[1].in_flight)},
               "pending_at_end": {"1107": int(info[0].pending), "300": int(info[1].pending)},
               "loop_launches": int(info[0].launches + info[1].launches), "clocks": clk.summary()}
        print(json.dumps({"serve_stream": shape, **res}), file=sys.stderr, flush=True)  # before the servers close
        if cut:  # requests still on the GPU: leave the servers to the process's exit instead of waiting
            open_servers.extend([s1107, s300])
        else:
            s1107.close()
            s300.close()
        return res

    open_servers = []
    shapes = args.serve_shapes.split(",")
    plain = serve_stream({}) if "plain" in shapes else None
    batched = serve_stream({"threads_per_zone": 32}) if "batched" in shapes and not open_servers else None
    first = plain if plain is not None else batched
    form = "one zone per warp" if first is batched else "one zone per CTA"
    line = {"metric": "zone-timesteps/s", "value": first["value"], "unit": "zone-timesteps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "serve: Poisson stream, 40% heshell-1107 zones, 40% hburn-300 zones, "
                                   "20% tppnp-1107 trajectories (21 points)",
                       "rate_req_per_s": args.rate, "arrival_window_s": args.serve_seconds,
                       "requests": int(arrive.size), "form": form + ", device-resident loop"},
            "latency_ms": first["latency_ms"], "requests_failed": first["requests_failed"],
            "drain_s": first["drain_s"], "requests": first["requests"], "zone_slots": first["zone_slots"],
            "e2e": {"value": first["value"], "unit": "zone-timesteps/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
            "gpu_launches": first["loop_launches"], "clocks": first["clocks"]}
    if batched is not None and plain is not None:
        line["batched_form"] = {k: batched[k] for k in ("value", "latency_ms", "requests_failed", "drain_s",
                                                        "requests", "zone_slots")}
        line["batched_over_plain"] = batched["value"] / plain["value"] if plain["value"] else None
    print(json.dumps(line), flush=True)
    if open_servers:  # a stream was cut at its limit: its requests end with the process, not waited for
        os._exit(0)


def run_mixed(args, rank, world):
    """The uneven-size batch: 4096 zones (args.nz) of three networks in one launch
    (nuppn_integrate_multi), 40 % H-burning zones on the ~200-species network, 50 % He-shell zones on
    the ~1100-species network, 10 % hot zones on the ~2500-species network (workloads.mixed_batch),
    one integrate_network call of 1e10 s each. A step is one call over the batch from the same state.
    Beside the one-launch FP64 form (value) the line gives the same zones as three separate launches
    (one per network, back to back on one stream) and the one-launch form with the FP32 factor and
    FP64 refinement (lu_precision = 1)."""
    if rank != 0:
        return
    wl = importlib.import_module(PKG + ".workloads")
    abi = importlib.import_module(PKG + ".abi")
    nets, parts, net_of = wl.mixed_batch(args.nz)
    ldx = max(n.nsp for n in nets)
    nz = args.nz
    X0 = np.full((nz, ldx), 1e-99)
    cols = {f: np.zeros(nz) for f in ("t9_0", "t9_1", "rho_0", "rho_1", "ye", "dtwant")}
    z = 0
    for i, zb in parts:
        X0[z:z + zb.nz, :nets[i].nsp] = zb.X
        for f in cols:
            cols[f][z:z + zb.nz] = getattr(zb, f)
        z += zb.nz
    cfg = {"workload": "mixed networks: 40% hburn-200, 50% heshell-1107, 10% hot-2500, BD 1e10 s",
           "zones": nz, "network_species": [int(n.nsp) for n in nets], "integrator": "bader-deuflhard",
           "arithmetic": "fp64"}
    if args.impl == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        cores = os.cpu_count() or 1
        take = {0: 16, 1: 16, 2: 8}  # a bounded sample: the 2500-species zones take seconds each
        times, steps = [], []
        for it in range(args.warmup + args.steps):
            t, n = 0.0, 0
            for i, zb in parts:
                sub = zb.take(np.arange(min(take[i], zb.nz)))
                ref = orc.Oracle(nets[i], abi.default_knobs(integration_method=1))
                t0 = time.perf_counter()
                _, _, _, st, _ = ref.integrate_network(sub.X, sub.t9_0, sub.t9_1, sub.rho_0, sub.rho_1, sub.ye,
                                                       sub.dtwant, nthreads=cores)
                t += time.perf_counter() - t0
                n += sum(s.nsucc for s in st)
            if it >= args.warmup:
                times.append(t)
                steps.append(n)
        v = sum(steps) / sum(times)
        print(json.dumps({"impl": "reference", "metric": "zone-timesteps/s", "value": v, "unit": "zone-timesteps/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": v, "unit": "zone-timesteps/s", "cores": cores, "kind": "port",
                                           "sample": "16 + 16 + 8 zones of the three networks per step"},
                          "e2e": {"value": v, "unit": "zone-timesteps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    solver = importlib.import_module(PKG + ".solver")
    dev = torch.cuda.current_device()
    cu = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    X0d = cu(X0)
    d = {f: cu(v) for f, v in cols.items()}
    nof = cu(net_of, torch.int32)
    X = X0d.clone()
    ye = d["ye"].clone()
    ierr = torch.zeros(nz, dtype=torch.int32, device="cuda")
    stats = torch.zeros((nz, 8), dtype=torch.int32, device="cuda")
    bd = torch.zeros(nz, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    offs = np.concatenate([[0], np.cumsum([zb.nz for _, zb in parts])])

    def form(lu_precision, one_launch):
        sv = [solver.NetworkSolver(n, abi.default_knobs(integration_method=1, lu_precision=lu_precision), device=dev)
              for n in nets]

        def step():
            X.copy_(X0d); ye.copy_(d["ye"]); bd.zero_()
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if one_launch:
                solver.integrate_multi_device(sv, nof, X, d["t9_0"], d["t9_1"], d["rho_0"], d["rho_1"], ye,
                                              d["dtwant"], ierr, stats, bd, stream=stream)
            else:
                for i in range(3):
                    a, b = int(offs[i]), int(offs[i + 1])
                    sl = lambda t: t[a:b]
                    sv[i].integrate_device(X[a:b], *(sl(d[f]) for f in ("t9_0", "t9_1", "rho_0", "rho_1")),
                                           ye[a:b], d["dtwant"][a:b], ierr[a:b], stats[a:b], bd[a:b], stream=stream)
            e1.record()
            return e0, e1

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        launches0 = sum(s.launches() for s in sv)
        ev = [step() for _ in range(args.steps)]
        torch.cuda.synchronize()
        ms = float(sum(a.elapsed_time(b) for a, b in ev)) / args.steps
        st = stats.cpu().numpy()
        res = {"ms_per_call": ms, "value": float(st[:, 0].sum()) / (ms * 1e-3),
               "failed_zones": int((ierr.cpu().numpy() != 0).sum()),
               "gpu_launches": int(sum(s.launches() for s in sv) - launches0),
               "X": X.cpu().numpy(), "stats": st}
        for s in sv:
            s.close()
        return res

    with ClockSampler(dev) as clk:
        clk.mark()
        one = form(0, True)
        clocks = clk.summary()
    sep = form(0, False)
    mixp = form(1, True)
    rel_mixed = parity_rel(mixp["X"], one["X"])
    per_net = {}
    for i, n in enumerate(nets):
        rows = np.nonzero(net_of == i)[0]
        per_net[n.name] = {"zones": int(rows.size), "accepted_steps": int(one["stats"][rows, 0].sum()),
                           "max_active_species": int(one["stats"][rows, 7].max())}
    line = {"metric": "zone-timesteps/s", "value": one["value"], "unit": "zone-timesteps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": one["ms_per_call"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "run": {"l2": "flushed: 256 MiB written before each timed call", "per_network": per_net,
                    "failed_zones": one["failed_zones"]},
            "gpu_launches": one["gpu_launches"],
            "separate_launches": {k: sep[k] for k in ("ms_per_call", "value", "failed_zones")},
            "one_launch_over_separate": one["value"] / sep["value"],
            "mixed_precision": {k: mixp[k] for k in ("ms_per_call", "value", "failed_zones")},
            "mixed_over_fp64": mixp["value"] / one["value"],
            "mixed_max_rel_dev_vs_fp64": rel_mixed, "clocks": clocks}
    print(json.dumps(line), flush=True)


def parity_rel(X, Xr):
    """Largest relative difference over entries with Xr > 1e-12 (other entries: ignored)."""
    big = Xr > 1e-12
    return float((np.abs(X - Xr)[big] / Xr[big]).max(initial=0.0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nz", type=int, default=None, help="zones (trajectories) per GPU: 4096 for mixed, else 1024")
    ap.add_argument("--cpu-zones", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="heshell", choices=["heshell", "traj", "serve", "hburn", "mixed"],
                    help="heshell: 1024 He-shell zones (the headline); traj: tppnp-style trajectories; "
                         "serve: Poisson request stream through nuppn_serve_*; hburn: the ppn frame of one "
                         "H-burning zone (200 backward-Euler frame steps)")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: mean requests per second")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serve: arrival window (s)")
    ap.add_argument("--serve-limit", type=float, default=600.0,
                    help="serve: seconds after the first arrival at which the stream stops being waited for")
    ap.add_argument("--serve-shapes", default="plain,batched",
                    help="serve: kernel shapes to serve the stream with, in order: plain (zone per CTA), batched")
    args = ap.parse_args()
    if args.nz is None:
        args.nz = 4096 if args.workload == "mixed" else 1024

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "traj":
        run_traj(args, rank, world, local)
        return
    if args.workload == "serve":
        run_serve(args, rank, world)
        return
    if args.workload == "hburn":
        run_hburn(args, rank, world)
        return
    if args.workload == "mixed":
        run_mixed(args, rank, world)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev_id = torch.cuda.current_device()

    abi = importlib.import_module(PKG + ".abi")
    wl = importlib.import_module(PKG + ".workloads")
    solver = importlib.import_module(PKG + ".solver")
    net = wl.network(1107)
    zb_all = wl.heshell_batch(args.nz * world, net=net, seed=2)
    hot = np.maximum(zb_all.t9_0, zb_all.t9_1)  # weak scaling, shards balanced by peak temperature
    zb = zb_all.take(importlib.import_module(PKG + ".sharding").snake_shards(hot, world)[rank])
    knobs = abi.default_knobs(integration_method=1)
    S = solver.NetworkSolver(net, knobs, device=dev_id)
    nz = zb.nz

    cu = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    X0, ye0 = cu(zb.X), cu(zb.ye)
    t9a, t9b, rha, rhb, dtw = cu(zb.t9_0), cu(zb.t9_1), cu(zb.rho_0), cu(zb.rho_1), cu(zb.dtwant)
    X, ye = X0.clone(), ye0.clone()
    ierr = torch.zeros(nz, dtype=torch.int32, device="cuda")
    stats = torch.zeros((nz, 8), dtype=torch.int32, device="cuda")
    bd = torch.zeros(nz, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # 2x the 126 MB L2

    def one_step():
        X.copy_(X0); ye.copy_(ye0); bd.zero_()
        flush.fill_(1)  # evict the previous call's lines from L2 before the timed region
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        S.integrate_device(X, t9a, t9b, rha, rhb, ye, dtw, ierr, stats, bd, stream=stream)
        e1.record()
        return e0, e1

    ev = []
    steps_done = 0
    with ClockSampler(dev_id) as clk:
        for _ in range(args.warmup):
            one_step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = S.launches()
        clk.mark()
        for _ in range(args.steps):
            ev.append(one_step())
        torch.cuda.synchronize()
    st_np = stats.cpu().numpy()
    steps_done = int(st_np[:, 0].sum()) * args.steps  # identical work every step (same inputs)
    kernel_ms = [a.elapsed_time(b) for a, b in ev]
    t_ms = float(sum(kernel_ms))
    gpu_launches = S.launches() - launches0
    sharding = importlib.import_module(PKG + ".sharding")
    t_ms, steps_done = sharding.reduce_time_and_steps(t_ms, steps_done, "cuda", dist if world > 1 else None)
    value = steps_done / (t_ms * 1e-3)

    # end to end through the host-buffer entry point (host <-> device copies inside)
    Xh = np.ascontiguousarray(zb.X)
    e2e_t, e2e_steps = 0.0, 0
    for it in range(2 + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Xo, yeo, ie, st, _ = S.integrate_network(Xh, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
        dt = time.perf_counter() - t0
        if it >= 2:
            e2e_t += dt
            e2e_steps += sum(s.nsucc for s in st)
    h2d = Xh.nbytes + 6 * 8 * nz + 4 * nz
    d2h = Xh.nbytes + 8 * nz + 4 * nz + 32 * nz + 4 * nz
    e2e_t, e2e_steps = sharding.reduce_time_and_steps(e2e_t, e2e_steps, "cuda", dist if world > 1 else None)
    e2e = e2e_steps / e2e_t

    if rank == 0:
        peak, peak_kind = load_peaks()
        per_launch_s = (sum(kernel_ms) / len(kernel_ms)) * 1e-3
        clocks = clk.summary()
        line = {
            "metric": "zone-timesteps/s", "value": value, "unit": "zone-timesteps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": heshell_config(nz * world, net.nsp),
            "run": {"zones_per_gpu": nz, "nnz_jac": S.info.nnz_jac, "nnz_lu": S.info.nnz_lu, "lu": "fp64",
                    "l2": "flushed: 256 MiB written before each timed call",
                    "accepted_steps_per_call": int(st_np[:, 0].sum()),
                    "rejected_steps_per_call": int(st_np[:, 1].sum())},
            "gpu_launches": int(gpu_launches),
            "e2e": {"value": e2e, "unit": "zone-timesteps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": roofline(nz, net.nsp, S.arena_bytes, per_launch_s, peak, peak_kind, clocks.get("sm_mhz")),
            "clocks": clocks,
        }
        if not args.no_cpu:
            dev_out = (X.cpu().numpy(), ierr.cpu().numpy(), st_np[:, 0])
            line["cpu_baseline"], line["error_vs_oracle"] = cpu_baseline(net, zb, args.cpu_zones, dev_out)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(net, zb, nzones, dev_out):
    """The checker on the host cores, on a fixed sample of the same workload (the 8 hottest zones and
    evenly spaced others): its throughput, and the device results of those zones against it
    (dev_out = final X, ierr and accepted steps of every zone from the last timed call). Zones beyond
    1e-6 are also measured against the checker's own spread under 1-ulp changes of their input,
    rounding-sized changes of its dX/dt and another elimination order of its LU."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import parity
    abi = importlib.import_module(PKG + ".abi")
    if not orc.available():
        return ({"value": None, "unit": "zone-timesteps/s", "cores": 0, "kind": "port", "sample": "unavailable"},
                None)
    cores = os.cpu_count() or 1
    idx = parity_sample(zb, max(nzones, cores))
    sub = zb.take(idx)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    t0 = time.perf_counter()
    Xr, ye, ierr_r, st, _ = ref.integrate_network(sub.X, sub.t9_0, sub.t9_1, sub.rho_0, sub.rho_1, sub.ye,
                                                  sub.dtwant, nthreads=cores)
    dt = time.perf_counter() - t0
    nsucc_r = np.array([s.nsucc for s in st])
    base = {"value": int(nsucc_r.sum()) / dt, "unit": "zone-timesteps/s", "cores": cores, "kind": "port",
            "sample": f"{len(idx)} zones of the batch (the 8 hottest and evenly spaced others; restated FP64 "
                      f"path + reference SuperLU), {dt:.1f} s"}
    X, ierr, nsucc = (a[idx] for a in dev_out)
    rel, ab = parity.zone_errors(X, Xr)
    off = np.nonzero((rel > parity.REL_TOL) | (ab > parity.ABS_TOL))[0]
    spread = np.zeros(len(idx))
    if off.size:
        spread[off] = parity.checker_spread(ref, sub.take(off), Xr[off], nthreads=cores)
    err = parity.summary(X, ierr, nsucc, Xr, ierr_r, nsucc_r, spread)
    err["sample"] = f"{len(idx)} zones: the 8 hottest and evenly spaced others"
    err["spread"] = ("per zone beyond 1e-6: max relative change of the checker under +-1-ulp input changes, "
                     "+-2^-52 changes of every dX/dt entry, and another SuperLU elimination order (2 draws each)")
    return base, err


if __name__ == "__main__":
    main()
