"""The multi-GPU path's host logic on two gloo ranks on the CPU.

bench.py --gpus N gives each rank (one process per GPU) a shard of the zones, balanced by peak
temperature, and reduces only the measurement: the slowest rank's time and the sum of accepted
steps. Here two
ranks run the same sharding and reduction code (the package's sharding module) with the checker
integrating each shard on the CPU: the shards partition the batch, the reduction gives the max and
the sum, and the gathered shard results equal one integration of the whole batch.
"""
import datetime
import importlib
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = "nuppn_modular2-ininet3_b200"
N_PER_RANK, WORLD = 2, 2


def _rank_main(rank, port, q):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        sharding = importlib.import_module(PKG + ".sharding")
        wl = importlib.import_module(PKG + ".workloads")
        abi = importlib.import_module(PKG + ".abi")
        net = wl.network(300)
        zb_all = wl.heshell_batch(N_PER_RANK * WORLD, net=net, seed=3)
        sel = sharding.snake_shards(np.maximum(zb_all.t9_0, zb_all.t9_1), WORLD)[rank]
        zb = zb_all.take(sel)
        ref = oracle.Oracle(net, abi.default_knobs(integration_method=1))
        X, _, ierr, st, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
        steps = sum(s.nsucc for s in st)
        t, total = sharding.reduce_time_and_steps(float(rank + 1), steps, "cpu", dist)
        xs = [torch.zeros(N_PER_RANK, net.nsp, dtype=torch.float64) for _ in range(WORLD)]
        dist.all_gather(xs, torch.from_numpy(np.ascontiguousarray(X)))
        ids = [torch.zeros(N_PER_RANK, dtype=torch.int64) for _ in range(WORLD)]
        dist.all_gather(ids, torch.from_numpy(sel.astype(np.int64)))
        if rank == 0:
            q.put((t, total, np.concatenate([x.numpy() for x in xs]), np.concatenate([i.numpy() for i in ids]),
                   int(np.count_nonzero(ierr))))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_and_reduce(orc, abi, wl):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        t, total, X, ids, nbad = q.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(ids.tolist()) == list(range(N_PER_RANK * WORLD))  # the shards partition the batch
    assert t == float(WORLD)  # the slowest rank's time
    net = wl.network(300)
    zb = wl.heshell_batch(N_PER_RANK * WORLD, net=net, seed=3)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    Xf, _, ierr, st, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant)
    assert nbad == 0 and (ierr == 0).all()
    assert total == sum(s.nsucc for s in st)  # the sum of the ranks' steps
    assert np.array_equal(X[np.argsort(ids)], Xf)  # zones are independent: sharded = whole batch


def test_balanced_shards_partition_and_balance(orc, abi, wl):
    """snake_shards and lpt_shards partition the batch; on the checker's measured work of a He-shell
    batch (1109 species; the hottest zones reject half their steps) both put a smaller maximum load
    on a rank than contiguous shards, snake dealing gives equal zone counts, and LPT is within 4/3 of
    the ideal (Graham's bound) of the measured work."""
    sharding = importlib.import_module(PKG + ".sharding")
    net = wl.network(1107)
    full = wl.heshell_batch(1024, net=net, seed=2)
    world = 4
    # 32 zones: the 8 hottest of the benchmarked batch first (the worst case for contiguous shards)
    pick = np.concatenate([np.argsort(-full.t9_0, kind="stable")[:8], np.arange(0, 1024, 43)[:24]])
    zb = full.take(pick)
    ref = orc.Oracle(net, abi.default_knobs(integration_method=1))
    _, _, ierr, st, _ = ref.integrate_network(zb.X, zb.t9_0, zb.t9_1, zb.rho_0, zb.rho_1, zb.ye, zb.dtwant,
                                              nthreads=8)
    assert (ierr == 0).all()
    work = sharding.work_from_stats([s.nsucc for s in st], [s.nfail for s in st], [s.nvar1_max for s in st])
    contiguous = [sharding.zone_shard(zb.nz // world, r) for r in range(world)]
    snake = sharding.snake_shards(np.maximum(zb.t9_0, zb.t9_1), world)
    lpt = sharding.lpt_shards(work, world)
    for shards in (snake, lpt):
        assert sorted(np.concatenate(shards).tolist()) == list(range(zb.nz))
    assert all(len(s) == zb.nz // world for s in snake)
    worst = lambda shards: sharding.shard_loads(shards, work).max()
    assert worst(snake) < worst(contiguous) and worst(lpt) < worst(contiguous)
    assert worst(lpt) <= (4.0 / 3.0) * max(work.sum() / world, work.max())
