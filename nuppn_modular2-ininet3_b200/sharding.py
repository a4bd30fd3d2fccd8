"""Zone sharding across ranks, one process per GPU.

Zones are independent within a cycle (mppnp's master/worker loop hands one zone to each worker,
mppnp.F90:653-753; tppnp's trajectories likewise, tppnp.F90:128-199), so each rank integrates its own
shard of a batch with no collective on the data path (weak scaling). The only collectives are the
measurement's: the slowest rank's time and the sum of the ranks' accepted steps.

A rank's time is set by its slowest zones (a zone costs about N^2 per solve, N the active species,
times its sub-steps, and hot He-shell zones reject half their steps), so contiguous shards leave a
rank that happens to hold the hot zones running alone. Two balanced assignments:
  - `snake_shards(key, world)`: when only an order of the zones' cost is known before any call (the
    peak temperature of each zone's interval), zones sorted by decreasing key are dealt to ranks
    0..w-1, then w-1..0, and so on; every rank gets the same number of zones and an equal share of
    each hotness level.
  - `lpt_shards(work, world)`: when a previous call measured each zone's work (mppnp's next cycle,
    tppnp's next interval), longest-processing-time-first: zones by decreasing work, each to the
    rank with the least work so far. `work_from_stats` gives that work from the per-zone statistics
    of `nuppn_integrate`: (accepted + rejected steps) * (largest active system)^2.
"""
from __future__ import annotations

import heapq

import numpy as np


def zone_shard(n_per_rank: int, rank: int) -> np.ndarray:
    """Zone indices of `rank` in a batch of n_per_rank * world zones, contiguous."""
    return np.arange(rank * n_per_rank, (rank + 1) * n_per_rank)


def snake_shards(key, world: int) -> list[np.ndarray]:
    """Zones sorted by decreasing key (ties by index) dealt in a snake order; each shard ascending."""
    key = np.asarray(key, dtype=np.float64)
    order = np.lexsort((np.arange(key.size), -key))
    shards = [[] for _ in range(world)]
    for i, z in enumerate(order):
        lap, pos = divmod(i, world)
        shards[pos if lap % 2 == 0 else world - 1 - pos].append(int(z))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def lpt_shards(work, world: int) -> list[np.ndarray]:
    """Longest-processing-time-first: zones by decreasing work (ties by index), each to the rank with
    the least work so far (ties by rank); each shard ascending."""
    work = np.asarray(work, dtype=np.float64)
    order = np.lexsort((np.arange(work.size), -work))
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for z in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(z))
        heapq.heappush(heap, (load + float(work[z]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def work_from_stats(nsucc, nfail, nvar1_max) -> np.ndarray:
    """Per-zone work of a finished call: (accepted + rejected steps) * max(active species, 1)^2."""
    steps = np.asarray(nsucc, dtype=np.float64) + np.asarray(nfail, dtype=np.float64)
    n = np.maximum(np.asarray(nvar1_max, dtype=np.float64), 1.0)
    return steps * n * n


def shard_loads(shards, work) -> np.ndarray:
    """Total work of each shard."""
    work = np.asarray(work, dtype=np.float64)
    return np.array([work[s].sum() for s in shards])


def reduce_time_and_steps(t: float, steps: int, device, dist=None) -> tuple[float, int]:
    """(max over ranks of t, sum over ranks of steps); the inputs unchanged on one rank."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return t, steps
    import torch
    a = torch.tensor([float(t)], device=device, dtype=torch.float64)
    dist.all_reduce(a, op=dist.ReduceOp.MAX)
    b = torch.tensor([float(steps)], device=device, dtype=torch.float64)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return float(a.item()), int(b.item())
