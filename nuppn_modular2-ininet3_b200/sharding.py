"""Zone sharding across ranks, one process per GPU.

Zones are independent within a cycle (mppnp's master/worker loop hands one zone to each worker,
mppnp.F90:653-753; tppnp's trajectories likewise, tppnp.F90:128-199), so rank r integrates the
contiguous shard [r*n, (r+1)*n) of a batch of n*world zones with no collective on the data path
(weak scaling). The only collectives are the measurement's: the slowest rank's time and the sum of
the ranks' accepted steps.
"""
from __future__ import annotations

import numpy as np


def zone_shard(n_per_rank: int, rank: int) -> np.ndarray:
    """Zone indices of `rank` in a batch of n_per_rank * world zones."""
    return np.arange(rank * n_per_rank, (rank + 1) * n_per_rank)


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
