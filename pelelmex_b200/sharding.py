"""How the reaction advance spreads over ranks (one process per GPU).

Cells are independent ODE systems with no exchange during the advance
(the reference splits them by boxes across MPI ranks the same way), so a
multi-GPU run needs no collective on the data path: each rank reacts its own
boxes, dealt round-robin, or its own strided subset of cells.  Only the
step time (maximum over ranks) and the integrator counters (sums) are
reduced, between steps, through torch.distributed (NCCL on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard_boxes(items, rank: int, world: int):
    """The boxes rank `rank` of `world` reacts: every world-th, from rank."""
    return list(items)[rank::world]


def shard_cells(n: int, rank: int, world: int) -> np.ndarray:
    """Cell indices (of n) rank `rank` reacts: a strided subset, so every
    rank sees all parts of a field (its cost profile)."""
    return np.arange(rank, n, world, dtype=np.int64)


def _world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist, dist.get_world_size()
    return None, 1


def step_time_max(ms: float, device=None) -> float:
    """The step time of the job: the maximum of the ranks' times."""
    dist, world = _world()
    if world == 1:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def counters_sum(counters: dict, device=None) -> dict:
    """Integrator counters (b200chem_stats as a dict) summed over ranks; the
    max_* entries take the maximum."""
    dist, world = _world()
    if world == 1 or counters is None:
        return counters
    import torch
    keys = sorted(counters)
    vals = torch.tensor([int(counters[k]) for k in keys], dtype=torch.int64, device=device)
    mx = torch.tensor([int(counters[k]) if k.startswith("max_") else 0 for k in keys], dtype=torch.int64,
                      device=device)
    dist.all_reduce(vals, op=dist.ReduceOp.SUM)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    return {k: int(mx[i]) if k.startswith("max_") else int(vals[i]) for i, k in enumerate(keys)}
