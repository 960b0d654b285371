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


# ---------------------------------------------------- cost-driven balance
# The reference balances the chemistry box layout by the measured cost of
# each box (Source/PeleLMeX_Utils.cpp:817-881, loadBalanceChemLev): a test
# distribution is built by a knapsack over the box costs with at most nmax
# boxes per rank, and adopted when its efficiency (mean rank cost / max rank
# cost) beats the current one by the threshold ratio.  The box cost here is
# the sum of the fctCount the reactor writes (right-hand-side evaluations per
# cell), the reference's functC.

def box_costs(fct_per_box) -> np.ndarray:
    """Cost of each box: the sum of its cells' fctCount."""
    return np.array([float(np.asarray(f).sum()) for f in fct_per_box])


def efficiency(costs, owner, world: int) -> float:
    """Mean rank cost / max rank cost of the assignment owner[box] -> rank."""
    load = np.zeros(world)
    np.add.at(load, np.asarray(owner, dtype=np.int64), np.asarray(costs, dtype=np.float64))
    return float(load.mean() / load.max()) if load.max() > 0 else 1.0


def knapsack(costs, world: int, nmax: int | None = None) -> np.ndarray:
    """Greedy knapsack (largest cost first onto the least-loaded rank that
    still has room for a box; ties by lower rank): owner[box] -> rank."""
    costs = np.asarray(costs, dtype=np.float64)
    n = costs.size
    if nmax is None:
        nmax = n
    nmax = max(int(nmax), -(-n // world))  # room for every box
    owner = np.empty(n, dtype=np.int64)
    load = np.zeros(world)
    count = np.zeros(world, dtype=np.int64)
    for b in sorted(range(n), key=lambda i: (-costs[i], i)):
        open_ranks = np.nonzero(count < nmax)[0]
        r = int(open_ranks[np.argmin(load[open_ranks])])
        owner[b] = r
        load[r] += costs[b]
        count[r] += 1
    return owner


def rebalance(costs, owner, world: int, threshold: float = 1.1, ks_factor: float = 1.5):
    """The reference's decision (loadBalanceChemLev with the knapsack
    method): test layout with nmax = max(round(ks_factor * boxes/ranks),
    ceil(boxes/ranks)); keep it when test efficiency > threshold x current.
    Returns (owner to use, current efficiency, test efficiency)."""
    n = len(costs)
    navg = n / world
    nmax = int(max(round(ks_factor * navg), np.ceil(navg)))
    test = knapsack(costs, world, nmax)
    cur_eff = efficiency(costs, owner, world)
    test_eff = efficiency(costs, test, world)
    return (test if test_eff > threshold * cur_eff else np.asarray(owner)), cur_eff, test_eff
