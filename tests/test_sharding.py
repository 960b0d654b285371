"""The multi-rank path on CPU: two gloo ranks (127.0.0.1) shard boxes and
cells with no overlap and full cover, and reduce the step time (maximum)
and the integrator counters (sums; maxima for max_*) the way bench.py does
on NCCL ranks."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from pelelmex_b200 import sharding  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        boxes = sharding.shard_boxes(list(range(40)), rank, world)
        cells = sharding.shard_cells(1001, rank, world)
        got_b, got_c = [None] * world, [None] * world
        dist.all_gather_object(got_b, boxes)
        dist.all_gather_object(got_c, cells.tolist())
        ms = sharding.step_time_max(5.0 + 2.0 * rank)
        cn = sharding.counters_sum({"nfe": 10 + rank, "nst": 3, "max_nfe": 7 * (rank + 1)})
        q.put((rank, got_b, got_c, ms, cn))
    finally:
        dist.destroy_process_group()


def test_single_rank_is_identity():
    assert sharding.step_time_max(3.5) == 3.5
    assert sharding.counters_sum({"nfe": 4}) == {"nfe": 4}
    assert sharding.shard_boxes([1, 2, 3], 0, 1) == [1, 2, 3]
    assert np.array_equal(sharding.shard_cells(5, 0, 1), np.arange(5))


def test_two_gloo_ranks_shard_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got_b, got_c, ms, cn in out:
        allb = sorted(b for part in got_b for b in part)
        assert allb == list(range(40)) and len(set(got_b[0]) & set(got_b[1])) == 0
        allc = sorted(c for part in got_c for c in part)
        assert allc == list(range(1001)) and len(set(got_c[0]) & set(got_c[1])) == 0
        assert ms == 7.0
        assert cn == {"nfe": 21, "nst": 6, "max_nfe": 14}


def test_knapsack_balances_uneven_boxes():
    rng = np.random.default_rng(3)
    # an AMR-like list: a few expensive igniting boxes among many cheap ones
    costs = np.concatenate([rng.uniform(1, 2, 30), rng.uniform(50, 80, 10)])
    world = 4
    rr = np.arange(costs.size) % world
    ks = sharding.knapsack(costs, world)
    assert sharding.efficiency(costs, ks, world) > 0.9  # 10 heavy boxes on 4 ranks: 3-3-2-2 at best
    assert sharding.efficiency(costs, ks, world) > sharding.efficiency(costs, rr, world)
    # every box owned once, box-count cap respected
    capped = sharding.knapsack(costs, world, nmax=10)
    assert np.bincount(capped, minlength=world).max() <= 10


def test_rebalance_follows_the_threshold_rule():
    costs = np.array([10.0, 1.0, 1.0, 1.0, 10.0, 1.0, 1.0, 1.0])
    world = 2
    skewed = np.array([0, 1, 1, 1, 0, 1, 1, 1])   # both heavy boxes on rank 0
    owner, cur, test = sharding.rebalance(costs, skewed, world, threshold=1.1)
    assert test > 1.1 * cur and not np.array_equal(owner, skewed)
    assert sharding.efficiency(costs, owner, world) == test
    balanced = sharding.knapsack(costs, world)
    owner2, cur2, test2 = sharding.rebalance(costs, balanced, world, threshold=1.1)
    assert np.array_equal(owner2, balanced)  # no gain above the threshold: keep
    # the cost of a box is the sum of its cells' fctCount
    assert np.allclose(sharding.box_costs([np.ones(8) * 3, np.arange(4)]), [24.0, 6.0])


def _leaver(rank, world, port, q):
    """Rank 1 leaves between steps (after the first step's reduction, with
    nothing in flight); rank 0's next step-time reduction must end with an
    error within the process group's short timeout, not hang."""
    import datetime
    import time
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    ms = sharding.step_time_max(1.0 + rank)
    if rank == 1:
        q.put((rank, ms, "left", 0.0))
        q.close()
        q.join_thread()
        os._exit(0)  # leaves without tearing the group down, as a crashed rank would
    t0 = time.time()
    try:
        sharding.step_time_max(2.0)
        q.put((rank, ms, "no error", time.time() - t0))
    except Exception as e:  # noqa: BLE001 - the failure surfaces as an error of the collective
        q.put((rank, ms, type(e).__name__, time.time() - t0))
    q.close()
    q.join_thread()
    os._exit(0)


def test_rank_leaving_between_steps_fails_the_next_reduction():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_leaver, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict((r[0], r) for r in (q.get(timeout=120) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert out[1][2] == "left" and out[0][1] == 2.0 and out[1][1] == 2.0
    # rank 0: the reduction of the second step raised instead of hanging
    assert out[0][2] != "no error"
    assert out[0][3] < 60.0
