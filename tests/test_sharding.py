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
