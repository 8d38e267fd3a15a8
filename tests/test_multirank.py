"""Multi-rank host logic on CPU: two gloo ranks, no GPU.

Covers the N > 1 path of the benchmark: per-rank seeds of the weak-scaling
batches, the max-over-ranks device time and the sum of processed units, and
the cost-balanced contiguous shards of one batch.
"""

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    import datetime

    import torch.distributed as dist

    from art import sharding

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        info = sharding.rank_info()
        ms = 10.0 + 5.0 * info.rank                     # a per-rank device time
        units = 100 * (info.rank + 1)
        res = (info.rank, info.world, sharding.rank_seed(2, info.rank), sharding.max_over_ranks(ms, device="cpu"),
               sharding.sum_over_ranks(units, device="cpu"))
        dist.barrier()
        out.put(res)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_units():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 2 for g in got)
    assert [g[2] for g in got] == [2, 3]                 # distinct weak-scaling batches
    assert all(g[3] == pytest.approx(15.0) for g in got)  # max over ranks, on every rank
    assert all(g[4] == pytest.approx(300.0) for g in got)


def test_single_process_reductions_are_identity():
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art import sharding

    assert sharding.max_over_ranks(3.5) == 3.5
    assert sharding.sum_over_ranks(7) == 7.0


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_balanced_shards_cover_every_segment_once(world):
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art import sharding

    rng = np.random.default_rng(0)
    n = np.floor(np.exp(rng.uniform(np.log(64), np.log(8192), 4096))).astype(int)
    p = rng.choice([9, 17, 45, 153], 4096)
    b = sharding.balanced_shards(n, p, world)
    assert b[0] == 0 and b[-1] == n.size and np.all(np.diff(b) >= 0)
    cost = n * (p + 1.0) ** 2
    shares = np.array([cost[b[r]:b[r + 1]].sum() for r in range(world)])
    assert shares.sum() == pytest.approx(cost.sum())
    assert np.all(np.abs(shares - cost.sum() / world) <= cost.max() + 1e-6)


def test_balanced_shards_edge_cases():
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art import sharding

    assert list(sharding.balanced_shards([], [], 2)) == [0, 0, 0]
    assert list(sharding.balanced_shards([0, 0, 0, 0], [3, 3, 3, 3], 2)) == [0, 2, 4]
    b = sharding.balanced_shards([10], [5], 4)
    assert b[0] == 0 and b[-1] == 1 and np.all(np.diff(b) >= 0)
    with pytest.raises(ValueError):
        sharding.balanced_shards([1, 2], [3], 2)
    with pytest.raises(ValueError):
        sharding.balanced_shards([1], [3], 0)
