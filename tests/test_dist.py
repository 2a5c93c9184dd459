"""Multi-rank host logic on CPU: two gloo ranks (127.0.0.1) check the
max-over-ranks timing reduction and that cost-balanced contiguous shards
partition a batch exactly (every matrix on exactly one rank)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lie_cliffalg_analog_svd_b200 import dist as D
from lie_cliffalg_analog_svd_b200 import profiles as P


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = D.max_over_ranks(10.0 + rank)
        ns, _, _ = P.uneven_batch_workload(500, seed=3)
        lo, hi = D.shard_bounds(ns.astype(np.float64) ** 3, world, rank)
        q.put((rank, got, lo, hi))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(r[1] == 10.0 + world - 1 for r in res)
    bounds = [(r[2], r[3]) for r in res]
    assert bounds[0][0] == 0 and bounds[-1][1] == 500
    for (a, b), (c, d) in zip(bounds, bounds[1:]):
        assert b == c


def test_shard_bounds_balance():
    ns, _, _ = P.uneven_batch_workload(10_000, seed=1)
    cost = ns.astype(np.float64) ** 3
    for w in (1, 2, 3, 8):
        cuts = [D.shard_bounds(cost, w, r) for r in range(w)]
        assert cuts[0][0] == 0 and cuts[-1][1] == cost.size
        loads = [cost[a:b].sum() for a, b in cuts]
        assert max(loads) - min(loads) <= 2 * cost.max()
    assert D.shard_bounds([], 4, 2) == (0, 0)
    with pytest.raises(ValueError):
        D.shard_bounds(cost, 2, 2)


def test_max_over_ranks_single_process():
    assert D.max_over_ranks(3.5) == 3.5
