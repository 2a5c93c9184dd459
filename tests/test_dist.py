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


def _oracle_solve(ns, a, precision):
    # stands in for the per-rank GPU solve on CPU ranks: the oracle, one call
    import oracle as O
    _, u, s, vt = O.svd_batch(ns, a, np.arange(len(ns)), 2)
    return u, s, vt, 0


def _failing_solve(ns, a, precision):
    raise RuntimeError("device lost")


def _shard_worker(rank, world, port, q, count, fail_rank, gather_to):
    import torch.distributed as dist
    from datetime import timedelta
    from lie_cliffalg_analog_svd_b200 import _lib as L
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ns, a, _ = P.uneven_batch_workload(count, seed=5)
        solve = _failing_solve if rank == fail_rank else _oracle_solve
        try:
            u, s, vt, st, rng = D.svd_batched_sharded(ns, a, gather_to=gather_to, solve=solve)
            q.put((rank, "ok", rng, st, u.tobytes(), s.tobytes(), vt.tobytes()))
        except L.LsvdError as e:
            q.put((rank, "error", str(e), None, b"", b"", b""))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run_shards(world, count, fail_rank=-1, gather_to=0):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q, count, fail_rank, gather_to))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("gather_to", [0, None])
def test_sharded_batch_gathers_the_whole_batch(gather_to):
    # two gloo ranks each solve their cost-balanced shard; the gathered packed
    # results equal one process solving the whole batch (the same solver)
    import oracle as O
    count = 400
    res = _run_shards(2, count, gather_to=gather_to)
    ns, a, _ = P.uneven_batch_workload(count, seed=5)
    _, u, s, vt = O.svd_batch(ns, a, np.arange(count), 2)
    receivers = [0] if gather_to == 0 else [0, 1]
    for r in res:
        assert r[1] == "ok" and r[3] == 0
        if r[0] in receivers:
            assert r[2] == (0, count)
            assert r[4] == u.tobytes() and r[5] == s.tobytes() and r[6] == vt.tobytes()
        else:
            lo, hi = r[2]
            assert 0 < lo < hi == count  # rank 1 holds the upper shard only


def test_sharded_batch_failure_reaches_every_rank():
    # a rank whose solve raises: every rank raises instead of waiting in the gather
    res = _run_shards(2, 64, fail_rank=1)
    assert [r[1] for r in res] == ["error", "error"]
    assert "device lost" in res[1][2] and "another rank failed" in res[0][2]


def test_sharded_batch_more_ranks_than_matrices():
    res = _run_shards(2, 1)
    assert res[0][1] == res[1][1] == "ok"
