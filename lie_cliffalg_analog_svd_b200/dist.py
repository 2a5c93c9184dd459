"""Host-side helpers for running the batched workloads on several GPUs of one
node, one process per GPU (``torch.distributed``; NCCL on GPUs, gloo on CPU).

The units of every sharded workload (matrices, families) are independent:
each rank solves its own contiguous, cost-balanced slice with no exchange
while it computes.  ``svd_batched_sharded`` is the library entry for one batch
over the ranks (a status reduction, then one gather of the solved shards);
the benchmark's weak-scaling runs keep their shards where they are and reduce
only the measured time (``max_over_ranks``).
"""
from __future__ import annotations

import os

import numpy as np


def world() -> tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_bounds(costs, world_size: int, rank: int) -> tuple[int, int]:
    """Contiguous slice [lo, hi) of the units for ``rank`` such that the
    cumulative cost is split as evenly as contiguous cuts allow (cut k is the
    first unit whose prefix cost reaches k/world of the total).  For the SVD
    batches the cost of a matrix is n^3."""
    c = np.asarray(costs, dtype=np.float64)
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad world_size / rank")
    if c.size == 0:
        return 0, 0
    pre = np.concatenate([[0.0], np.cumsum(c)])
    tot = pre[-1]

    def cut(k):
        if k <= 0:
            return 0
        if k >= world_size:
            return c.size
        return int(np.searchsorted(pre, tot * k / world_size, side="left"))

    return cut(rank), cut(rank + 1)


def max_over_ranks(value: float, device=None) -> float:
    """Max of ``value`` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _status_over_ranks(code: int) -> int:
    """Largest status code over all ranks (every rank learns of a failure
    before any data moves, so no rank waits in a gather that another skips)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return int(code)
    dev = None
    if dist.get_backend() == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    t = torch.tensor([int(code)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return int(t.item())


# status of a rank whose solve raised (above every lsvd_status)
RANK_FAILED = 1000


def svd_batched_sharded(ns, a, precision: str = "fp64", gather_to: int | None = 0, solve=None):
    """Batched uneven SVD of one batch over the ranks of the process group,
    one GPU per rank.  Every rank passes the same ``ns`` and packed ``a``
    (host arrays); rank r solves the cost-balanced contiguous shard
    ``shard_bounds(ns**3, world, r)`` on its own GPU (``svd_batched``), and the
    shards are gathered on rank ``gather_to`` (all ranks when ``None``).

    Returns ``(U, S, Vt, status, (lo, hi))``: the packed results of the whole
    batch on the receiving ranks (the rank's own shard elsewhere, with its
    matrix range ``(lo, hi)``) and the largest library status over the ranks.
    The only collectives are the status reduction and the gather of results;
    a rank whose solve raises makes every rank raise ``LsvdError``.
    ``solve(ns, a, precision) -> (U, S, Vt, status)`` replaces the GPU solve
    (the default is ``svd_batched`` on this rank's default context)."""
    import torch.distributed as dist

    from . import _lib as L
    from .api import packed_offsets, svd_batched

    ns = np.ascontiguousarray(ns, dtype=np.int32)
    a = np.ascontiguousarray(a, dtype=np.float64)
    ao, so = packed_offsets(ns)
    if a.size != ao[-1]:
        raise L.LsvdError(L.BAD_SHAPE, "svd_batched_sharded: packed A has the wrong length for ns")
    grouped = dist.is_available() and dist.is_initialized()
    world, rank = (dist.get_world_size(), dist.get_rank()) if grouped else (1, 0)
    lo, hi = shard_bounds(ns.astype(np.float64) ** 3, world, rank)
    if solve is None:
        def solve(n_, a_, p_):
            u_, s_, vt_, _, st_ = svd_batched(n_, a_, precision=p_)
            return u_, s_, vt_, st_
    err = None
    try:
        if hi > lo:
            u, s, vt, st = solve(ns[lo:hi], a[ao[lo]:ao[hi]], precision)
        else:
            u, s, vt, st = np.empty(0), np.empty(0), np.empty(0), L.OK
    except Exception as e:  # reported to every rank below
        err, st = e, RANK_FAILED
    status = _status_over_ranks(int(st))
    if status >= RANK_FAILED:
        raise L.LsvdError(L.CUDA_ERROR, f"svd_batched_sharded: a rank failed ({err!r})" if err else
                          "svd_batched_sharded: another rank failed")
    if world == 1:
        return u, s, vt, status, (lo, hi)
    part = (lo, hi, np.asarray(u), np.asarray(s), np.asarray(vt))
    if gather_to is None:
        parts = [None] * world
        dist.all_gather_object(parts, part)
    else:
        parts = [None] * world if rank == gather_to else None
        dist.gather_object(part, parts, dst=gather_to)
        if rank != gather_to:
            return u, s, vt, status, (lo, hi)
    U = np.empty(int(ao[-1]))
    S = np.empty(int(so[-1]))
    Vt = np.empty(int(ao[-1]))
    for plo, phi, pu, ps, pv in parts:
        U[ao[plo]:ao[phi]] = pu
        S[so[plo]:so[phi]] = ps
        Vt[ao[plo]:ao[phi]] = pv
    return U, S, Vt, status, (0, int(ns.size))
