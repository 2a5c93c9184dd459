"""Host-side helpers for running the batched workloads on several GPUs of one
node, one process per GPU (``torch.distributed``; NCCL on GPUs, gloo on CPU).

The units of every sharded workload (matrices, families) are independent, so
there is no data-path collective: each rank solves its own contiguous slice
and the only collective is the max-over-ranks reduction of a measured time.
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
