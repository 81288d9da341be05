"""Multi-GPU sharding of one exact solve (one process per GPU).

The Gray-index space of a solve splits into contiguous shards with no
communication while they run (`ld_options.shard_index / shard_count`); the
only exchange is the 16-byte candidate of each rank: the global value is the
maximum, and among the ranks that reach it the smallest Gray index wins (the
reference's host argmax keeps the lowest worker on ties, L_CUDA.cu:345-348,
which is the smallest index because ranges are contiguous and ordered).

`combine` works on any torch.distributed backend: CUDA tensors over NCCL on
GPU ranks, CPU tensors over gloo (the tests run it that way).
"""
from __future__ import annotations

import numpy as np

INT64_MAX = np.iinfo(np.int64).max


def shard_bounds(units: int, index: int, count: int) -> tuple[int, int]:
    """[lo, hi) of shard `index` of `count` over `units` (the calc_jmin_jmax
    split, L_CUDA.cu:5-12, which the library applies to its walks)."""
    if count <= 1:
        return 0, units
    q, r = divmod(units, count)
    lo = index * q + min(index, r)
    return lo, lo + q + (1 if index < r else 0)


def combine(value: int, index: int, group=None, device=None) -> tuple[int, int]:
    """Global (max value, smallest index attaining it) over the ranks."""
    import torch
    import torch.distributed as dist

    dev = device if device is not None else "cpu"
    v = torch.tensor([value], dtype=torch.int64, device=dev)
    dist.all_reduce(v, op=dist.ReduceOp.MAX, group=group)
    mine = index if value == int(v.item()) else INT64_MAX
    i = torch.tensor([mine], dtype=torch.int64, device=dev)
    dist.all_reduce(i, op=dist.ReduceOp.MIN, group=group)
    return int(v.item()), int(i.item())


def solve_sharded(ld, a, d: int, marginal: bool, rank: int, world: int, device: int = 0,
                  group=None):
    """One rank's part of a sharded exact solve, combined over the group.
    `ld` is the loaded package.  Returns (value, gray_index, local Solution)."""
    import torch

    plan = ld.Plan(a, d, marginal, ld.options(device=device, shard_index=rank, shard_count=world))
    sol = plan.solve()
    plan.close()
    dev = torch.device("cuda", device) if torch.cuda.is_available() else None
    value, index = combine(sol.value, sol.gray_index, group=group, device=dev)
    return value, index, sol
