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


def combine_tensor(val_idx, group=None):
    """Global (max value, smallest index attaining it) of a 2-element int64
    tensor (value, Gray index) per rank, without leaving the device: two
    all-reduces (MAX on the value, MIN on the index of the ranks at the
    maximum) queued on the current stream.  Returns two 1-element tensors.
    Gray indices are below 2^63, so an index read as int64 keeps its order."""
    import torch
    import torch.distributed as dist

    v = val_idx[0:1].clone()
    dist.all_reduce(v, op=dist.ReduceOp.MAX, group=group)
    i = torch.where(val_idx[0:1] == v, val_idx[1:2], torch.full_like(val_idx[1:2], INT64_MAX))
    dist.all_reduce(i, op=dist.ReduceOp.MIN, group=group)
    return v, i


def combine(value: int, index: int, group=None, device=None) -> tuple[int, int]:
    """Global (max value, smallest index attaining it) over the ranks, from
    host integers (combine_tensor on a tensor of the given device)."""
    import torch

    dev = device if device is not None else "cpu"
    v, i = combine_tensor(torch.tensor([value, index], dtype=torch.int64, device=dev), group=group)
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
