"""Multi-GPU sharding of independent units (one process per GPU).

The transforms of different signals, images or volumes are independent, so
N GPUs split the units and need no collective on the data path: each rank
plans and runs its own shard (for a batch, its own persistent launch).  The
only collectives are host-side bookkeeping: gathering results when a caller
wants them on one rank, and the max over ranks of a device time.

``shard_signals`` splits a batch into contiguous ranges of signals with
nearly equal sample counts (the work of a transform is proportional to its
samples); ``rank_batch`` cuts a rank's share out of packed signal arrays.
"""
from __future__ import annotations

import numpy as np


def shard_signals(lengths, world: int):
    """Boundaries b (len world+1) such that rank r owns signals
    [b[r], b[r+1]); cumulative sample counts are split as evenly as
    contiguous ranges allow."""
    if world < 1:
        raise ValueError("world must be >= 1")
    lengths = np.asarray(lengths, dtype=np.int64)
    n = len(lengths)
    cum = np.concatenate([[0], np.cumsum(lengths)])
    total = int(cum[-1])
    b = [0]
    for r in range(1, world):
        target = total * r / world
        i = int(np.searchsorted(cum, target, side="left"))
        # the boundary nearer the target, never before the previous one
        if i > 0 and abs(cum[i - 1] - target) <= abs(cum[min(i, n)] - target):
            i -= 1
        b.append(min(max(i, b[-1]), n))
    b.append(n)
    return b


def rank_batch(lengths, wavelets, levels, rank: int, world: int):
    """This rank's (first, last, lengths, wavelets, levels, offset) where
    offset is the element offset of its first signal in the packed layout."""
    b = shard_signals(lengths, world)
    lo, hi = b[rank], b[rank + 1]
    lengths = np.asarray(lengths, dtype=np.int64)
    off = int(lengths[:lo].sum())
    wl = list(wavelets[lo:hi]) if not isinstance(wavelets, (int, str)) else wavelets
    lv = list(levels[lo:hi]) if np.ndim(levels) else levels
    return lo, hi, lengths[lo:hi], wl, lv, off


def max_over_ranks(value: float, group=None) -> float:
    """Max of a per-rank float over the default (or given) process group."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
