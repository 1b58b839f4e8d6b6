"""Work sharding over GPUs for the batched and served builds (one process per GPU).

Chunks are independent units, so the path shards with no collective on the data
path: every rank derives the same assignment from the same inputs and builds only
its own chunks; results stay on the GPU that built them. The only communication is
host-side bookkeeping after the timed work (the max of the ranks' device times, the
sum of their voxels), over whatever process group the caller has (NCCL on GPUs, gloo
in the CPU tests).

The reference's world streaming builds one batch per update on one GPU
(src/world.zig:1014-1020); this module is the multi-GPU extension of that loop.
"""
from __future__ import annotations

import numpy as np


def chunk_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of `total` chunk indices for `rank` (sizes differ by at most one)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def partition_chunks(sizes, world: int) -> list[np.ndarray]:
    """Longest-processing-time split of chunks (by voxel count) over `world` ranks:
    the largest chunk goes to the rank with the smallest load so far (ties: lowest
    rank, then lowest chunk index). Deterministic, so every rank computes the same
    split. Returns each rank's chunk indices in ascending order."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.lexsort((np.arange(len(sizes)), -sizes))
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(sizes), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += sizes[i]
    return [np.nonzero(owner == r)[0] for r in range(world)]


def route_requests(sizes, world: int, rates=None) -> np.ndarray:
    """Rank of each request of an arrival stream (in arrival order): the rank with the
    least voxels routed so far, weighted by its relative speed `rates[r]` (default
    equal). Deterministic, so every rank routes the same stream the same way and
    serves only its own requests."""
    w = np.ones(world) if rates is None else np.asarray(rates, dtype=np.float64)
    load = np.zeros(world)
    out = np.empty(len(sizes), dtype=np.int64)
    for i, s in enumerate(np.asarray(sizes, dtype=np.int64)):
        r = int(np.argmin(load / w))
        out[i] = r
        load[r] += s
    return out


def combine(values: dict, group=None) -> dict:
    """Host bookkeeping after the timed work: sums of counts ('voxels', 'entries',
    'chunks', 'requests') and the max of times ('ms') over the ranks of `group`."""
    import torch
    import torch.distributed as dist
    keys = sorted(values)
    if not dist.is_available() or not dist.is_initialized():
        return dict(values)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    sums = [k for k in keys if not k.endswith("ms")]
    maxes = [k for k in keys if k.endswith("ms")]
    out = {}
    if sums:
        t = torch.tensor([float(values[k]) for k in sums], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out.update({k: float(v) for k, v in zip(sums, t.tolist())})
    if maxes:
        t = torch.tensor([float(values[k]) for k in maxes], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        out.update({k: float(v) for k, v in zip(maxes, t.tolist())})
    return out
