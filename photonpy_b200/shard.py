"""Sharding a batch of ROIs over ranks (one process per GPU).

ROIs are independent, so a batch splits into contiguous ranges, one per rank, with no
exchange on the data path. Each rank fits its range on its own GPU; the results are
concatenated on rank 0 (host-side gather) when the caller wants them in one place. This
is the partitioning photonpy implies (one estimator per device, Context(deviceIndex)).

The helpers use torch.distributed only for plumbing: ``gloo`` on CPU for tests, ``nccl``
on GPUs. Timings are reduced with MAX so a step's time is that of the slowest rank.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, stop) of rank `rank`; the first n % world ranks get one extra ROI."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(int(n), world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return start, stop


def max_over_ranks(value: float, group=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_to_rank0(local: np.ndarray, group=None):
    """Concatenate each rank's rows on rank 0 in rank order (None on other ranks). Shapes may
    differ in the first dimension only."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return local
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    row = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    maxn = max(counts)
    buf = torch.zeros((maxn, row), dtype=torch.from_numpy(np.zeros(0, local.dtype)).dtype, device=dev)
    if local.shape[0]:
        buf[: local.shape[0]] = torch.from_numpy(np.ascontiguousarray(local).reshape(local.shape[0], row)).to(dev)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    if rank != 0:
        return None
    parts = [b[:c].cpu().numpy().reshape((c,) + local.shape[1:]) for b, c in zip(bufs, counts)]
    return np.concatenate(parts, axis=0)
