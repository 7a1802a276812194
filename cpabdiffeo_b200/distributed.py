"""One process per GPU: independent shards of a batch, no collective on the
data path.  Transform instances, point ranges and MCMC chains never exchange
data, so each rank integrates a contiguous shard; collectives appear only for
bookkeeping (timing = max over ranks) and for gathering results when a caller
wants them on one rank.  Works with the nccl (GPU) and gloo (CPU) backends.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    """(rank, world size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(n: int, rank: int, size: int) -> tuple[int, int]:
    """Contiguous [start, end) of n items for `rank` of `size` (sizes differ by at most one)."""
    base, extra = divmod(n, size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_ragged(offsets: np.ndarray, rank: int, size: int) -> tuple[int, int]:
    """Contiguous range of instances with about equal point counts for `rank`."""
    offsets = np.asarray(offsets)
    total = int(offsets[-1])
    n = len(offsets) - 1
    cut = lambda r: int(np.searchsorted(offsets, total * r / size, side="left"))  # noqa: E731
    a = 0 if rank == 0 else min(cut(rank), n)
    b = n if rank == size - 1 else min(cut(rank + 1), n)
    return a, max(a, b)


def max_over_ranks(value: float, device=None) -> float:
    rank, size = world()
    if size == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    rank, size = world()
    if size == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_to_rank0(local: torch.Tensor) -> torch.Tensor | None:
    """Concatenate every rank's [n_r, ...] tensor on rank 0 (rank order); None elsewhere."""
    rank, size = world()
    if size == 1:
        return local
    dev = local.device
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(size)]
    dist.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes)
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=dev)
    pad[:local.shape[0]] = local
    bufs = [torch.zeros_like(pad) for _ in range(size)]
    dist.all_gather(bufs, pad)
    if rank != 0:
        return None
    return torch.cat([b[:s] for b, s in zip(bufs, sizes)])
