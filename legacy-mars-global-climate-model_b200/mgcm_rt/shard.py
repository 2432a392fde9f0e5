"""Column sharding over ranks (one process per GPU).

Radiation columns are independent (code/comp3.f:411-1044 touches only (J,I)
for the radiation), so the data path needs no collective: each rank owns a
contiguous range of the global columns (latitude bands of the J,I grid) and
runs it alone.  Two collectives exist around it: the max over ranks of a
timing (every multi-GPU number is the slowest rank's) and, for a caller that
wants global arrays, an all-gather of the per-rank outputs.  Both work on
the `nccl` (CUDA tensors) and `gloo` (CPU tensors) backends.
"""
from __future__ import annotations

import numpy as np


def column_shard(ncol_global: int, rank: int, world: int) -> tuple[int, int]:
    """[c0, c1) of rank `rank`: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world or ncol_global < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(ncol_global, world)
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


def _device(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float, dist=None) -> float:
    """The slowest rank's value (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_columns(arr, dist, ncol_global: int):
    """All-gather a rank's [c1-c0, ...] output into the global [ncol, ...]
    array on every rank (ranks hold column_shard ranges, in rank order)."""
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    dev = _device(dist)
    t = torch.as_tensor(np.ascontiguousarray(arr) if isinstance(arr, np.ndarray) else arr).to(dev)
    sizes = [column_shard(ncol_global, r, world) for r in range(world)]
    width = max(c1 - c0 for c0, c1 in sizes)
    pad = torch.zeros((width,) + tuple(t.shape[1:]), dtype=t.dtype, device=dev)
    pad[: t.shape[0]] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    full = torch.cat([p[: c1 - c0] for p, (c0, c1) in zip(parts, sizes)])
    return full.cpu().numpy() if isinstance(arr, np.ndarray) else full
