"""Slice-parallel replicas across GPUs (one process per GPU).

Slices are independent in filtered backprojection: the reference spreads
them over OpenCL devices as replicas (ctas src/common/lct.cpp:628-641) and
over threads (src/executables/ct.cpp:156-206).  Here each rank owns a
contiguous range of slices and reconstructs it alone; the only collective is
the max-over-ranks of a timing, and the gather a caller may want at the end.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous range of items owned by `rank` (sizes differ by at most 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (the
    value itself when torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device_sync: bool = True) -> None:
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
    if device_sync and torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()
