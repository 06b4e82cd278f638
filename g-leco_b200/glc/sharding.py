"""Multi-GPU placement for the decode path: one process per GPU, no data-path collective.

Columns (and partition ranges of one column) are independent, so work is split across ranks
with no exchange step; the only collective is the max over ranks of the measured time.
"""
from __future__ import annotations


def shard_range(n_units: int, rank: int, world: int):
    """Contiguous [first, last) units of `rank` out of `world` (the first ranks take one more)."""
    base, extra = divmod(n_units, world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (a device time) over all ranks of the default process group."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
