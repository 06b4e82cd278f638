"""Multi-GPU placement for the decode and serving paths: one process per GPU, no data-path
collective.

Columns (and partition ranges of one column) are independent, so work is split across ranks
with no exchange step; the only collectives are the max over ranks of a measured time and, for
serving, the merge of each rank's measured rate points (every rank serves its own columns).
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


def column_owner(column_id: int, world: int) -> int:
    """The rank that serves a column: whole columns per GPU, round robin."""
    return column_id % world


def merge_serving_points(per_rank):
    """Merge the rate points each rank measured on its own server (same offered rate per GPU, in
    the same order): throughputs add up, latency percentiles take the worst rank, counts add up."""
    if not per_rank:
        return []
    n = len(per_rank[0])
    assert all(len(p) == n for p in per_rank), "every rank runs the same rate points"
    add = ("requests", "lookups_per_s", "range_gb_s", "launches", "admitted_during", "refused_during", "evictions")
    worst = ("lookup_p50_us", "lookup_p99_us", "range_p50_us", "range_p99_us", "span_s", "admit_s")
    out = []
    for i in range(n):
        pts = [p[i] for p in per_rank]
        assert len({pt["rate_req_s"] for pt in pts}) == 1 and len({pt["lookup_share"] for pt in pts}) == 1
        m = {"rate_req_s_per_gpu": pts[0]["rate_req_s"], "rate_req_s": pts[0]["rate_req_s"] * len(pts),
             "lookup_share": pts[0]["lookup_share"], "gpus": len(pts)}
        for k in add:
            if k in pts[0]:
                m[k] = round(sum(pt[k] for pt in pts), 2)
        for k in worst:
            vals = [pt[k] for pt in pts if pt.get(k) is not None]
            m[k] = max(vals) if vals else None
        m["requests_per_launch"] = round(m["requests"] / max(1, m.get("launches", 1)), 2)
        out.append(m)
    return out


def gather_objects(obj):
    """All ranks' objects in rank order (one rank: [obj])."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
