"""The N > 1 host logic on CPU: 2 gloo ranks shard units and agree on the max time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from glc.sharding import shard_range


def test_shard_range_covers_everything_once():
    for n in (0, 1, 7, 100, 4096, 10_001):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert max(b - a for a, b in parts) - min(b - a for a, b in parts) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _point(rate, share, rank):
    return {"rate_req_s": rate, "lookup_share": share, "requests": 100 + rank, "lookups_per_s": 1e9 * (rank + 1),
            "range_gb_s": 10.0, "launches": 50, "lookup_p50_us": 20.0 + rank, "lookup_p99_us": 90.0 + 10 * rank,
            "range_p50_us": None if share == 1.0 else 30.0, "range_p99_us": None if share == 1.0 else 300.0 - rank,
            "span_s": 0.5, "admitted_during": 1, "refused_during": 0, "evictions": rank, "admit_s": 0.01}


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from glc.sharding import gather_objects, max_over_ranks, merge_serving_points, shard_range as sr
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    first, last = sr(1000, rank, world)
    t = max_over_ranks(10.0 + rank)
    # serving: every rank measured its own server; rank 0 merges the points
    mine = [_point(1e5, 0.5, rank), _point(1e6, 1.0, rank)]
    merged = merge_serving_points(gather_objects(mine))
    q.put((rank, first, last, t, merged))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted((q.get(timeout=10) for _ in range(2)), key=lambda r: r[0])
    assert [r[:4] for r in res] == [(0, 0, 500, 11.0), (1, 500, 1000, 11.0)]
    m0, m1 = res[0][4], res[1][4]
    assert m0 == m1 and len(m0) == 2
    mix, lk = m0
    assert mix["rate_req_s"] == 2e5 and mix["gpus"] == 2 and mix["requests"] == 201
    assert mix["lookups_per_s"] == 3e9 and mix["lookup_p99_us"] == 100.0 and mix["range_p99_us"] == 300.0
    assert lk["range_p99_us"] is None and lk["evictions"] == 1 and lk["requests_per_launch"] == round(201 / 100, 2)


def test_column_owner_spreads_columns():
    from glc.sharding import column_owner
    owners = [column_owner(c, 4) for c in range(64)]
    assert [owners.count(r) for r in range(4)] == [16, 16, 16, 16]
