"""Serving (glc_server_*): resident columns, admission budget and continuously batched requests.

Every request's result must be the same when it runs alone and when it shares launches with the
rest of a mixed stream (lookups and range decodes over columns of every element type, ranges
split into pieces, outputs that need staging), and must equal the column's values.
"""
import time

import numpy as np
import pytest
import torch

import glc

pytestmark = pytest.mark.gpu

DT = {glc.I32: (np.int32, torch.int32), glc.I64: (np.int64, torch.int64), glc.U64: (np.uint64, torch.int64),
      glc.U32: (np.uint32, torch.int32)}


def _values(dt, n, seed):
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    noise = rng.integers(0, 1 << int(rng.integers(1, 18)), n)
    if dt in (glc.I32, glc.U32):
        return ((int(rng.integers(0, 1 << 20)) + 37 * i + noise) % (1 << 31)).astype(DT[dt][0])
    v = int(rng.integers(0, 1 << 40)) + 9001 * i + noise
    if dt == glc.U64 and seed % 2:
        v[n // 3: n // 3 + 5000] += 1 << 60  # partitions above 2^53: direct copy
    return v.astype(DT[dt][0])


def _columns(ctx, server, specs):
    cols = []
    for k, (dt, n, mode) in enumerate(specs):
        v = _values(dt, n, seed=100 + k)
        c = glc.compress_device(ctx, dt, v.ctypes.data, n, mode, host=True)
        cols.append((server.admit(c), dt, v))
    return cols


def _mixed_requests(cols, nreq, seed, big=400_000):
    rng = np.random.default_rng(seed)
    reqs = []
    for t in range(nreq):
        cid, dt, v = cols[int(rng.integers(0, len(cols)))]
        n = len(v)
        if rng.random() < 0.5:
            q = int(np.exp(rng.uniform(0, np.log(20_000))))
            pos = rng.integers(-5, n + 5, q).astype(np.int32)  # a few outside the column: 0
            want = np.where((pos >= 0) & (pos < n), v[np.clip(pos, 0, n - 1)], 0).astype(v.dtype)
            reqs.append(dict(kind=glc.REQ_LOOKUP, col=cid, dt=dt, pos=pos, want=want, tag=t))
        else:
            cnt = int(np.exp(rng.uniform(np.log(1), np.log(big))))
            cnt = min(cnt, n)
            first = int(rng.integers(0, n - cnt + 1))
            skew = int(rng.integers(0, 4))  # output offset in elements: some need staging
            reqs.append(dict(kind=glc.REQ_RANGE, col=cid, dt=dt, first=first, count=cnt, skew=skew,
                             want=v[first:first + cnt], tag=t))
    return reqs


def _device_buffers(reqs):
    for r in reqs:
        np_t, th_t = DT[r["dt"]]
        if r["kind"] == glc.REQ_LOOKUP:
            r["dpos"] = torch.from_numpy(r["pos"]).cuda()
            r["dout"] = torch.full((len(r["pos"]),), -7, dtype=th_t, device="cuda:0")
            r["optr"] = r["dout"].data_ptr()
        else:
            r["dout"] = torch.full((r["count"] + 8,), -7, dtype=th_t, device="cuda:0")
            r["optr"] = r["dout"].data_ptr() + r["skew"] * np.dtype(np_t).itemsize
    torch.cuda.synchronize()  # the server's streams do not wait for torch's


def _as_array(reqs, not_before=None):
    a = glc.requests(len(reqs))
    for i, r in enumerate(reqs):
        a[i]["kind"] = r["kind"]
        a[i]["column"] = r["col"]
        a[i]["tag"] = r["tag"]
        a[i]["out"] = r["optr"]
        if r["kind"] == glc.REQ_LOOKUP:
            a[i]["count"] = len(r["pos"])
            a[i]["positions"] = r["dpos"].data_ptr()
        else:
            a[i]["first"] = r["first"]
            a[i]["count"] = r["count"]
        if not_before is not None:
            a[i]["not_before_ns"] = not_before[i]
    return a


def _results(reqs):
    torch.cuda.synchronize()
    got = []
    for r in reqs:
        np_t = DT[r["dt"]][0]
        h = r["dout"].cpu().numpy().view(np_t)
        if r["kind"] == glc.REQ_LOOKUP:
            got.append(h.copy())
        else:
            s = r["skew"]
            assert np.all(h[:s] == np.array(-7).astype(np_t)), "write before the output"
            assert np.all(h[s + r["count"]:] == np.array(-7).astype(np_t)), "write past the output"
            got.append(h[s:s + r["count"]].copy())
    return got


SPECS = [(glc.I32, 300_001, glc.FIXED), (glc.I64, 1_000_003, glc.VARIABLE), (glc.U64, 777_777, glc.VARIABLE),
         (glc.U32, 123_456, glc.FIXED), (glc.U64, 2_000_000, glc.FIXED), (glc.I64, 4_097, glc.FIXED)]


def test_each_result_same_alone_and_in_the_mix():
    ctx = glc.Context(0)
    server = glc.Server(ctx, budget_bytes=1 << 32, slots=3, max_range_values=100_000, max_lookups=50_000)
    cols = _columns(ctx, server, SPECS)
    reqs = _mixed_requests(cols, 160, seed=5)
    _device_buffers(reqs)

    for r in reqs:  # alone: one request in flight at a time
        torch.cuda.synchronize()
        server.submit(_as_array([r]))
        server.drain(60_000)
    alone = _results(reqs)
    recs = server.poll()
    assert len(recs) == len(reqs) and np.all(recs["status"] == glc.OK)
    for r, g in zip(reqs, alone):
        assert np.array_equal(g, r["want"]), (r["kind"], r["tag"])

    alone_launches = server.stats().launches
    for r in reqs:
        r["dout"].fill_(-7)
    torch.cuda.synchronize()
    t0 = server.now_ns()
    rng = np.random.default_rng(9)
    arrivals = t0 + np.sort(rng.integers(0, 30_000_000, len(reqs)))  # spread over 30 ms
    torch.cuda.synchronize()
    server.submit(_as_array(reqs, arrivals))
    server.drain(60_000)
    mixed = _results(reqs)
    recs = server.poll()
    assert len(recs) == len(reqs) and np.all(recs["status"] == glc.OK)
    for r, g in zip(reqs, mixed):
        assert np.array_equal(g, r["want"]), (r["kind"], r["tag"])
    by_tag = {int(c["tag"]): c for c in recs}
    for r in reqs:
        c = by_tag[r["tag"]]
        assert c["arrival_ns"] >= arrivals[r["tag"]] and c["done_ns"] > c["arrival_ns"]
        if r["kind"] == glc.REQ_RANGE:
            assert c["launches"] >= -(-r["count"] // 100_000)  # split into pieces
    st = server.stats()
    assert st.completed == st.submitted == 2 * len(reqs)
    assert st.launches - alone_launches < alone_launches  # in the mix, requests shared launches
    assert st.lookups == 2 * sum(len(r["pos"]) for r in reqs if r["kind"] == glc.REQ_LOOKUP)
    server.close()


def test_everything_submitted_at_once_shares_launches():
    ctx = glc.Context(0)
    server = glc.Server(ctx, budget_bytes=1 << 32, slots=2)
    cols = _columns(ctx, server, SPECS[:4])
    reqs = _mixed_requests(cols, 400, seed=6, big=50_000)
    _device_buffers(reqs)
    torch.cuda.synchronize()
    server.submit(_as_array(reqs))
    server.drain(60_000)
    for r, g in zip(reqs, _results(reqs)):
        assert np.array_equal(g, r["want"])
    st = server.stats()
    assert st.launches <= 20, st.launches  # 400 requests in a handful of shared launches
    server.close()


def test_admission_budget_and_lru_eviction():
    ctx = glc.Context(0)
    v = _values(glc.I64, 500_000, 1)
    probe = glc.compress_device(ctx, glc.I64, v.ctypes.data, len(v), glc.FIXED, host=True)
    server = glc.Server(ctx, budget_bytes=1 << 40)
    a = server.admit(probe)
    one = server.stats().resident_bytes
    server.close()

    server = glc.Server(ctx, budget_bytes=int(2.5 * one))  # room for two such columns
    ids = []
    for k in range(2):
        ids.append(server.admit(glc.compress_device(ctx, glc.I64, v.ctypes.data, len(v), glc.FIXED, host=True)))
    assert server.stats().resident_columns == 2
    # touch column 0 so that column 1 is the least recently used
    pos = torch.arange(10, dtype=torch.int32, device="cuda:0")
    out = torch.zeros(10, dtype=torch.int64, device="cuda:0")
    r = glc.requests(1)
    r[0] = (glc.REQ_LOOKUP, ids[0], 0, 10, pos.data_ptr(), out.data_ptr(), 0, 0)
    torch.cuda.synchronize()
    server.submit(r)
    server.drain(10_000)
    ids.append(server.admit(glc.compress_device(ctx, glc.I64, v.ctypes.data, len(v), glc.FIXED, host=True)))
    st = server.stats()
    assert st.resident_columns == 2 and st.evictions == 1 and st.resident_bytes <= int(2.5 * one)
    with pytest.raises(glc.GlcError) as e:  # evicted column: the request is refused on the host
        r[0]["column"] = ids[1]
        torch.cuda.synchronize()
        server.submit(r)
    assert e.value.status == glc.ERR_INVALID_ARG

    # requests waiting (arrival far ahead) pin both columns: admission is refused, nothing evicted
    far = server.now_ns() + 300_000_000
    r2 = glc.requests(2)
    r2[0] = (glc.REQ_LOOKUP, ids[0], 0, 10, pos.data_ptr(), out.data_ptr(), 1, far)
    out2 = torch.zeros(10, dtype=torch.int64, device="cuda:0")
    r2[1] = (glc.REQ_LOOKUP, ids[2], 0, 10, pos.data_ptr(), out2.data_ptr(), 2, far)
    torch.cuda.synchronize()
    server.submit(r2)
    extra = glc.compress_device(ctx, glc.I64, v.ctypes.data, len(v), glc.FIXED, host=True)
    with pytest.raises(glc.GlcError) as e:
        server.admit(extra)
    assert e.value.status == glc.ERR_BUDGET
    assert extra.handle is not None  # the caller keeps the refused column
    st = server.stats()
    assert st.admissions_refused == 1 and st.resident_columns == 2
    server.drain(10_000)
    assert np.array_equal(out.cpu().numpy(), v[:10]) and np.array_equal(out2.cpu().numpy(), v[:10])
    server.admit(extra)  # idle again: admission evicts the LRU column
    assert server.stats().resident_columns == 2
    server.close()


def test_evict_waits_for_submitted_requests():
    ctx = glc.Context(0)
    server = glc.Server(ctx, budget_bytes=1 << 32)
    v = _values(glc.U32, 200_000, 3)
    cid = server.admit(glc.compress_device(ctx, glc.U32, v.ctypes.data, len(v), glc.VARIABLE, host=True))
    out = torch.zeros(len(v), dtype=torch.int32, device="cuda:0")
    r = glc.requests(1)
    r[0] = (glc.REQ_RANGE, cid, 0, len(v), 0, out.data_ptr(), 0, server.now_ns() + 100_000_000)
    torch.cuda.synchronize()
    server.submit(r)
    before = server.stats().resident_bytes
    server.evict(cid)
    assert server.stats().resident_bytes == before  # still pinned by the waiting request
    with pytest.raises(glc.GlcError):
        torch.cuda.synchronize()
        server.submit(r)
    server.drain(10_000)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), v)
    st = server.stats()
    assert st.resident_bytes == 0 and st.resident_columns == 0
    server.close()


def test_invalid_requests_queue_nothing():
    ctx = glc.Context(0)
    server = glc.Server(ctx, budget_bytes=1 << 32)
    v = _values(glc.I32, 10_000, 4)
    cid = server.admit(glc.compress_device(ctx, glc.I32, v.ctypes.data, len(v), glc.FIXED, host=True))
    out = torch.zeros(100, dtype=torch.int32, device="cuda:0")
    r = glc.requests(2)
    r[0] = (glc.REQ_RANGE, cid, 0, 100, 0, out.data_ptr(), 0, 0)
    r[1] = (glc.REQ_RANGE, cid, 9_950, 100, 0, out.data_ptr(), 1, 0)  # past the end
    with pytest.raises(glc.GlcError):
        torch.cuda.synchronize()
        server.submit(r)
    r[1] = (glc.REQ_LOOKUP, cid, 0, 0, 0, out.data_ptr(), 1, 0)  # count 0
    with pytest.raises(glc.GlcError):
        torch.cuda.synchronize()
        server.submit(r)
    r[1] = (glc.REQ_RANGE, cid + 7, 0, 10, 0, out.data_ptr(), 1, 0)  # unknown column
    with pytest.raises(glc.GlcError):
        torch.cuda.synchronize()
        server.submit(r)
    assert server.stats().submitted == 0
    torch.cuda.synchronize()
    server.submit(r[:1])
    server.drain(10_000)
    assert np.array_equal(out.cpu().numpy(), v[:100])
    server.close()


@pytest.mark.parametrize("reserve", [False, True])
def test_admit_blob_from_device_memory(oracle, reserve):
    ctx = glc.Context(0)
    server = glc.Server(ctx, budget_bytes=1 << 30, reserve=reserve)
    v = _values(glc.U64, 300_000, 5)
    blob = oracle.serialize(oracle.compress(v, "fixed", 2048))
    dblob = torch.from_numpy(np.frombuffer(blob, np.uint8).copy()).cuda()
    cid = server.admit_blob(glc.U64, dblob.data_ptr(), len(blob))
    out = torch.zeros(len(v), dtype=torch.int64, device="cuda:0")
    r = glc.requests(1)
    r[0] = (glc.REQ_RANGE, cid, 0, len(v), 0, out.data_ptr(), 0, 0)
    torch.cuda.synchronize()
    server.submit(r)
    server.drain(10_000)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), v)
    # blob columns live in the server's pool: evicting and re-admitting reuses it
    server.evict(cid)
    host_blob = np.frombuffer(blob, np.uint8).copy()
    cid2 = server.admit_blob(glc.U64, host_blob.ctypes.data, len(blob), host=True)
    out.zero_()
    torch.cuda.synchronize()
    r[0]["column"] = cid2
    torch.cuda.synchronize()
    server.submit(r)
    server.drain(10_000)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), v)
    assert server.columns() == [cid2]
    server.close()


def test_arrivals_out_of_submission_order():
    """Requests submitted out of arrival order are scheduled by arrival time (not before it) and
    all complete with the right values."""
    ctx = glc.Context(0)
    server = glc.Server(ctx, budget_bytes=1 << 32, slots=2)
    cols = _columns(ctx, server, SPECS[:3])
    reqs = _mixed_requests(cols, 120, seed=21, big=30_000)
    _device_buffers(reqs)
    t0 = server.now_ns() + 5_000_000
    rng = np.random.default_rng(3)
    arrivals = t0 + rng.permutation(len(reqs)) * 100_000  # 0.1 ms apart, shuffled against submission
    torch.cuda.synchronize()
    for lo in range(0, len(reqs), 17):  # several submissions, each out of order
        part = reqs[lo:lo + 17]
        server.submit(_as_array(part, arrivals[lo:lo + 17]))
    server.drain(60_000)
    recs = server.poll()
    assert len(recs) == len(reqs) and np.all(recs["status"] == glc.OK)
    for r, g in zip(reqs, _results(reqs)):
        assert np.array_equal(g, r["want"])
    by_tag = {int(c["tag"]): c for c in recs}
    for r in reqs:
        assert by_tag[r["tag"]]["arrival_ns"] == arrivals[r["tag"]]
        assert by_tag[r["tag"]]["done_ns"] > arrivals[r["tag"]]
    server.close()
