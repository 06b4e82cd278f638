"""Batches of many columns per launch (glc_batch_*), checked against the single-column path.

A column compressed in a batch must serialize to the same bytes as glc_compress of the same
values with the same fixed partition length (and therefore match the oracle); the one-launch
batched decode, plain and replayed from a CUDA graph, must return every column exactly.
"""
import numpy as np
import pytest
import torch

import glc

pytestmark = pytest.mark.gpu

DT = {glc.I32: (np.int32, torch.int32), glc.I64: (np.int64, torch.int64), glc.U64: (np.uint64, torch.int64),
      glc.U32: (np.uint32, torch.int32)}


def _columns(ncols, seed=0, max_len=300_000):
    rng = np.random.default_rng(seed)
    cols = []
    for c in range(ncols):
        dt = [glc.I32, glc.I64, glc.U64, glc.U32][c % 4]
        n = int(rng.choice([0, 1, 7, 128, 4095, 4096, 4097, int(rng.integers(1, max_len))]))
        i = np.arange(n, dtype=np.int64)
        w = int(rng.integers(0, 21))
        noise = rng.integers(0, 1 << w, n) if w else np.zeros(n, np.int64)
        if dt in (glc.I32, glc.U32):
            slope = int(rng.integers(0, 400))
            v = (int(rng.integers(0, 1 << 20)) + slope * i + noise) % (1 << 31)
            if c % 13 in (5, 8):  # unpredictable values: fields of 32-33 bits (the wide-field packing)
                v = rng.integers(0, 1 << 31, n)
        else:
            slope = int(rng.integers(0, 10_000))
            v = int(rng.integers(0, 1 << 40)) + slope * i + noise
            if c % 11 == 0 and dt == glc.U64 and n > 5:  # some values above 2^53: direct copy
                v = v + (1 << 60)
        cols.append((dt, v.astype(DT[dt][0])))
    return cols


def _to_device(values):
    return torch.from_numpy(values.view(np.int64) if values.dtype.itemsize == 8 else values.view(np.int32)).cuda()


@pytest.mark.parametrize("fixed_len", [0, 1024, 4096, 3000])
def test_batch_compress_matches_single_column(oracle, fixed_len):
    ctx = glc.Context(0)
    cols = _columns(40, seed=fixed_len)
    dev = [_to_device(v) for _, v in cols]
    batch = glc.Batch.compress(ctx, [d for d, _ in cols], [t.data_ptr() for t in dev], [len(v) for _, v in cols],
                               fixed_len=fixed_len)
    total = 0
    for (dt, v), bc in zip(cols, batch.columns):
        info = bc.info()
        assert info.total_values == len(v)
        L = info.fixed_partition_len
        if fixed_len:
            assert L == fixed_len
        else:
            assert L in (1024, 2048, 4096)
        if len(v) == 0:
            continue
        total += info.compressed_size_bytes
        if not fixed_len:  # the chosen length is the first of 1024 / 2048 / 4096 with the smallest size
            sizes = []
            for cand in (1024, 2048, 4096):
                sc = glc.compress_device(ctx, dt, v.ctypes.data, len(v), glc.FIXED, fixed_len=cand, host=True)
                sizes.append(sc.info().compressed_size_bytes)
                sc.free()
            assert L == (1024, 2048, 4096)[int(np.argmin(sizes))], (L, sizes)
        single = glc.compress_device(ctx, dt, v.ctypes.data, len(v), glc.FIXED, fixed_len=L, host=True)
        blob = glc.serialize_host(ctx, bc)
        assert blob == glc.serialize_host(ctx, single)
        assert blob == oracle.serialize(oracle.compress(v, "fixed", L))
        single.free()
    assert batch.compressed_size == total
    batch.free()


def _mode_columns(n=150_001, seed=5):
    """Columns whose residuals take each arithmetic form of the compress kernels: predictions
    above 2^51 (nanosecond timestamps), non-positive lines, lines through zero, uint64 values at
    and just above 2^53 (tiles kept in the line form and tiles copied), 32-bit extremes."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    ns = (1_700_000_000_000_000_000 + np.cumsum(rng.integers(900_000, 1_100_000, n))).astype(np.int64)
    down = (-10 ** 12 - np.cumsum(rng.integers(0, 100_000, n))).astype(np.int64)
    cross = (-(n // 2) * 37 + 37 * i + rng.integers(-300, 300, n)).astype(np.int64)
    edge = (np.uint64(2 ** 53) - np.uint64(n)) + i.astype(np.uint64) * np.uint64(2)
    edge[:4096] = np.minimum(edge[:4096], np.uint64(2 ** 53))
    edge[4095] = np.uint64(2 ** 53)
    high = (np.uint64(1) << np.uint64(51)) + i.astype(np.uint64) * np.uint64(1_000_003)
    i32 = rng.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, dtype=np.int64).astype(np.int32)
    u32 = (np.uint32(0xFFFFFFF0) - (i % 7).astype(np.uint32)).astype(np.uint32)
    return [(glc.I64, ns), (glc.I64, down), (glc.I64, cross), (glc.U64, edge), (glc.U64, high), (glc.I32, i32),
            (glc.U32, u32), (glc.U64, ns.view(np.uint64)), (glc.I64, cross[: 4096 * 3 + 11])]


@pytest.mark.parametrize("fixed_len", [0, 4096, 256])
def test_batch_compress_residual_forms(oracle, fixed_len):
    ctx = glc.Context(0)
    cols = _mode_columns()
    dev = [_to_device(v) for _, v in cols]
    batch = glc.Batch.compress(ctx, [d for d, _ in cols], [t.data_ptr() for t in dev], [len(v) for _, v in cols],
                               fixed_len=fixed_len)
    for (dt, v), bc in zip(cols, batch.columns):
        L = bc.info().fixed_partition_len
        if not fixed_len:
            sizes = [oracle.compress(v, "fixed", cand).reported_size() for cand in (1024, 2048, 4096)]
            assert L == (1024, 2048, 4096)[int(np.argmin(sizes))], (L, sizes)
        assert glc.serialize_host(ctx, bc) == oracle.serialize(oracle.compress(v, "fixed", L))
    batch.free()


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_decode(use_graph):
    ctx = glc.Context(0)
    cols = _columns(60, seed=7)
    dev = [_to_device(v) for _, v in cols]
    batch = glc.Batch.compress(ctx, [d for d, _ in cols], [t.data_ptr() for t in dev], [len(v) for _, v in cols])
    outs = [torch.full((max(len(v), 1) + 4,), -1, dtype=DT[dt][1], device="cuda:0") for dt, v in cols]
    for rep in range(3):  # replays of the same graph / launch
        for o in outs:
            o.fill_(-1)
        torch.cuda.synchronize()  # the library runs on its own stream
        batch.decompress([o.data_ptr() for o in outs], use_graph=use_graph)
        ctx.sync()
        torch.cuda.synchronize()
        for (dt, v), o in zip(cols, outs):
            got = o.cpu().numpy().view(DT[dt][0])[: len(v)]
            assert np.array_equal(got, v), (rep, dt, len(v))
    # new outputs rebuild the work list (and the graph)
    outs2 = [torch.zeros(max(len(v), 1), dtype=DT[dt][1], device="cuda:0") for dt, v in cols]
    torch.cuda.synchronize()
    batch.decompress([o.data_ptr() for o in outs2], use_graph=use_graph)
    torch.cuda.synchronize()
    for (dt, v), o in zip(cols, outs2):
        assert np.array_equal(o.cpu().numpy().view(DT[dt][0])[: len(v)], v)
    batch.free()


def test_batch_over_existing_columns():
    ctx = glc.Context(0)
    cols = _columns(12, seed=3)
    singles = [glc.compress_device(ctx, dt, v.ctypes.data, len(v), glc.VARIABLE, host=True) for dt, v in cols]
    batch = glc.Batch.of(ctx, singles)
    outs = [torch.zeros(max(len(v), 1), dtype=DT[dt][1], device="cuda:0") for dt, v in cols]
    torch.cuda.synchronize()
    batch.decompress([o.data_ptr() for o in outs], use_graph=True)
    torch.cuda.synchronize()
    for (dt, v), o in zip(cols, outs):
        assert np.array_equal(o.cpu().numpy().view(DT[dt][0])[: len(v)], v)
    batch.free()
    for s in singles:
        s.free()


def test_batch_column_random_access_and_range():
    ctx = glc.Context(0)
    cols = _columns(8, seed=11)
    dev = [_to_device(v) for _, v in cols]
    batch = glc.Batch.compress(ctx, [d for d, _ in cols], [t.data_ptr() for t in dev], [len(v) for _, v in cols])
    for (dt, v), bc in zip(cols, batch.columns):
        if len(v) == 0:
            continue
        pos = np.random.default_rng(1).integers(0, len(v), 1000).astype(np.int32)
        out = np.zeros(len(pos), DT[dt][0])
        torch.cuda.synchronize()
        glc.random_access_into(ctx, bc, pos.ctypes.data, len(pos), out.ctypes.data, host_in=True, host_out=True)
        assert np.array_equal(out, v[pos])
        first = len(v) // 3
        r = np.zeros(len(v) - first, DT[dt][0])
        torch.cuda.synchronize()
        glc.decompress_range_into(ctx, bc, first, len(r), r.ctypes.data, host_out=True)
        assert np.array_equal(r, v[first:])
    with pytest.raises(glc.GlcError):
        ctx.check(ctx.lib.glc_column_free(batch.columns[0].handle))  # owned by the batch
    batch.free()


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_recompress_new_values(oracle, use_graph):
    """glc_batch_recompress: new values for the same columns, each at the length the batch chose;
    after glc_batch_sync every column equals glc_compress of the new values at that length, and the
    batched decode returns them.  With a CUDA graph the second call replays the first's capture on
    other values written into the same device buffers."""
    ctx = glc.Context(0)
    cols = _columns(24, seed=5)
    dev = [_to_device(v) for _, v in cols]
    batch = glc.Batch.compress(ctx, [d for d, _ in cols], [t.data_ptr() for t in dev], [len(v) for _, v in cols],
                               fixed_len=0)
    lens = [bc.info().fixed_partition_len for bc in batch.columns]
    for round_ in range(2):
        fresh = _columns(24, seed=100 + round_)
        for (dt, v), (_, w), t in zip(cols, fresh, dev):  # the same sizes, other values, same buffers
            w = np.resize(w, len(v)).astype(v.dtype) if len(v) else v
            t.copy_(_to_device(w))
        torch.cuda.synchronize()
        batch.recompress([t.data_ptr() for t in dev], use_graph=use_graph)
        total = batch.sync()
        want_total = 0
        outs = []
        for (dt, v), t, bc, L in zip(cols, dev, batch.columns, lens):
            host = t.cpu().numpy().view(v.dtype)
            if len(v) == 0:
                outs.append(torch.zeros(16, dtype=torch.uint8, device="cuda:0"))
                continue
            info = bc.info()
            assert info.fixed_partition_len == L
            single = glc.compress_device(ctx, dt, host.ctypes.data, len(host), glc.FIXED, fixed_len=L, host=True)
            assert glc.serialize_host(ctx, bc) == glc.serialize_host(ctx, single)
            assert info.compressed_size_bytes == single.info().compressed_size_bytes
            want_total += info.compressed_size_bytes
            single.free()
            outs.append(torch.zeros(len(v) + 8, dtype=DT[dt][1], device="cuda:0"))
        assert total == want_total
        torch.cuda.synchronize()
        batch.decompress([o.data_ptr() for o in outs], use_graph=use_graph)
        ctx.sync()
        for (dt, v), t, o in zip(cols, dev, outs):
            if len(v):
                assert torch.equal(o[:len(v)], t)
    # the last recompress against the oracle, column by column
    for (dt, v), t, bc, L in zip(cols, dev, batch.columns, lens):
        if len(v):
            host = t.cpu().numpy().view(v.dtype)
            assert glc.serialize_host(ctx, bc) == oracle.serialize(oracle.compress(host, "fixed", L))
    batch.free()
