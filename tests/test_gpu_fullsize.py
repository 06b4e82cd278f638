"""Full-size workloads, checked through size-independent properties: every value round-trips
bit-exactly (compared on the device), lookups equal direct indexing, and the batched and
per-column paths agree; the 200M decode-benchmark column's blobs also equal the oracle's (SHA-256
digests in tests/golden/c2_oracle_blobs.json, made by tests/golden/make_c2_oracle_blobs.py).
Inputs are generated on the device with the workloads' distributions."""
import hashlib
import json
import os

import numpy as np
import pytest
import torch

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu


def _ctx():
    return glc.Context(0)


def test_piecewise_u64_200m_variable_round_trip():
    """200M uint64 piecewise-linear values, device split/merge partitioner: exact round trip,
    range decodes at awkward offsets, and the blob re-reads to the same values."""
    ctx = _ctx()
    v = W.piecewise_linear(200_000_000, seed=42)
    d = torch.from_numpy(v.view(np.int64)).cuda()
    s = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    col = glc.compress_device(ctx, glc.U64, d.data_ptr(), len(v), glc.VARIABLE, stream=s)
    info = col.info()
    assert info.num_partitions > 1000 and info.compressed_size_bytes < len(v) * 8 // 4
    out = torch.empty_like(d)
    glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED, stream=s)
    torch.cuda.synchronize()
    assert torch.equal(out, d)
    for first, count in ((0, 1), (123_456_789, 4097), (199_999_000, 1000), (7, 10_000_001)):
        r = torch.empty(count + 2, dtype=torch.int64, device="cuda:0")
        glc.decompress_range_into(ctx, col, first, count, r.data_ptr() + 8, glc.SRC_PACKED, stream=s)
        torch.cuda.synchronize()
        assert torch.equal(r[1:count + 1], d[first:first + count])
    blob = glc.serialize_host(ctx, col)
    back = glc.deserialize_host(ctx, glc.U64, blob)
    out.zero_()
    torch.cuda.synchronize()
    glc.decompress_into(ctx, back, out.data_ptr(), glc.SRC_PACKED, stream=s)
    torch.cuda.synchronize()
    assert torch.equal(out, d)
    col.free()
    back.free()


@pytest.mark.parametrize("mode", ["variable", "fixed4096"])
def test_piecewise_u64_200m_blob_equals_oracle(mode):
    """The whole 200M-value blob of the decode benchmark's column (device partitioner and compress,
    or the one-pass fixed compress) is byte for byte the oracle's."""
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_oracle_blobs.json")) as f:
        fx = json.load(f)
    ctx = _ctx()
    v = W.piecewise_linear(fx["values"], seed=fx["seed"])
    d = torch.from_numpy(v.view(np.int64)).cuda()
    s = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    if mode == "variable":
        col = glc.compress_device(ctx, glc.U64, d.data_ptr(), len(v), glc.VARIABLE, stream=s)
    else:
        col = glc.compress_device(ctx, glc.U64, d.data_ptr(), len(v), glc.FIXED, fixed_len=4096, stream=s)
    ctx.sync()
    info = col.info()
    assert info.num_partitions == fx[mode]["partitions"]
    assert info.compressed_size_bytes == fx[mode]["reported_size"]
    blob = glc.serialize_host(ctx, col)
    col.free()
    assert len(blob) == fx[mode]["blob_bytes"]
    assert hashlib.sha256(blob).hexdigest() == fx[mode]["blob_sha256"]


@pytest.mark.parametrize("mode", ["packed", "preunpacked"])
def test_timestamps_64m_100m_lookups(mode):
    """64M int64 timestamps, fixed partitions of 4096, 100M positions (half uniform, half Zipf over
    partitions): every lookup equals direct indexing."""
    ctx = _ctx()
    n, q = 64 * 1024 * 1024, 100_000_000
    v = W.timestamps(n, seed=42)
    pos = W.lookup_positions(n, q, 4096, seed=42)
    dv = torch.from_numpy(v).cuda()
    dp = torch.from_numpy(pos).cuda()
    s = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    col = glc.compress_device(ctx, glc.I64, dv.data_ptr(), n, glc.FIXED, fixed_len=4096, stream=s)
    src = glc.SRC_PACKED
    if mode == "preunpacked":
        glc.preunpack(ctx, col, stream=s)
        src = glc.SRC_PREUNPACKED
    out = torch.empty(q, dtype=torch.int64, device="cuda:0")
    glc.random_access_into(ctx, col, dp.data_ptr(), q, out.data_ptr(), source=src, fixed_len=4096, stream=s)
    torch.cuda.synchronize()
    assert torch.equal(out, dv[dp.long()])
    col.free()


def test_batch_4096_columns_full_size():
    """4096 mixed columns (~2.5 GB raw): the batched compress + one-launch decode equals the input,
    and every column equals its per-column compression."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location("bench", os.path.join(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    ctx = _ctx()
    specs = bench.batch_columns(4096, 2.5e9)
    code = {0: glc.I32, 1: glc.I64, 2: glc.U64}
    cols = []
    gen = torch.Generator(device="cuda:0")
    for dt, n, slope, icpt, w, seed in specs:
        gen.manual_seed(seed)
        x = icpt + slope * torch.arange(n, device="cuda:0", dtype=torch.int64)
        if w:
            x = x + torch.randint(0, 1 << w, (n,), device="cuda:0", generator=gen, dtype=torch.int64)
        cols.append(x.to(torch.int32) if dt == 0 else x)
    torch.cuda.synchronize()
    batch = glc.Batch.compress(ctx, [code[s[0]] for s in specs], [c.data_ptr() for c in cols], [s[1] for s in specs])
    outs = [torch.empty_like(c) for c in cols]
    torch.cuda.synchronize()
    batch.decompress([o.data_ptr() for o in outs], use_graph=True)
    ctx.sync()
    torch.cuda.synchronize()
    assert all(torch.equal(o, c) for o, c in zip(outs, cols))
    # spot-check per-column equality of the compressed form on a sample of columns
    for i in range(0, 4096, 257):
        bc = batch.columns[i]
        L = bc.info().fixed_partition_len
        host = cols[i].cpu().numpy()
        if specs[i][0] == 2:
            host = host.view(np.uint64)
        single = glc.compress_device(ctx, code[specs[i][0]], host.ctypes.data, len(host), glc.FIXED, fixed_len=L,
                                     host=True)
        assert glc.serialize_host(ctx, bc) == glc.serialize_host(ctx, single)
        single.free()
    batch.free()


@pytest.mark.parametrize("dt,mode", [(glc.I32, glc.FIXED), (glc.I32, glc.VARIABLE), (glc.U64, glc.FIXED)])
def test_longest_column(dt, mode):
    """n = 2^31 - 1 values, the longest column int32 positions address: decode, a range at the end
    and lookups of the last positions.  The outputs carry 64 sentinel elements past their end,
    so a write past n would show instead of landing outside the allocation."""
    n = 2 ** 31 - 1
    ctx = _ctx()
    s = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda:0")
    g.manual_seed(5)
    tdt = torch.int32 if dt == glc.I32 else torch.int64
    v = torch.randint(0, 1 << 12, (n,), device="cuda:0", generator=g, dtype=torch.int64)
    v += torch.arange(n, device="cuda:0", dtype=torch.int64) >> 4
    v = v.to(tdt)
    torch.cuda.synchronize()
    col = glc.compress_device(ctx, dt, v.data_ptr(), n, mode, fixed_len=4096, stream=s)
    assert col.info().total_values == n
    pad = 64
    out = torch.full((n + pad,), -5, dtype=tdt, device="cuda:0")
    torch.cuda.synchronize()
    glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED, stream=s)
    ctx.sync()
    torch.cuda.synchronize()
    assert torch.equal(out[:n], v)
    assert bool((out[n:] == -5).all()), "write past the end of the output"
    del out
    r = torch.full((1000 + pad,), -5, dtype=tdt, device="cuda:0")
    torch.cuda.synchronize()
    glc.decompress_range_into(ctx, col, n - 1000, 1000, r.data_ptr(), glc.SRC_PACKED, stream=s)
    ctx.sync()
    torch.cuda.synchronize()
    assert torch.equal(r[:1000], v[n - 1000:]) and bool((r[1000:] == -5).all())
    pos = torch.arange(n - 5000, n, dtype=torch.int32, device="cuda:0")
    q = torch.empty(5000, dtype=tdt, device="cuda:0")
    torch.cuda.synchronize()
    glc.random_access_into(ctx, col, pos.data_ptr(), 5000, q.data_ptr(), stream=s)
    ctx.sync()
    torch.cuda.synchronize()
    assert torch.equal(q, v[n - 5000:])
    col.free()
