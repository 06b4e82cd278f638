"""Parity of the CUDA path (through the C ABI) with the CPU oracle, bit for bit.

Every compressed column made on the GPU is serialized and compared byte for byte with the
oracle's blob for the same input: that covers partition boundaries, theta, bit widths, bit
offsets, error bounds and every packed word.  Decoders are compared with the input (round trip)
and with the oracle's decode of the same column.
"""
import numpy as np
import pytest

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu


def _data(kind: str, n: int, seed: int = 1):
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    if kind == "i32_linear":
        return (1000 * i + rng.integers(0, 256, n)).astype(np.int32)
    if kind == "i32_neg":
        return (-37 * i + rng.integers(-5000, 5000, n)).astype(np.int32)
    if kind == "i64_walk":
        return np.cumsum(rng.integers(-1000, 100000, n), dtype=np.int64)
    if kind == "i64_extreme":
        v = rng.integers(-(2 ** 62), 2 ** 62, n, dtype=np.int64)
        v[:: 7] = np.iinfo(np.int64).max
        v[3:: 11] = np.iinfo(np.int64).min
        return v
    if kind == "u64_piecewise":
        return W.piecewise_linear(n, seed=seed, mean_segment=5000)
    if kind == "u64_big":  # values above 2^53 in some partitions -> direct copy
        v = (np.uint64(1) << np.uint64(40)) + i.astype(np.uint64) * np.uint64(3)
        hi = (np.uint64(1) << np.uint64(60)) + rng.integers(0, 1 << 20, n).astype(np.uint64)
        sel = (i // 3000) % 3 == 1
        v[sel] = hi[sel]
        return v
    if kind == "u32_noise":
        return (i * 50 + rng.integers(0, 1 << 12, n)).astype(np.uint32)
    if kind == "u32_const":
        return np.full(n, 123456789, np.uint32)
    if kind == "timestamps":
        return W.timestamps(n, seed=seed)
    if kind == "i32_extreme":  # residuals near +-2^32: 33-bit fields in a 4-byte type
        v = rng.integers(-(2 ** 31), 2 ** 31, n, dtype=np.int64).astype(np.int32)
        v[:: 5] = np.iinfo(np.int32).max
        v[2:: 5] = np.iinfo(np.int32).min
        return v
    if kind == "i64_runs":  # runs of whole constant tiles between noisy ones: tiles without bits,
        # and tile boundaries in the middle of a word (odd widths)
        v = np.zeros(n, np.int64)
        pos = 0
        while pos < n:
            run = int(rng.integers(1, 4)) * 4096 + int(rng.integers(0, 3)) * 1024
            if rng.random() < 0.5:
                v[pos:pos + run] = rng.integers(-10 ** 12, 10 ** 12)
            else:
                w = int(rng.choice([1, 3, 5, 7, 13]))
                seg = v[pos:pos + run]
                v[pos:pos + run] = 12345 * np.arange(len(seg)) + rng.integers(0, 1 << w, len(seg))
            pos += run
        return v
    if kind == "i64_ns":  # nanosecond timestamps near 2^60: predictions far above 2^51 (offset residuals)
        return (1_700_000_000_000_000_000 + np.cumsum(rng.integers(900_000, 1_100_000, n))).astype(np.int64)
    if kind == "u64_high":  # a smooth line in [2^51, 2^52]
        return ((np.uint64(1) << np.uint64(51)) + i.astype(np.uint64) * np.uint64(1_000_003)
                + rng.integers(0, 1 << 16, n).astype(np.uint64))
    if kind == "u64_2p53":  # values across 2^53: some tiles hold 2^53 itself (not copied), some 2^53 + 1 (copied)
        v = (np.uint64(2 ** 53) - np.uint64(n)) + i.astype(np.uint64) * np.uint64(2)
        for t0 in range(0, n, 4096 * 3):
            v[t0:t0 + 4096] = np.minimum(v[t0:t0 + 4096], np.uint64(2 ** 53))
            v[min(t0 + 4095, n - 1)] = np.uint64(2 ** 53)
        return v
    if kind == "i64_negwalk":  # a falling line of negative values (non-positive predictions)
        return (-10 ** 12 - np.cumsum(rng.integers(0, 100_000, n))).astype(np.int64)
    if kind == "i64_cross":  # lines crossing zero
        return (-(n // 2) * 37 + 37 * i + rng.integers(-300, 300, n)).astype(np.int64)
    if kind == "u32_extreme":
        v = rng.integers(0, 2 ** 32, n, dtype=np.int64).astype(np.uint32)
        v[:: 3] = np.iinfo(np.uint32).max
        v[1:: 3] = 0
        return v
    raise ValueError(kind)


KINDS = ["i32_linear", "i32_neg", "i64_walk", "i64_extreme", "u64_piecewise", "u64_big", "u32_noise", "u32_const",
         "timestamps", "i64_runs", "i64_ns", "u64_high", "u64_2p53", "i64_negwalk", "i64_cross"]


def _codec(values):
    return glc.LeCoGPU(values.dtype, device=0)


def _check_column(codec, col, values, oracle_col, oracle):
    blob = codec.serialize(col)
    assert blob == oracle.serialize(oracle_col), "device column differs from the oracle's"
    out = codec.decompressFullFile(col)
    assert np.array_equal(out, values)
    return blob


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n,L", [(100_003, 1024), (65_536, 4096), (5_000, 128), (777, 1000), (20_000, 6000),
                                 (50_001, 10_000),
                                 # lengths that divide the 4096-value tile (>= 256): the one-pass kernel
                                 (1, 4096), (255, 256), (4_097, 256), (300_001, 512), (123_457, 2048),
                                 (4096 * 37 + 5, 4096), (1 << 20, 1024)])
def test_fixed_compress_bit_exact(oracle, kind, n, L):
    v = _data(kind, n)
    codec = _codec(v)
    col, size = codec.compress(v, False, fixed_partition_size=L)
    ocol = oracle.compress(v, "fixed", L)
    assert size == ocol.reported_size()
    _check_column(codec, col, v, ocol, oracle)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 100, 128, 129, 4_000, 50_001, 300_000])
def test_variable_compress_bit_exact(oracle, kind, n):
    v = _data(kind, n, seed=n)
    codec = _codec(v)
    col, size = codec.compress(v, True)
    s, e = oracle.partition_variable(v)
    ocol = oracle.compress(v, starts=s, ends=e)
    assert col.num_partitions == len(s)
    assert size == ocol.reported_size()
    _check_column(codec, col, v, ocol, oracle)


@pytest.mark.parametrize("kind", ["timestamps", "i32_linear", "u64_piecewise", "u64_high", "i64_ns", "i64_cross"])
def test_variable_walks_over_many_ranges(oracle, kind):
    """1.5M values span 6 ranges of 2048 blocks of the split walk: lines without slope changes
    (the ranges' walks never meet, so every start is evaluated), piecewise lines (only the starts
    the walks visit), and values beyond 2^51 (the walks' offset form)."""
    v = _data(kind, 1_500_000, seed=7)
    codec = _codec(v)
    col, size = codec.compress(v, True)
    s, e = oracle.partition_variable(v)
    ocol = oracle.compress(v, starts=s, ends=e)
    assert col.num_partitions == len(s)
    assert size == ocol.reported_size()
    _check_column(codec, col, v, ocol, oracle)


def test_partitioner_matches_oracle_large(oracle, glc_ctx):
    v = W.piecewise_linear(3_000_000, seed=5)
    ds, de = glc.partition_variable(glc_ctx, v)
    s, e = oracle.partition_variable(v)
    assert np.array_equal(ds, s) and np.array_equal(de, e)


@pytest.mark.parametrize("kind", ["i32_linear", "i64_walk", "u64_piecewise", "u32_noise", "u64_big"])
def test_random_access(oracle, kind):
    n = 200_000
    v = _data(kind, n)
    codec = _codec(v)
    rng = np.random.default_rng(3)
    pos = np.concatenate([rng.integers(0, n, 50_000), [0, n - 1, 1, n - 2, 4095, 4096, 4097]]).astype(np.int32)
    for variable in (False, True):
        col, _ = codec.compress(v, variable, fixed_partition_size=4096)
        assert np.array_equal(codec.decompress(col, pos), v[pos])
        if not variable:
            assert np.array_equal(codec.randomAccessFixed(col, pos, 4096), v[pos])
        glc.preunpack(codec.ctx, col)
        assert np.array_equal(codec.randomAccessPreUnpacked(col, pos), v[pos])
        assert np.array_equal(codec.decompressFullFile_PreUnpacked(col), v)
        if not variable:
            assert np.array_equal(codec.randomAccessFixedPreUnpacked(col, pos, 4096), v[pos])


def test_random_access_outside_is_zero():
    v = _data("i64_walk", 10_000)
    codec = _codec(v)
    col, _ = codec.compress(v, False, fixed_partition_size=1024)
    pos = np.array([-1, 10_000, 2 ** 31 - 1, -(2 ** 31), 5], np.int32)
    out = codec.decompress(col, pos)
    assert list(out[:4]) == [0, 0, 0, 0] and out[4] == v[5]
    out = codec.randomAccessFixed(col, pos, 1024)
    assert list(out[:4]) == [0, 0, 0, 0] and out[4] == v[5]


def test_fixed_length_mismatch_is_an_error():
    v = _data("i32_linear", 10_000)
    codec = _codec(v)
    col, _ = codec.compress(v, False, fixed_partition_size=1024)
    with pytest.raises(glc.GlcError):
        codec.randomAccessFixed(col, np.arange(10, dtype=np.int32), 4096)


@pytest.mark.parametrize("kind", ["i32_extreme", "u32_extreme", "i64_extreme"])
@pytest.mark.parametrize("L", [100, 108, 1000, 4096])
def test_widest_fields_each_packer(oracle, kind, L):
    """Fields as wide as the type allows (33 bits for 4-byte types, 64 for 8-byte ones), with
    partitions short enough for the output-word packer (100) and long enough for the value-tile
    packer (108 and up)."""
    v = _data(kind, 20_001, seed=L)
    codec = _codec(v)
    col, size = codec.compress(v, False, fixed_partition_size=L)
    ocol = oracle.compress(v, "fixed", L)
    assert size == ocol.reported_size()
    _check_column(codec, col, v, ocol, oracle)


@pytest.mark.parametrize("mode", ["fixed", "variable"])
@pytest.mark.parametrize("skip", [1, 2, 3])
def test_compress_from_unaligned_device_values(oracle, glc_ctx, mode, skip):
    """Device input that starts 8, 16 or 24 bytes into a buffer (not 16-byte aligned in two cases):
    the staged bulk copies start on the enclosing 16-byte boundary and skip the head."""
    import torch
    v = _data("u64_piecewise", 30_000 + skip, seed=skip)
    d = torch.from_numpy(v.view(np.int64)).cuda()
    sub = v[skip:]
    col = glc.compress_device(glc_ctx, glc.U64, d.data_ptr() + 8 * skip, len(sub),
                              glc.FIXED if mode == "fixed" else glc.VARIABLE, fixed_len=1024)
    ocol = oracle.compress(sub, mode, 1024)
    assert glc.serialize_host(glc_ctx, col) == oracle.serialize(ocol)
    col.free()


@pytest.mark.parametrize("L", [1, 3, 7, 64])
def test_tiny_partitions(oracle, L):
    """More partitions per decode tile than the shared-memory descriptor cache holds."""
    v = _data("i64_walk", 20_000)
    codec = _codec(v)
    col, _ = codec.compress(v, False, fixed_partition_size=L)
    ocol = oracle.compress(v, "fixed", L)
    _check_column(codec, col, v, ocol, oracle)
    pos = np.random.default_rng(0).integers(0, len(v), 5000).astype(np.int32)
    assert np.array_equal(codec.decompress(col, pos), v[pos])


@pytest.mark.parametrize("kind", ["i32_linear", "u64_piecewise", "i64_extreme"])
def test_range_decode(oracle, kind, glc_ctx):
    n = 123_457
    v = _data(kind, n)
    codec = _codec(v)
    col, _ = codec.compress(v, True)
    rng = np.random.default_rng(9)
    cases = [(0, n), (1, 1), (4095, 2), (4096, 4096), (n - 1, 1), (17, 40_000)]
    cases += [(int(a), int(rng.integers(1, n - a))) for a in rng.integers(0, n - 1, 20)]
    for first, count in cases:
        out = np.empty(count, v.dtype)
        glc.decompress_range_into(codec.ctx, col, first, count, out.ctypes.data, host_out=True)
        assert np.array_equal(out, v[first:first + count]), (first, count)


def test_empty_column():
    codec = glc.LeCoGPU(np.int64, device=0)
    col, size = codec.compress(np.zeros(0, np.int64), False)
    assert size == 0 and col.total_values == 0
    assert codec.decompressFullFile(col).shape == (0,)
    assert codec.decompress(col, np.array([0, 1], np.int32)).tolist() == [0, 0]


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.uint64, np.uint32])
def test_prediction_ties(oracle, dtype):
    """Predictions landing exactly on .5 round half away from zero in every decoder."""
    n = 6000
    i = np.arange(n)
    rng = np.random.default_rng(2)
    base = (i + 1) if np.dtype(dtype).kind == "u" else (i - 3000)
    v = (base + rng.integers(-3, 4, n)).astype(dtype)
    if np.dtype(dtype).kind == "u":
        v = np.maximum(v.astype(np.int64), 0).astype(dtype)
    starts, ends = np.array([0, 3000], np.int32), np.array([3000, n], np.int32)
    # theta0 = 0.5 / -0.5 with theta1 = 1: every prediction is an exact .5 tie
    ocol = oracle.column_with_lines(v, starts, ends, [(0.5, 1.0), (-0.5, 1.0)])
    assert np.array_equal(oracle.decode_full(ocol), v)
    codec = glc.LeCoGPU(dtype, device=0)
    col = codec.deserialize(oracle.serialize(ocol))
    assert col is not None
    assert np.array_equal(codec.decompressFullFile(col), v)
    pos = rng.integers(0, n, 3000).astype(np.int32)
    assert np.array_equal(codec.decompress(col, pos), v[pos])
    glc.preunpack(codec.ctx, col)
    assert np.array_equal(codec.decompressFullFile_PreUnpacked(col), v)
    assert np.array_equal(codec.randomAccessPreUnpacked(col, pos), v[pos])


@pytest.mark.parametrize("kind", ["u64_piecewise", "i32_linear", "u64_big"])
def test_serialize_roundtrip_and_oracle_blobs(oracle, kind):
    v = _data(kind, 80_000)
    codec = _codec(v)
    ocol = oracle.compress(v, "fixed", 2048)
    blob = oracle.serialize(ocol)
    col = codec.deserialize(blob)
    assert np.array_equal(codec.decompressFullFile(col), v)
    assert codec.serialize(col) == blob
    col2 = codec.deserializeGPU(blob, True)  # pre-unpacked, bitstream dropped
    assert np.array_equal(codec.decompressFullFile(col2), v)
    with pytest.raises(glc.GlcError):
        codec.serialize(col2)  # api/G-LeCo.cuh:2005-2011
    crc = oracle.serialize(ocol, crc32c=True)
    assert codec.deserialize(crc) is None
    assert np.array_equal(codec.decompressFullFile(codec.deserialize(crc, crc32c=True)), v)


def test_bad_blobs_rejected(oracle):
    v = _data("i32_linear", 10_000)
    codec = _codec(v)
    blob = bytearray(oracle.serialize(oracle.compress(v, "fixed", 1024)))
    assert codec.deserialize(bytes(blob[:100])) is None                     # short
    for off in (0, 4, 96, 112):                                             # magic, version, type size, reserved
        b = bytearray(blob)
        b[off] ^= 0x07
        assert codec.deserialize(bytes(b)) is None
    b = bytearray(blob)
    b[20] ^= 1                                                               # header byte -> checksum
    assert codec.deserialize(bytes(b)) is None
    assert codec.deserialize(bytes(blob[:-16])) is None                     # truncated bitstream
    assert glc.LeCoGPU(np.int64, device=0).deserialize(bytes(blob)) is None  # wrong element type


@pytest.mark.parametrize("n", [2_000_000])
def test_piecewise_scale_roundtrip(oracle, n):
    """Size-independent properties on a larger piecewise-linear column."""
    v = W.piecewise_linear(n, seed=11)
    codec = _codec(v)
    col, size = codec.compress(v, True)
    assert np.array_equal(codec.decompressFullFile(col), v)
    s, e = oracle.ref_partition_cpu(v)
    ref_size = oracle.compress(v, starts=s, ends=e).reported_size()
    assert size <= ref_size * 1.01, (size, ref_size)


def test_c1_plain_config(oracle):
    """The plain small workload at its stated size: 1,048,576 int32 v[i] = 1000 i + U{0..255}
    (seed 42), fixed partitions of 1024: the device blob equals the oracle's byte for byte, the
    full decode and 10,000 uniform lookups (fixed-length and binary-search paths) are exact, and
    the variable partitioning stays within 1% of the size of the reference partitioner's layout."""
    v = W.plain_small(1 << 20, seed=42)
    codec = _codec(v)
    col, size = codec.compress(v, False, fixed_partition_size=1024)
    ocol = oracle.compress(v, "fixed", 1024)
    assert size == ocol.reported_size() and col.info().num_partitions == 1024
    assert codec.serialize(col) == oracle.serialize(ocol)
    assert np.array_equal(codec.decompressFullFile(col), v)
    pos = np.random.default_rng(42).integers(0, len(v), 10_000).astype(np.int32)
    assert np.array_equal(codec.randomAccessFixed(col, pos, 1024), v[pos])
    assert np.array_equal(codec.decompress(col, pos), v[pos])
    vcol, vsize = codec.compress(v, True)
    assert np.array_equal(codec.decompressFullFile(vcol), v)
    s, e = oracle.ref_partition_cpu(v)
    assert vsize <= 1.01 * oracle.compress(v, starts=s, ends=e).reported_size()


def test_cpp_dropin_caller():
    """A C++ caller written against the reference's LeCoGPU<T> API runs on include/glc_leco.hpp."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "g-leco_b200", "_build",
                       "leco_dropin")
    if not os.path.exists(exe):
        pytest.fail("drop-in caller not built (run __graft_entry__.build())")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(": ok") == 6 and "MISMATCH" not in r.stdout, r.stdout


@pytest.mark.parametrize("offset_bytes", [4, 8, 12])
def test_decode_into_misaligned_device_buffer(offset_bytes):
    """Device outputs that are not 16-byte aligned are still written exactly."""
    import torch
    v = _data("i32_linear", 50_000)
    codec = _codec(v)
    col, _ = codec.compress(v, True)
    buf = torch.zeros(len(v) + 8, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()  # the library runs on its own stream
    ptr = buf.data_ptr() + offset_bytes
    glc.decompress_into(codec.ctx, col, ptr, glc.SRC_PACKED)
    glc.decompress_range_into(codec.ctx, col, 3, 1000, ptr, glc.SRC_PACKED)
    torch.cuda.synchronize()
    codec.ctx.sync()
    got = buf.cpu().numpy()[offset_bytes // 4: offset_bytes // 4 + len(v)]
    want = v.copy()
    want[:1000] = v[3:1003]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("kind,n", [("u64_piecewise", 0), ("u64_piecewise", 1), ("i32_linear", 70_001),
                                    ("u64_piecewise", 20_000_000), ("i32_linear", 40_000_000),
                                    ("u64_big", 300_000)])
def test_streaming_blob_decode_to_host(oracle, kind, n):
    """glc_decode_blob_to_host: host blob in, host values out, chunks overlapped on three streams;
    the same values as deserialize + full decode, and the kept column works afterwards."""
    import torch
    v = _data(kind, n) if n else np.zeros(0, _data(kind, 10).dtype)
    dt = glc.DTYPE_OF[v.dtype]
    codec = _codec(v) if n else glc.LeCoGPU(v.dtype)
    if n:
        col, _ = codec.compress(v, True)
        blob = glc.serialize_host(codec.ctx, col)
        col.free()
    else:
        blob = oracle.serialize(oracle.compress(v, "fixed", 4096))
    hb = torch.from_numpy(np.frombuffer(blob, np.uint8).copy()).pin_memory()
    out = torch.empty(max(n, 1) * v.dtype.itemsize, dtype=torch.uint8).pin_memory()
    out.fill_(0xAB)
    glc.decode_blob_to_host(codec.ctx, dt, hb.data_ptr(), len(blob), out.data_ptr())
    assert np.array_equal(out.numpy()[: n * v.dtype.itemsize].view(v.dtype), v)
    kept = glc.decode_blob_to_host(codec.ctx, dt, hb.data_ptr(), len(blob), 0, keep=True)
    if n:
        pos = np.random.default_rng(2).integers(0, n, 10_000).astype(np.int32)
        got = np.zeros(len(pos), v.dtype)
        glc.random_access_into(codec.ctx, kept, pos.ctypes.data, len(pos), got.ctypes.data, host_in=True,
                               host_out=True)
        assert np.array_equal(got, v[pos])
    kept.free()
    bad = np.frombuffer(blob, np.uint8).copy()  # kept alive across the call
    bad[8] ^= 1
    with pytest.raises(glc.GlcError):
        glc.decode_blob_to_host(codec.ctx, dt, bad.ctypes.data, len(bad), out.data_ptr())


@pytest.mark.parametrize("n", [524_288, 4_194_305, 12_500_001])
def test_large_pageable_host_buffers(n):
    """Host (pageable) buffers of several MB go through the context's pinned chunks: compress from
    host memory, decode into host memory (also at an odd offset), random access with host positions
    and outputs, and a host blob round trip all return the input."""
    v = _data("u64_piecewise", n)
    codec = _codec(v)
    col, _ = codec.compress(v, True)
    assert np.array_equal(codec.decompressFullFile(col), v)
    buf = np.zeros(n + 1, np.uint64)
    glc.decompress_range_into(codec.ctx, col, 0, n, buf[1:].ctypes.data, glc.SRC_PACKED, host_out=True)
    assert np.array_equal(buf[1:], v) and buf[0] == 0
    pos = np.random.default_rng(3).integers(0, n, 2 * n).astype(np.int32)
    out = np.zeros(len(pos), np.uint64)
    glc.random_access_into(codec.ctx, col, pos.ctypes.data, len(pos), out.ctypes.data, host_in=True, host_out=True)
    assert np.array_equal(out, v[pos])
    blob = glc.serialize_host(codec.ctx, col)
    back = glc.deserialize_host(codec.ctx, glc.U64, blob)
    assert np.array_equal(codec.decompressFullFile(back), v)
    back.free()
    col.free()


def test_host_transfers_from_two_threads_on_one_context():
    """Two host threads share one context: their pageable transfers go through the same pinned
    chunks (one transfer at a time) and every result is still exact."""
    import threading
    ctx = glc.Context(0)
    cols = [_data("u64_piecewise", 9_000_001, seed=s) for s in (1, 2)]
    errors = []

    def work(v):
        try:
            for _ in range(3):
                col = glc.compress_device(ctx, glc.U64, v.ctypes.data, len(v), glc.VARIABLE, host=True)
                out = np.zeros(len(v), np.uint64)
                glc.decompress_into(ctx, col, out.ctypes.data, glc.SRC_PACKED, host_out=True)
                if not np.array_equal(out, v):
                    errors.append("mismatch")
                col.free()
        except Exception as ex:  # reported below
            errors.append(repr(ex))

    ts = [threading.Thread(target=work, args=(v,)) for v in cols]
    for t in ts:
        t.start()
    for t in ts:
        t.join(300)
    assert not errors, errors
