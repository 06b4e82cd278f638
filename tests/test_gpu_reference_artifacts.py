"""Parity of the CUDA path with the reference's own artefacts, on the GPU.

* Every blob in tests/golden/ was made by the reference's stock compress + serialize on a B200
  (tests/golden/make_golden.py).  Each goes through this library's device deserialize, full
  decode, range decode, random access (binary search and fixed length), the pre-unpacked
  deserialize with its full decode and random access, the streaming host decode, and serialize
  back to the same bytes.
* Blobs made by this library go through the reference's own GPU decoders and random access,
  compiled from the reference's sources (oracle/_ref/ref_harness gpudecode / gpura): no value
  may differ, except in randomAccessFixedPreUnpacked, which rounds ties to even
  (decompression/FixedPartitionKernels.cuh:204); its output must equal the oracle's restatement
  of that kernel exactly.
* The reference's host decoder directRandomAccessCPU (api/G-LeCo.cuh:1337-1672) on a 16M-value
  piecewise column made by this library: the values it gets wrong are exactly the positions where
  its prediction without fma rounds differently from the format's fma prediction, as the oracle
  predicts.
* Compressed-size parity at the full 200M-value size of the piecewise workload: this library's
  variable partitioning gives a size at most 1.01x the size the reference's own compress (CPU
  partitioner) reports for the same column (api/G-LeCo.cuh:589-603).
"""
import json
import os
import tempfile

import numpy as np
import pytest

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
NP = {glc.I32: np.int32, glc.I64: np.int64, glc.U64: np.uint64, glc.U32: np.uint32}
CODE = {"i32": glc.I32, "i64": glc.I64, "u64": glc.U64, "u32": glc.U32}
TWO_MB = 2 << 20


def _golden():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return sorted(json.load(f).items())


def _positions(n, starts, k, seed):
    rng = np.random.default_rng(seed)
    pos = np.concatenate([rng.integers(0, n, k), [0, n - 1], starts, np.maximum(0, starts - 1)])
    return np.clip(pos, 0, n - 1).astype(np.int32)


@pytest.mark.parametrize("name,meta", _golden(), ids=[g[0] for g in _golden()])
def test_reference_blob_through_device(oracle, name, meta):
    values = np.load(os.path.join(GOLDEN, f"{name}.values.npy"))
    with open(os.path.join(GOLDEN, f"{name}.blob"), "rb") as f:
        blob = f.read()
    n = len(values)
    codec = glc.LeCoGPU(values.dtype, device=0)
    col = codec.deserializeGPU(blob)
    assert col is not None
    info = col.info()
    assert info.total_values == n and info.compressed_size_bytes == meta["reported_size"]
    assert np.array_equal(codec.decompressFullFile(col), values)
    ocol = oracle.deserialize(blob, meta["dtype"])
    pos = _positions(n, ocol.starts, 20_000, 5)
    assert np.array_equal(codec.decompress(col, pos), values[pos])
    if meta["mode"] == "fixed":
        assert np.array_equal(codec.randomAccessFixed(col, pos, glc.TILE_SIZE), values[pos])
    a, b = n // 3, n // 3 + max(1, n // 2)
    out = np.zeros(b - a, values.dtype)
    glc.decompress_range_into(codec.ctx, col, a, b - a, out.ctypes.data, host_out=True)
    assert np.array_equal(out, values[a:b])
    # serialize gives back the reference's bytes
    assert codec.serialize(col) == blob
    # the pre-unpacked deserialize (deserializeGPU(blob, true), api/G-LeCo.cuh:2249-2288)
    cu = codec.deserializeGPU(blob, True)
    assert np.array_equal(codec.decompressFullFile_PreUnpacked(cu), values)
    assert np.array_equal(codec.randomAccessPreUnpacked(cu, pos), values[pos])
    if meta["mode"] == "fixed":
        assert np.array_equal(codec.randomAccessFixedPreUnpacked(cu, pos, glc.TILE_SIZE), values[pos])
    # the streaming host decode of the host blob
    hb = np.frombuffer(blob, np.uint8).copy()
    hout = np.zeros(n, values.dtype)
    glc.decode_blob_to_host(codec.ctx, CODE[meta["dtype"]], hb.ctypes.data, len(hb), hout.ctypes.data)
    assert np.array_equal(hout, values)
    cu.free()
    col.free()


def _device_columns():
    rng = np.random.default_rng(17)
    i = np.arange(3_000_000, dtype=np.int64)
    big = (np.uint64(1) << np.uint64(58)) + (i[:600_000].astype(np.uint64) * np.uint64(977))
    big[100_000:140_000] = rng.integers(0, 1 << 62, 40_000).astype(np.uint64)  # direct-copy partitions
    return [
        ("i32_plain_1M_fixed1024", W.plain_small(1 << 20, seed=42), glc.FIXED, 1024),
        ("i64_timestamps_fixed4096", W.timestamps(3_000_000, seed=5), glc.FIXED, 4096),
        ("u64_piecewise_variable", W.piecewise_linear(2_000_000, seed=9, mean_segment=20_000), glc.VARIABLE, 0),
        ("u32_noise_variable", (i[:1_500_000] * 37 + rng.integers(0, 1 << 10, 1_500_000)).astype(np.uint32),
         glc.VARIABLE, 0),
        ("i64_walk_variable", np.cumsum(rng.integers(-5000, 3000, 1_200_000), dtype=np.int64), glc.VARIABLE, 0),
        ("u64_direct_copy_fixed4096", big, glc.FIXED, 4096),
        ("i32_descending_fixed2048", (-7 * i[:900_000] + rng.integers(0, 64, 900_000)).astype(np.int32),
         glc.FIXED, 2048),
        ("u64_piecewise_v6", W.piecewise_linear(1_000_000, seed=21, mean_segment=9_000), glc.VARIABLE_V6, 0),
    ]


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built (make -C oracle ref)")
@pytest.mark.parametrize("name,values,mode,plen", _device_columns(), ids=[c[0] for c in _device_columns()])
def test_reference_gpu_decoders_read_device_blobs(oracle, name, values, mode, plen):
    codec = glc.LeCoGPU(values.dtype, device=0)
    col, _ = codec.compress(values, mode != glc.FIXED, use_gpu_partitioning=mode == glc.VARIABLE_V6,
                            fixed_partition_size=plen or glc.TILE_SIZE)
    info = col.info()
    # the reference's decoders read the word after a field; keep the bitstream's last word off a
    # 2 MB allocation boundary (the harness refuses such a blob)
    assert ((info.total_bits + 31) // 32 * 4) % TWO_MB != 0
    blob = codec.serialize(col)
    dt = oracle.NP_TO_CODE[values.dtype]
    with tempfile.TemporaryDirectory() as td:
        dec = oracle.ref_gpudecode(blob, values, dt, td)
        assert set(dec) == {"decompressFullFile_BitPacked", "decompressFullFile_OnTheFly_Optimized_V2",
                            "decompressFullFile_WorkStealingAdvanced", "decompressFullFile_PreUnpacked"}
        assert all(bad == 0 for _, bad in dec.values()), dec
        # random access: at most 1,212,416 positions (randomAccessPreUnpacked has no grid-stride loop)
        pos = _positions(len(values), np.zeros(0, np.int64), 400_000, 3)
        ra = oracle.ref_gpura(blob, values, pos, dt, plen, td)
    want = values[pos]
    assert np.array_equal(ra["decompress"], want)
    assert np.array_equal(ra["randomAccessPreUnpacked"], want)
    if plen:
        assert np.array_equal(ra["randomAccessFixed"], want)
        ocol = oracle.deserialize(blob, dt)
        assert np.array_equal(ra["randomAccessFixedPreUnpacked"],
                              oracle.decode_variant(ocol, pos, oracle.PRED_FIXED_PREUNPACKED))
    # and this library answers every position exactly
    assert np.array_equal(codec.decompress(col, pos), want)
    col.free()


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built (make -C oracle ref)")
def test_reference_host_decoder_mismatches_are_the_predicted_ties(oracle):
    values = W.piecewise_linear(16_000_000, seed=42)
    codec = glc.LeCoGPU(np.uint64, device=0)
    col, _ = codec.compress(values, True)
    blob = codec.serialize(col)
    with tempfile.TemporaryDirectory() as td:
        bp, vp, mp = (os.path.join(td, f) for f in ("b.bin", "v.bin", "m.bin"))
        with open(bp, "wb") as f:
            f.write(blob)
        values.tofile(vp)
        _, mism = oracle.ref_hostdecode_all(bp, vp, "u64", min(8, os.cpu_count() or 1), 1, mp)
        where = np.fromfile(mp, np.int64)
    ocol = oracle.deserialize(blob, "u64")
    pos = np.arange(len(values), dtype=np.int32)
    predicted = np.flatnonzero(oracle.decode_variant(ocol, pos, oracle.PRED_HOST)
                               != oracle.decode_variant(ocol, pos, oracle.PRED_CONTRACT))
    assert mism == len(where) and np.array_equal(where, predicted)
    # the device decodes every one of them (and every other value) exactly
    assert np.array_equal(codec.decompressFullFile(col), values)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built (make -C oracle ref)")
def test_c2_compressed_size_within_one_percent_of_reference(oracle):
    """200M uint64 piecewise column (seed 42, the decode benchmark's column): this library's
    variable partitioning against the reference's own compress with its CPU partitioner."""
    import torch

    values = W.piecewise_linear(200_000_000, seed=42)
    ctx = glc.Context(0)
    d = torch.from_numpy(values.view(np.int64)).to("cuda:0")
    col = glc.compress_device(ctx, glc.U64, d.data_ptr(), len(values), glc.VARIABLE)
    ctx.sync()
    mine = col.info().compressed_size_bytes
    out = torch.empty_like(d)
    glc.decompress_into(ctx, col, out.data_ptr())
    ctx.sync()
    assert torch.equal(out, d)
    col.free()
    del d, out
    with tempfile.TemporaryDirectory() as td:
        vp = os.path.join(td, "c2.values.bin")
        values.tofile(vp)
        ref = oracle.ref_compress_blob(vp, "u64", "var", os.path.join(td, "c2"))
    print(f"C2 compressed size: this library {mine:,} B, reference {ref:,} B, ratio {mine / ref:.5f}")
    with open(os.path.join(GOLDEN, "c2_reference_size.json")) as f:
        fixture = json.load(f)
    assert fixture["reference_compressed_bytes"] == ref
    assert mine <= 1.01 * ref
