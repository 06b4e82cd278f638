"""Launch-shape tuning (glc_autotune / glc_tune_*): every candidate shape decodes and looks up
bit-exactly, and measured tables round-trip through the cache file."""
import os

import numpy as np
import pytest
import torch

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu

NP = {glc.I32: np.int32, glc.I64: np.int64, glc.U64: np.uint64, glc.U32: np.uint32}
TH = {glc.I32: torch.int32, glc.I64: torch.int64, glc.U64: torch.int64, glc.U32: torch.int32}


def _column_values(dt, n, noise_bits, seed):
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    if dt in (glc.I32, glc.U32):
        noise_bits = min(noise_bits, 28)
        return (1000 + 3 * i + rng.integers(0, 1 << noise_bits, n)).astype(NP[dt])
    if dt == glc.U64:
        return W.piecewise_linear(n, seed=seed, mean_segment=20_000)
    return ((1 << 40) + 1000 * i + rng.integers(0, 1 << noise_bits, n)).astype(np.int64)


def _set_all(ctx, dt, plain, stages, unroll, ra_shape, warps=0):
    for b in (8, 16, 24, 32, 48, 64):  # every bucket, whatever the column's widest field
        glc.tune_set(ctx, dt, b, plain, stages, unroll, ra_shape, warps=warps)


@pytest.mark.parametrize("dt", [glc.I32, glc.I64, glc.U64, glc.U32])
@pytest.mark.parametrize("mode", [glc.FIXED, glc.VARIABLE])
def test_every_shape_is_bit_exact(dt, mode):
    ctx = glc.Context(0)
    v = _column_values(dt, 300_001, 21, seed=3 + dt)
    col = glc.compress_device(ctx, dt, v.ctypes.data, len(v), mode, host=True)
    pos = np.random.default_rng(5).integers(-3, len(v) + 3, 50_000).astype(np.int32)
    want_ra = np.where((pos >= 0) & (pos < len(v)), v[np.clip(pos, 0, len(v) - 1)], 0).astype(v.dtype)
    d_pos = torch.from_numpy(pos).cuda()
    out = torch.zeros(len(v), dtype=TH[dt], device="cuda:0")
    ra = torch.zeros(len(pos), dtype=TH[dt], device="cuda:0")
    for plain in (False, True):
        if plain:
            glc.preunpack(ctx, col)
        src = glc.SRC_PREUNPACKED if plain else glc.SRC_PACKED
        for stages in (2, 3, 4):
            for unroll in ((1, 2, 4) if not plain else (2,)):
                for warps in ((8, 4) if not plain else (8,)):  # consumer warps per CTA
                    _set_all(ctx, dt, plain, stages, unroll, 0, warps)
                    out.fill_(0)
                    torch.cuda.synchronize()  # the library runs on its own stream
                    glc.decompress_into(ctx, col, out.data_ptr(), source=src)
                    ctx.sync()
                    assert np.array_equal(out.cpu().numpy().view(NP[dt]), v), (plain, stages, unroll, warps)
        # a range decode with a partial first and last tile on 4 warps
        if not plain:
            _set_all(ctx, dt, plain, 3, 2, 0, 4)
            part = torch.zeros(len(v), dtype=TH[dt], device="cuda:0")
            torch.cuda.synchronize()
            glc.decompress_range_into(ctx, col, 1001, 200_003, part.data_ptr() + 1001 * v.itemsize, source=src)
            ctx.sync()
            assert np.array_equal(part.cpu().numpy().view(NP[dt])[1001:201_004], v[1001:201_004])
        for ra_shape in range(5):
            _set_all(ctx, dt, plain, 2, 2, ra_shape)
            ra.fill_(0)
            torch.cuda.synchronize()
            glc.random_access_into(ctx, col, d_pos.data_ptr(), len(pos), ra.data_ptr(), source=src)
            ctx.sync()
            assert np.array_equal(ra.cpu().numpy().view(NP[dt]), want_ra), (plain, ra_shape)
    col.free()


def test_autotune_measures_and_caches(tmp_path):
    path = str(tmp_path / "tune.txt")
    ctx = glc.Context(0)
    assert glc.tune_get(ctx, glc.U64, 25).measured == 0
    glc.autotune(ctx, path)
    assert os.path.exists(path)
    got = {}
    for dt in (glc.I32, glc.I64, glc.U64, glc.U32):
        for b in (8, 16, 24, 32, 48, 64):
            for plain in (False, True):
                e = glc.tune_get(ctx, dt, b, plain)
                assert e.measured == 1 and e.decode_gbs > 0 and e.ra_glookups > 0
                assert e.decode_stages in (2, 3, 4) and e.decode_unroll in (1, 2, 4) and 0 <= e.ra_shape <= 4
                assert e.decode_warps in (4, 8) and e.partition_len in (1024, 2048, 4096)
                got[(dt, b, plain)] = (e.decode_stages, e.decode_unroll, e.ra_shape, e.decode_warps, e.partition_len)
    # a second context loads the file instead of measuring
    ctx2 = glc.Context(0)
    glc.autotune(ctx2, path)
    for (dt, b, plain), shape in got.items():
        e = glc.tune_get(ctx2, dt, b, plain)
        assert e.measured == 1 and (e.decode_stages, e.decode_unroll, e.ra_shape, e.decode_warps,
                                    e.partition_len) == shape
    # a file written for another device is ignored by a new context
    with open(path) as f:
        lines = f.read().splitlines()
    lines[0] = lines[0] + "_other_device"
    other = str(tmp_path / "other.txt")
    with open(other, "w") as f:
        f.write("\n".join(lines) + "\n")
    os.environ["GLC_TUNE_CACHE"] = other
    try:
        ctx3 = glc.Context(0)
    finally:
        del os.environ["GLC_TUNE_CACHE"]
    assert glc.tune_get(ctx3, glc.U64, 25).measured == 0


@pytest.mark.parametrize("dt", [glc.I64, glc.U64])
def test_wide_fields_with_a_whole_tile_staged(dt):
    """Columns with fields wider than 48 bits (and direct-copy partitions) decode the same whether
    their tiles are staged in shared memory (capacity 8208 words) or read from global memory."""
    ctx = glc.Context(0)
    rng = np.random.default_rng(9)
    n = 200_003
    i = np.arange(n, dtype=np.int64)
    v = ((1 << 40) + 1000 * i + rng.integers(0, 1 << 59, n)).astype(np.int64)
    if dt == glc.U64:
        v = v.astype(np.uint64)
        v[50_000:60_000] += np.uint64(1 << 62)  # above 2^53: direct copy
    col = glc.compress_device(ctx, dt, v.ctypes.data, n, glc.FIXED, host=True)
    out = torch.zeros(n, dtype=torch.int64, device="cuda:0")
    for cap in (0, 8208):
        for stages in (2, 3, 4):
            for b in (8, 16, 24, 32, 48, 64):
                glc.tune_set(ctx, dt, b, False, stages, 2, 4, cap)
            out.fill_(0)
            torch.cuda.synchronize()
            glc.decompress_into(ctx, col, out.data_ptr(), source=glc.SRC_PACKED)
            ctx.sync()
            assert np.array_equal(out.cpu().numpy().view(v.dtype), v), (cap, stages)
    col.free()
