"""glc_attach_blob: a column that reads a serialized blob where it lies (the reference's
createDirectAccessHandle + directRandomAccessGPU, api/G-LeCo.cuh:1157-1334).

Random access, range decode and full decode on the attached blob must equal deserialize + the
same calls, for the reference's own golden blobs and for blobs made here, whether the blob is a
host blob copied once, a device blob read in place (its bitstream 16-byte aligned or not, with
arbitrary bytes after it), or a device blob that ends at the end of its allocation (only its
bitstream is then copied).
"""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
CODE = {"i32": glc.I32, "i64": glc.I64, "u64": glc.U64, "u32": glc.U32}
NPC = {np.dtype(np.int32): glc.I32, np.dtype(np.int64): glc.I64, np.dtype(np.uint64): glc.U64,
       np.dtype(np.uint32): glc.U32}


def _cudart():
    import glob
    cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "lib", "libcudart*.so*"))
    cands += glob.glob("/usr/local/cuda/lib64/libcudart.so*")
    for c in cands:
        try:
            lib = ctypes.CDLL(c)
            lib.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
            lib.cudaFree.argtypes = [ctypes.c_void_p]
            return lib
        except OSError:
            continue
    pytest.skip("no CUDA runtime library to allocate with")


def _check_same(ctx, att, ref, values):
    n = len(values)
    assert att.info().total_values == n and att.info().compressed_size_bytes == ref.info().compressed_size_bytes
    dt = values.dtype
    full = torch.empty(max(n, 1), dtype=torch.int64 if dt.itemsize == 8 else torch.int32, device="cuda:0")
    glc.decompress_into(ctx, att, full.data_ptr())
    ctx.sync()
    assert np.array_equal(full.cpu().numpy().view(dt)[:n], values)
    rng = np.random.default_rng(n)
    pos = np.concatenate([rng.integers(0, n, 50_000), [0, n - 1, n, -1]]).astype(np.int32)
    a = np.zeros(len(pos), dt)
    b = np.zeros(len(pos), dt)
    glc.random_access_into(ctx, att, pos.ctypes.data, len(pos), a.ctypes.data, host_in=True, host_out=True)
    glc.random_access_into(ctx, ref, pos.ctypes.data, len(pos), b.ctypes.data, host_in=True, host_out=True)
    assert np.array_equal(a, b)
    inside = (pos >= 0) & (pos < n)
    assert np.array_equal(a[inside], values[pos[inside]])
    first, count = n // 5, max(1, n // 3)
    r = np.zeros(count, dt)
    glc.decompress_range_into(ctx, att, first, count, r.ctypes.data, host_out=True)
    assert np.array_equal(r, values[first:first + count])
    if att.info().fixed_partition_len > 0:
        f = np.zeros(len(pos[inside]), dt)
        p = np.ascontiguousarray(pos[inside])
        glc.random_access_into(ctx, att, p.ctypes.data, len(p), f.ctypes.data,
                               fixed_len=att.info().fixed_partition_len, host_in=True, host_out=True)
        assert np.array_equal(f, values[p])


def _golden():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return sorted(json.load(f).items())


@pytest.mark.parametrize("name,meta", _golden(), ids=[g[0] for g in _golden()])
def test_attach_reference_blobs(name, meta):
    values = np.load(os.path.join(GOLDEN, f"{name}.values.npy"))
    with open(os.path.join(GOLDEN, f"{name}.blob"), "rb") as f:
        blob = f.read()
    ctx = glc.Context(0)
    hb = np.frombuffer(blob, np.uint8).copy()
    att = glc.attach_blob(ctx, CODE[meta["dtype"]], hb.ctypes.data, len(hb), host=True)
    ref = glc.deserialize_host(ctx, CODE[meta["dtype"]], blob)
    assert att is not None and att.info().compressed_size_bytes == meta["reported_size"]
    _check_same(ctx, att, ref, values)
    assert glc.serialize_host(ctx, att) == blob
    # the drop-in class: createDirectAccessHandle / directRandomAccessGPU / destroyDirectAccessHandle
    codec = glc.LeCoGPU(values.dtype, device=0)
    h = codec.createDirectAccessHandle(blob)
    pos = np.random.default_rng(1).integers(0, len(values), 1000).astype(np.int32)
    assert np.array_equal(codec.directRandomAccessGPU(h, pos), values[pos])
    codec.destroyDirectAccessHandle(h)
    att.free()
    ref.free()


def _device_columns():
    rng = np.random.default_rng(4)
    i = np.arange(2_000_000, dtype=np.int64)
    return [
        ("u64_piecewise_var", W.piecewise_linear(1_500_000, seed=3, mean_segment=30_000), glc.VARIABLE, 0),
        ("i64_timestamps_fixed", W.timestamps(1_000_003, seed=2), glc.FIXED, 4096),
        ("i32_plain_fixed1024", W.plain_small(1 << 20, seed=5), glc.FIXED, 1024),
        ("u32_noise_var", (i[:700_001] * 13 + rng.integers(0, 1 << 9, 700_001)).astype(np.uint32), glc.VARIABLE, 0),
        ("i64_walk_fixed1000", np.cumsum(rng.integers(-300, 900, 500_000), dtype=np.int64), glc.FIXED, 1000),
    ]


@pytest.mark.parametrize("lead", [0, 8])
@pytest.mark.parametrize("name,values,mode,L", _device_columns(), ids=[c[0] for c in _device_columns()])
def test_attach_device_blob_in_place(name, values, mode, L, lead):
    """A device blob read in place, at an offset of 0 or 8 bytes (the bitstream 16-byte aligned or
    not), with 0xFF bytes after it."""
    ctx = glc.Context(0)
    code = NPC[values.dtype]
    col = glc.compress_device(ctx, code, values.ctypes.data, len(values), mode, fixed_len=L or 4096, host=True)
    blob = glc.serialize_host(ctx, col)
    buf = torch.full((lead + len(blob) + 4096,), 0xFF, dtype=torch.uint8, device="cuda:0")
    buf[lead:lead + len(blob)] = torch.from_numpy(np.frombuffer(blob, np.uint8).copy()).cuda()
    torch.cuda.synchronize()
    att = glc.attach_blob(ctx, code, buf.data_ptr() + lead, len(blob))
    assert att is not None
    _check_same(ctx, att, col, values)
    assert glc.serialize_host(ctx, att) == blob
    # the batch decode reads attached columns like any other
    batch = glc.Batch.of(ctx, [att, col])
    outs = [torch.zeros(len(values) + 8, dtype=torch.int64 if values.dtype.itemsize == 8 else torch.int32,
                        device="cuda:0") for _ in range(2)]
    batch.decompress([o.data_ptr() for o in outs])
    ctx.sync()
    for o in outs:
        assert np.array_equal(o.cpu().numpy().view(values.dtype)[:len(values)], values)
    batch.free()
    att.free()
    col.free()
    del buf


def test_attach_device_blob_at_the_end_of_its_allocation():
    """A device blob whose allocation ends right after it: only its bitstream is copied, the values
    are the same."""
    rt = _cudart()
    values = W.piecewise_linear(600_000, seed=8, mean_segment=10_000)
    ctx = glc.Context(0)
    col = glc.compress_device(ctx, glc.U64, values.ctypes.data, len(values), glc.VARIABLE, host=True)
    blob = glc.serialize_host(ctx, col)
    size = (len(blob) + (2 << 20) - 1) // (2 << 20) * (2 << 20)
    p = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(p), size) == 0
    try:
        at = p.value + size - len(blob)  # blob sizes are multiples of 8: still 8-byte aligned
        t = torch.from_numpy(np.frombuffer(blob, np.uint8).copy())
        torch.cuda.synchronize()
        cp = rt.cudaMemcpy
        cp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        assert cp(ctypes.c_void_p(at), ctypes.c_void_p(t.data_ptr()), len(blob), 1) == 0  # host -> device
        att = glc.attach_blob(ctx, glc.U64, at, len(blob))
        _check_same(ctx, att, col, values)
        att.free()
    finally:
        torch.cuda.synchronize()
        rt.cudaFree(p)
    col.free()


def test_attach_rejects_bad_blobs_and_misalignment():
    values = W.timestamps(50_000, seed=1)
    ctx = glc.Context(0)
    col = glc.compress_device(ctx, glc.I64, values.ctypes.data, len(values), glc.FIXED, fixed_len=4096, host=True)
    blob = bytearray(glc.serialize_host(ctx, col))
    bad = bytearray(blob)
    bad[20] ^= 1  # header byte: checksum
    hb = np.frombuffer(bytes(bad), np.uint8).copy()
    assert glc.attach_blob(ctx, glc.I64, hb.ctypes.data, len(hb), host=True) is None
    hb = np.frombuffer(bytes(blob), np.uint8).copy()
    assert glc.attach_blob(ctx, glc.U32, hb.ctypes.data, len(hb), host=True) is None  # element size
    assert glc.attach_blob(ctx, glc.I64, hb.ctypes.data, len(hb) - 16, host=True) is None  # short
    d = torch.from_numpy(np.frombuffer(bytes(blob), np.uint8).copy()).cuda()
    with pytest.raises(glc.GlcError):
        glc.attach_blob(ctx, glc.I64, d.data_ptr() + 4, len(blob) - 8)  # not 8-byte aligned
    # an attached blob keeps its bitstream
    att = glc.attach_blob(ctx, glc.I64, d.data_ptr(), len(blob))
    with pytest.raises(glc.GlcError):
        glc.preunpack(ctx, att, drop_packed=True)
    glc.preunpack(ctx, att)  # pre-unpacking alone is fine
    out = np.zeros(len(values), np.int64)
    glc.decompress_into(ctx, att, out.ctypes.data, glc.SRC_PREUNPACKED, host_out=True)
    assert np.array_equal(out, values)
    att.free()
    col.free()
