"""CPU oracle for the G-LeCo learned-compression path -- TEST INFRASTRUCTURE ONLY.

Thin ctypes binding over ``liboracle.so`` (built from ``glc_oracle.cpp``).  The product
library never imports this package; tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline are its only users.  Each function restates the reference behaviour named in the
docstring (paths relative to the G-LeCo source tree).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
REF_HARNESS = os.path.join(_HERE, "_ref", "ref_harness")

DTYPES = {"i32": (0, np.int32), "i64": (1, np.int64), "u64": (2, np.uint64), "u32": (3, np.uint32)}
NP_TO_CODE = {np.dtype(np.int32): "i32", np.dtype(np.int64): "i64",
              np.dtype(np.uint64): "u64", np.dtype(np.uint32): "u32"}
MODEL_LINEAR = 1
MODEL_DIRECT_COPY = 4

_lib = None


def build() -> None:
    """Compile liboracle.so (and nothing else)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _declare(L):
    c_i64, c_i32, c_u64, c_vp, c_int = ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int
    L.orc_i128_to_double.restype = ctypes.c_double
    L.orc_i128_to_double.argtypes = [c_i64, c_u64]
    L.orc_solve_line.restype = None
    L.orc_solve_line.argtypes = [c_i64, c_i64, c_u64, c_i64, c_u64, c_vp, c_vp]
    L.orc_checksum.restype = ctypes.c_uint32
    L.orc_checksum.argtypes = [c_vp, c_u64, c_int]
    L.orc_partition_fixed.restype = c_i64
    L.orc_partition_fixed.argtypes = [c_i64, c_i32, c_vp, c_vp, c_i64]
    for name in ("orc_partition_v6", "orc_v6_variances"):
        f = getattr(L, name)
        f.restype = c_i64
        f.argtypes = [c_int, c_vp, c_i64, c_i32, c_vp] + ([c_vp, c_i64] if name == "orc_partition_v6" else [c_i64])
    for name in ("orc_partition_variable", "orc_ref_partition_cpu"):
        f = getattr(L, name)
        f.restype = c_i64
        f.argtypes = [c_int, c_vp, c_i64, c_vp, c_vp, c_i64]
    L.orc_split_best_end.restype = c_i64
    L.orc_split_best_end.argtypes = [c_int, c_vp, c_i64, c_i64]
    L.orc_range_bits.restype = c_int
    L.orc_range_bits.argtypes = [c_int, c_vp, c_i64, c_i64, c_i64]
    L.orc_fit.restype = c_int
    L.orc_fit.argtypes = [c_int, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp]
    L.orc_max_err_for_line.restype = c_i64
    L.orc_max_err_for_line.argtypes = [c_int, c_vp, c_i64, ctypes.c_double, ctypes.c_double]
    L.orc_bits_for.restype = c_int
    L.orc_bits_for.argtypes = [c_i64]
    L.orc_bit_offsets.restype = c_i64
    L.orc_bit_offsets.argtypes = [c_vp, c_vp, c_vp, c_i64, c_vp]
    L.orc_reported_size.restype = c_i64
    L.orc_reported_size.argtypes = [c_i64, c_i64]
    L.orc_pack.restype = c_int
    L.orc_pack.argtypes = [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64]
    L.orc_decode_full.restype = c_int
    L.orc_decode_full.argtypes = [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_i64, c_vp]
    L.orc_random_access.restype = c_int
    L.orc_random_access.argtypes = [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_vp, c_i64, c_vp]
    L.orc_decode_variant.restype = c_int
    L.orc_decode_variant.argtypes = [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_vp, c_i64, c_int,
                                     c_vp]
    L.orc_unpack_deltas.restype = c_int
    L.orc_unpack_deltas.argtypes = [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_i64, c_vp]
    L.orc_decode_preunpacked.restype = c_int
    L.orc_decode_preunpacked.argtypes = [c_int, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_vp]
    L.orc_blob_size.restype = c_u64
    L.orc_blob_size.argtypes = [c_i64, c_i64]
    L.orc_serialize.restype = c_i64
    L.orc_serialize.argtypes = [c_int, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_u64, c_int]
    L.orc_blob_check.restype = c_int
    L.orc_blob_check.argtypes = [c_vp, c_u64, c_int, c_int, c_vp, c_vp, c_vp]
    L.orc_deserialize.restype = c_int
    L.orc_deserialize.argtypes = [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]


def dtype_code(values: np.ndarray) -> str:
    return NP_TO_CODE[values.dtype]


@dataclass
class Column:
    """Host copy of a compressed column: the reference's CompressedData<T> SoA
    (api/G-LeCo_Types.cuh:18-42) plus the packed words."""
    dtype: str
    total_values: int
    starts: np.ndarray      # int32[P]
    ends: np.ndarray        # int32[P]
    types: np.ndarray       # int32[P]
    params: np.ndarray      # float64[4P]
    bits: np.ndarray        # int32[P]
    offsets: np.ndarray     # int64[P]
    errors: np.ndarray      # int64[P]
    words: np.ndarray       # uint32[ceil(total_bits/32)]
    total_bits: int

    @property
    def num_partitions(self) -> int:
        return int(self.starts.shape[0])

    def reported_size(self) -> int:
        """api/G-LeCo.cuh:589-603."""
        return int(lib().orc_reported_size(self.num_partitions, self.total_bits))


def partition_fixed(n: int, length: int):
    P = max(0, (n + length - 1) // length) if n > 0 else 0
    s = np.zeros(max(P, 1), np.int32)
    e = np.zeros(max(P, 1), np.int32)
    got = lib().orc_partition_fixed(n, length, _p(s), _p(e), len(s))
    return s[:got].copy(), e[:got].copy()


def _partition_call(fn, values: np.ndarray):
    values = np.ascontiguousarray(values)
    code, _ = DTYPES[dtype_code(values)]
    cap = max(16, len(values) // 64 + 16)
    while True:
        s = np.zeros(cap, np.int32)
        e = np.zeros(cap, np.int32)
        got = fn(code, _p(values), len(values), _p(s), _p(e), cap)
        if got >= 0:
            return s[:got].copy(), e[:got].copy()
        cap = -got


def partition_variable(values: np.ndarray):
    """This implementation's split/merge partitioner (restated on the CPU)."""
    return _partition_call(lib().orc_partition_variable, values)


def ref_partition_cpu(values: np.ndarray):
    """The reference's VariableLengthPartitioner (compression/CpuPartitioner.cuh), restated."""
    return _partition_call(lib().orc_ref_partition_cpu, values)


def partition_v6(values: np.ndarray, base: int = 2048):
    """The reference's GPU partitioner boundaries (GPUVariableLengthPartitionerV6, restated)."""
    values = np.ascontiguousarray(values)
    code, _ = DTYPES[dtype_code(values)]
    cap = len(values) // max(1, base // 2) + 64
    s = np.zeros(cap, np.int32)
    e = np.zeros(cap, np.int32)
    got = lib().orc_partition_v6(code, _p(values), len(values), base, _p(s), _p(e), cap)
    assert got >= 0
    return s[:got].copy(), e[:got].copy()


def v6_variances(values: np.ndarray, base: int = 2048) -> np.ndarray:
    """The per-block values the V6 thresholds come from."""
    values = np.ascontiguousarray(values)
    code, _ = DTYPES[dtype_code(values)]
    cap = len(values) // (8 * base) + 2
    out = np.zeros(cap, np.float32)
    got = lib().orc_v6_variances(code, _p(values), len(values), base, _p(out), cap)
    assert got >= 0
    return out[:got].copy()


def split_best_end(values: np.ndarray, start: int) -> int:
    values = np.ascontiguousarray(values)
    return int(lib().orc_split_best_end(DTYPES[dtype_code(values)][0], _p(values), len(values), start))


def range_bits(values: np.ndarray, a: int, b: int) -> int:
    values = np.ascontiguousarray(values)
    return int(lib().orc_range_bits(DTYPES[dtype_code(values)][0], _p(values), len(values), a, b))


def compress(values: np.ndarray, mode: str = "fixed", length: int = 4096, starts=None, ends=None) -> Column:
    """compress() of api/G-LeCo.cuh:349-614: partition, fit, offsets, pack."""
    values = np.ascontiguousarray(values)
    code_s = dtype_code(values)
    code = DTYPES[code_s][0]
    n = len(values)
    if starts is None:
        if mode == "fixed":
            starts, ends = partition_fixed(n, length)
        elif mode == "variable":
            starts, ends = partition_variable(values)
        elif mode == "ref_cpu":
            starts, ends = ref_partition_cpu(values)
        else:
            raise ValueError(mode)
    starts = np.ascontiguousarray(starts, np.int32)
    ends = np.ascontiguousarray(ends, np.int32)
    P = len(starts)
    types = np.zeros(P, np.int32)
    params = np.zeros(4 * P, np.float64)
    bits = np.zeros(P, np.int32)
    errs = np.zeros(P, np.int64)
    offs = np.zeros(P, np.int64)
    if P:
        lib().orc_fit(code, _p(values), _p(starts), _p(ends), P, _p(types), _p(params), _p(bits), _p(errs))
    total_bits = int(lib().orc_bit_offsets(_p(starts), _p(ends), _p(bits), P, _p(offs))) if P else 0
    nwords = (total_bits + 31) // 32
    words = np.zeros(max(nwords, 1), np.uint32)
    if P and nwords:
        lib().orc_pack(code, _p(values), _p(starts), _p(ends), _p(types), _p(params), _p(bits), _p(offs), P,
                       _p(words), nwords)
    return Column(code_s, n, starts, ends, types, params, bits, offs, errs, words[:nwords].copy(), total_bits)


def column_with_lines(values: np.ndarray, starts, ends, thetas) -> Column:
    """A LINEAR column whose partitions use the given (theta0, theta1) instead of a fit; bits
    and residuals follow the format rules.  Used to plant exact .5 prediction ties."""
    values = np.ascontiguousarray(values)
    code_s = dtype_code(values)
    code = DTYPES[code_s][0]
    starts = np.ascontiguousarray(starts, np.int32)
    ends = np.ascontiguousarray(ends, np.int32)
    P = len(starts)
    types = np.full(P, MODEL_LINEAR, np.int32)
    params = np.zeros(4 * P, np.float64)
    bits = np.zeros(P, np.int32)
    errs = np.zeros(P, np.int64)
    for p, (t0, t1) in enumerate(thetas):
        params[4 * p], params[4 * p + 1] = t0, t1
        seg = np.ascontiguousarray(values[starts[p]:ends[p]])
        errs[p] = lib().orc_max_err_for_line(code, _p(seg), len(seg), t0, t1)
        bits[p] = lib().orc_bits_for(int(errs[p]))
    offs = np.zeros(P, np.int64)
    total_bits = int(lib().orc_bit_offsets(_p(starts), _p(ends), _p(bits), P, _p(offs)))
    nwords = (total_bits + 31) // 32
    words = np.zeros(max(nwords, 1), np.uint32)
    if nwords:
        lib().orc_pack(code, _p(values), _p(starts), _p(ends), _p(types), _p(params), _p(bits), _p(offs), P,
                       _p(words), nwords)
    return Column(code_s, len(values), starts, ends, types, params, bits, offs, errs, words[:nwords].copy(), total_bits)


def _words_padded(col: Column):
    w = np.zeros(len(col.words) + 4, np.uint32)
    w[: len(col.words)] = col.words
    return w


def decode_full(col: Column) -> np.ndarray:
    """FullDecompressionKernels.cuh:47-192 (all full-decode variants produce these values)."""
    code, npdt = DTYPES[col.dtype]
    out = np.zeros(col.total_values, npdt)
    w = _words_padded(col)
    lib().orc_decode_full(code, _p(col.starts), _p(col.ends), _p(col.types), _p(col.params), _p(col.bits),
                          _p(col.offsets), col.num_partitions, _p(w), len(col.words), col.total_values, _p(out))
    return out


def random_access(col: Column, positions: np.ndarray) -> np.ndarray:
    """RandomAccessKernels.cuh:55-169 / FixedPartitionKernels.cuh:50-130."""
    code, npdt = DTYPES[col.dtype]
    pos = np.ascontiguousarray(positions, np.int32)
    out = np.zeros(len(pos), npdt)
    w = _words_padded(col)
    lib().orc_random_access(code, _p(col.starts), _p(col.ends), _p(col.types), _p(col.params), _p(col.bits),
                            _p(col.offsets), col.num_partitions, _p(w), len(col.words), _p(pos), len(pos), _p(out))
    return out


# prediction variants of the reference's decoders (glc_oracle.cpp PredVariant)
PRED_CONTRACT = 0          # fma, round half away: every full decoder and packed random access
PRED_HOST = 1              # directRandomAccessCPU (api/G-LeCo.cuh:1470-1646): no fma
PRED_FIXED_PREUNPACKED = 2  # randomAccessFixedPreUnpackedKernel (FixedPartitionKernels.cuh:185-206): ties to even


def decode_variant(col: Column, positions: np.ndarray, variant: int) -> np.ndarray:
    """Values that the reference decoder named by ``variant`` returns at ``positions``."""
    code, npdt = DTYPES[col.dtype]
    pos = np.ascontiguousarray(positions, np.int32)
    out = np.zeros(len(pos), npdt)
    w = _words_padded(col)
    lib().orc_decode_variant(code, _p(col.starts), _p(col.ends), _p(col.types), _p(col.params), _p(col.bits),
                             _p(col.offsets), col.num_partitions, _p(w), len(col.words), _p(pos), len(pos), variant,
                             _p(out))
    return out


def unpack_deltas(col: Column) -> np.ndarray:
    """decompression/UnpackKernel.cuh:31-98."""
    code, _ = DTYPES[col.dtype]
    out = np.zeros(col.total_values, np.int64)
    w = _words_padded(col)
    lib().orc_unpack_deltas(code, _p(col.starts), _p(col.ends), _p(col.types), _p(col.bits), _p(col.offsets),
                            col.num_partitions, _p(w), len(col.words), col.total_values, _p(out))
    return out


def decode_preunpacked(col: Column, plain: np.ndarray) -> np.ndarray:
    """FullDecompressionKernels.cuh:196-288."""
    code, npdt = DTYPES[col.dtype]
    out = np.zeros(col.total_values, npdt)
    plain = np.ascontiguousarray(plain, np.int64)
    lib().orc_decode_preunpacked(code, _p(col.starts), _p(col.ends), _p(col.types), _p(col.params),
                                 col.num_partitions, _p(plain), col.total_values, _p(out))
    return out


def checksum(data: bytes, crc32c: bool = False) -> int:
    b = np.frombuffer(data, np.uint8)
    return int(lib().orc_checksum(_p(b), len(b), 1 if crc32c else 0))


def serialize(col: Column, crc32c: bool = False) -> bytes:
    """Blob v5, api/G-LeCo.cuh:826-1016."""
    size = int(lib().orc_blob_size(col.num_partitions, col.total_bits))
    blob = np.zeros(size, np.uint8)
    w = _words_padded(col)
    tsize = np.dtype(DTYPES[col.dtype][1]).itemsize
    got = lib().orc_serialize(tsize, col.total_values, _p(col.starts), _p(col.ends), _p(col.types),
                              _p(col.params), _p(col.bits), _p(col.offsets), _p(col.errors), col.num_partitions,
                              _p(w), _p(blob), size, 1 if crc32c else 0)
    assert got == size, (got, size)
    return blob.tobytes()


class BlobError(ValueError):
    pass


def deserialize(blob: bytes, dtype: str, crc32c: bool = False) -> Column:
    """api/G-LeCo.cuh:1019-1154, with bounds checks on every array.  Raises BlobError
    where the reference returns nullptr."""
    b = np.frombuffer(blob, np.uint8)
    tv = ctypes.c_int64()
    P = ctypes.c_int64()
    db = ctypes.c_uint64()
    tsize = np.dtype(DTYPES[dtype][1]).itemsize
    rc = lib().orc_blob_check(_p(b), len(b), tsize, 1 if crc32c else 0, ctypes.byref(tv), ctypes.byref(P),
                              ctypes.byref(db))
    if rc != 0:
        raise BlobError(f"blob rejected (reason {rc})")
    P = P.value
    nw = (db.value + 3) // 4
    starts = np.zeros(P, np.int32); ends = np.zeros(P, np.int32); types = np.zeros(P, np.int32)
    params = np.zeros(4 * P, np.float64); bits = np.zeros(P, np.int32)
    offs = np.zeros(P, np.int64); errs = np.zeros(P, np.int64)
    words = np.zeros(max(nw, 1), np.uint32)
    lib().orc_deserialize(_p(b), _p(starts), _p(ends), _p(types), _p(params), _p(bits), _p(offs), _p(errs),
                          _p(words))
    total_bits = 0
    if P:
        total_bits = int(max(int(offs[p]) + int(ends[p] - starts[p]) * int(bits[p]) for p in range(P)))
    return Column(dtype, tv.value, starts, ends, types, params, bits, offs, errs, words[:nw].copy(), total_bits)


def reported_size(P: int, total_bits: int) -> int:
    return int(lib().orc_reported_size(P, total_bits))


# ---------------------------------------------------------------------------------------
# The reference harness (oracle/_ref/ref_harness), built from the reference's own sources.
# ---------------------------------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(REF_HARNESS)


def _ref_run(args, cpu_only=True):
    env = dict(os.environ)
    if cpu_only:
        env["GLC_REF_CPU_ONLY"] = "1"
    r = subprocess.run([REF_HARNESS] + [str(a) for a in args], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout


def ref_partition(values: np.ndarray, workdir: str):
    """The reference's own VariableLengthPartitioner, run from the compiled reference."""
    vin = os.path.join(workdir, "ref_values.bin")
    vout = os.path.join(workdir, "ref_parts.bin")
    np.ascontiguousarray(values).tofile(vin)
    _ref_run(["partition", dtype_code(values), vin, vout])
    raw = np.fromfile(vout, np.uint8)
    P = int(raw[:8].view(np.int64)[0])
    rec = raw[8:].view(np.int32).reshape(P, 3)
    return rec[:, 0].copy(), rec[:, 1].copy(), rec[:, 2].copy()


def ref_partition_v6(values: np.ndarray, workdir: str):
    """The reference's own GPUVariableLengthPartitionerV6 (base 2048, as compress uses it), run
    from the compiled reference on a GPU: (starts, ends)."""
    vin = os.path.join(workdir, "ref_values.bin")
    vout = os.path.join(workdir, "ref_parts_v6.bin")
    np.ascontiguousarray(values).tofile(vin)
    _ref_run(["v6", dtype_code(values), vin, vout], cpu_only=False)
    raw = np.fromfile(vout, np.uint8)
    P = int(raw[:8].view(np.int64)[0])
    rec = raw[8:].view(np.int32).reshape(P, 3)
    return rec[:, 0].copy(), rec[:, 1].copy()


def ref_hostdecode(blob: bytes, dtype: str, positions: np.ndarray, workdir: str, repeat: int = 1):
    """The reference's directRandomAccessCPU over a blob; returns (values, best seconds)."""
    bpath = os.path.join(workdir, "ref_blob.bin")
    ppath = os.path.join(workdir, "ref_pos.bin")
    opath = os.path.join(workdir, "ref_out.bin")
    with open(bpath, "wb") as f:
        f.write(blob)
    np.ascontiguousarray(positions, np.int32).tofile(ppath)
    secs = float(_ref_run(["hostdecode", dtype, bpath, ppath, opath, repeat]).strip().splitlines()[-1])
    return np.fromfile(opath, DTYPES[dtype][1]), secs


def ref_compress_blob(values_path: str, dtype: str, how: str, blob_prefix: str) -> int:
    """The reference's own stock LeCoGPU<T>::compress (fixed TILE_SIZE, its CPU partitioner
    ("var") or its GPU partitioner ("v6"), api/G-LeCo.cuh:349) + serialize (:826) of the raw
    values in ``values_path``, run from the compiled reference on a GPU.  Writes
    ``blob_prefix + ".blob"`` and returns the compressed size the reference reports."""
    return int(_ref_run(["golden", dtype, values_path, blob_prefix, how], cpu_only=False).strip().splitlines()[-1])


def ref_hostdecode_all(blob_path: str, values_path: str, dtype: str, threads: int, passes: int,
                       mism_path: str = None):
    """The reference's directRandomAccessCPU over every position of a blob, split across
    ``threads`` host threads; returns (seconds of each pass, values differing from the input)."""
    args = ["hostdecode_all", dtype, blob_path, values_path, threads, passes] + ([mism_path] if mism_path else [])
    lines = _ref_run(args).strip().splitlines()
    secs = [float(ln.split()[1]) for ln in lines if ln.startswith("pass ")]
    return secs, int(lines[-1].split()[1])


def ref_gpudecode(blob: bytes, values: np.ndarray, dtype: str, workdir: str, repeat: int = 1) -> dict:
    """The reference's own full decoders (deserializeGPU + _BitPacked, _OnTheFly_Optimized_V2,
    _WorkStealingAdvanced, and deserializeGPU(blob, true) + _PreUnpacked; api/G-LeCo.cuh:1739,
    :1842, :220, :1790) on a GPU: {decoder: (best API seconds, values differing from ``values``)}."""
    bp = os.path.join(workdir, "gd_blob.bin")
    vp = os.path.join(workdir, "gd_values.bin")
    with open(bp, "wb") as f:
        f.write(blob)
    np.ascontiguousarray(values).tofile(vp)
    res = {}
    for ln in _ref_run(["gpudecode", dtype, bp, vp, repeat], cpu_only=False).strip().splitlines():
        parts = ln.split()
        if len(parts) == 3 and parts[0].startswith("decompressFullFile"):
            res[parts[0]] = (float(parts[1]), int(parts[2]))
    return res


def ref_gpura(blob: bytes, values: np.ndarray, positions: np.ndarray, dtype: str, partition_len: int, workdir: str,
              repeat: int = 1) -> dict:
    """The reference's own random access on a GPU (randomAccessFixed when partition_len > 0,
    decompress, and on a pre-unpacked deserialization randomAccessPreUnpacked and, when
    partition_len > 0, randomAccessFixedPreUnpacked; api/G-LeCo.cuh:1878, :615, :696, :1931):
    {method: output array}."""
    bp = os.path.join(workdir, "ra_blob.bin")
    pp = os.path.join(workdir, "ra_pos.bin")
    vp = os.path.join(workdir, "ra_values.bin")
    prefix = os.path.join(workdir, "ra_out")
    with open(bp, "wb") as f:
        f.write(blob)
    np.ascontiguousarray(positions, np.int32).tofile(pp)
    np.ascontiguousarray(values).tofile(vp)
    out = {}
    for ln in _ref_run(["gpura", dtype, bp, pp, vp, partition_len, repeat, prefix], cpu_only=False).strip().splitlines():
        parts = ln.split()
        if len(parts) == 3 and not parts[0][0].isdigit():
            out[parts[0]] = np.fromfile(f"{prefix}.{parts[0]}.bin", DTYPES[dtype][1])
    return out
