"""Python binding of libglc (include/glc.h) over ctypes.

``LeCoGPU`` mirrors the reference's class (api/G-LeCo.cuh:39-2304): the same method names,
argument meaning and error behaviour (a rejected blob gives ``None`` where the reference
returns ``nullptr``; other failures raise ``GlcError``).  Every call goes through the C ABI to
the CUDA kernels in libglc.so; there is no host fallback, and importing this module without
the built library raises.

Lower-level functions (``compress_device``, ``decompress_into`` ...) take raw device pointers
and a CUDA stream handle so callers can keep data resident in HBM.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libglc.so")

I32, I64, U64, U32 = 0, 1, 2, 3
FIXED, VARIABLE, VARIABLE_V6 = 0, 1, 2
SRC_AUTO, SRC_PACKED, SRC_PREUNPACKED = 0, 1, 2
HOST_IN, HOST_OUT = 1, 2
OK, ERR_INVALID_ARG, ERR_BAD_BLOB, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_BUDGET, ERR_UNSUPPORTED = range(8)

NP_DTYPE = {I32: np.int32, I64: np.int64, U64: np.uint64, U32: np.uint32}
DTYPE_OF = {np.dtype(np.int32): I32, np.dtype(np.int64): I64, np.dtype(np.uint64): U64, np.dtype(np.uint32): U32}
TILE_SIZE = 4096  # the reference's default fixed partition length (core/CudaUtils.cuh:18)

EXPORTS = [
    "glc_create", "glc_destroy", "glc_last_error", "glc_status_string", "glc_sync", "glc_compress",
    "glc_partition_variable", "glc_partition_v6", "glc_column_free", "glc_column_get_info", "glc_decompress_full",
    "glc_decompress_range", "glc_random_access", "glc_preunpack", "glc_blob_size", "glc_serialize",
    "glc_deserialize", "glc_attach_blob", "glc_decode_blob_to_host", "glc_decompress_range_noalloc",
    "glc_batch_create", "glc_batch_compress",
    "glc_batch_column", "glc_batch_decompress", "glc_batch_recompress", "glc_batch_sync", "glc_batch_free", "glc_server_create", "glc_server_destroy",
    "glc_server_admit", "glc_server_admit_blob", "glc_server_evict", "glc_server_submit", "glc_server_poll",
    "glc_server_drain", "glc_server_get_stats", "glc_server_now_ns", "glc_server_columns",
    "glc_autotune", "glc_tune_get", "glc_tune_set",
]
REQ_LOOKUP, REQ_RANGE = 0, 1
SERVER_RESERVE = 1
NOALLOC_MAX_OUTPUT_BYTES = 4 << 20


class GlcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"glc status {status}: {msg}")
        self.status = status


class ColumnInfo(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int), ("total_values", ctypes.c_int64), ("num_partitions", ctypes.c_int64),
        ("total_bits", ctypes.c_int64), ("compressed_size_bytes", ctypes.c_int64),
        ("fixed_partition_len", ctypes.c_int32), ("has_packed", ctypes.c_int32), ("has_preunpacked", ctypes.c_int32),
        ("d_start_indices", ctypes.c_void_p), ("d_end_indices", ctypes.c_void_p), ("d_model_types", ctypes.c_void_p),
        ("d_model_params", ctypes.c_void_p), ("d_delta_bits", ctypes.c_void_p),
        ("d_delta_array_bit_offsets", ctypes.c_void_p), ("d_error_bounds", ctypes.c_void_p),
        ("delta_array", ctypes.c_void_p), ("d_plain_deltas", ctypes.c_void_p), ("max_delta_bits", ctypes.c_int32),
    ]


class TuneEntry(ctypes.Structure):
    _fields_ = [("decode_stages", ctypes.c_int32), ("decode_unroll", ctypes.c_int32), ("ra_shape", ctypes.c_int32),
                ("measured", ctypes.c_int32), ("decode_cap_words", ctypes.c_int32), ("decode_warps", ctypes.c_int32),
                ("decode_gbs", ctypes.c_float), ("ra_glookups", ctypes.c_float), ("partition_len", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


TUNE_FORCE = 1


class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("slots", ctypes.c_int32), ("max_requests", ctypes.c_int32),
                ("max_lookups", ctypes.c_int64), ("max_range_values", ctypes.c_int64), ("flags", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("column", ctypes.c_int32), ("first", ctypes.c_int64),
                ("count", ctypes.c_int64), ("positions", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("tag", ctypes.c_int64), ("not_before_ns", ctypes.c_int64)]


class Completion(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_int64), ("status", ctypes.c_int32), ("launches", ctypes.c_int32),
                ("arrival_ns", ctypes.c_int64), ("done_ns", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("resident_bytes", ctypes.c_uint64), ("resident_columns", ctypes.c_int32),
                ("in_flight", ctypes.c_int32), ("launches", ctypes.c_int64), ("submitted", ctypes.c_int64),
                ("completed", ctypes.c_int64), ("lookups", ctypes.c_int64), ("range_values", ctypes.c_int64),
                ("evictions", ctypes.c_int64), ("admissions_refused", ctypes.c_int64)]


# numpy mirrors of the structures, for building many requests at once
REQUEST_DTYPE = np.dtype([("kind", np.int32), ("column", np.int32), ("first", np.int64), ("count", np.int64),
                          ("positions", np.uint64), ("out", np.uint64), ("tag", np.int64),
                          ("not_before_ns", np.int64)])
COMPLETION_DTYPE = np.dtype([("tag", np.int64), ("status", np.int32), ("launches", np.int32),
                             ("arrival_ns", np.int64), ("done_ns", np.int64)])
assert REQUEST_DTYPE.itemsize == ctypes.sizeof(Request) and COMPLETION_DTYPE.itemsize == ctypes.sizeof(Completion)

_lib = None


def load() -> ctypes.CDLL:
    """Load libglc.so; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libglc.so is not built ({LIB_PATH}); run __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    vp, i64, i32, u64, c_int = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int
    pvp, pi64, pu64 = ctypes.POINTER(vp), ctypes.POINTER(i64), ctypes.POINTER(u64)
    sig = {
        "glc_create": ([pvp, c_int], c_int),
        "glc_destroy": ([vp], c_int),
        "glc_last_error": ([vp], ctypes.c_char_p),
        "glc_status_string": ([c_int], ctypes.c_char_p),
        "glc_sync": ([vp, vp], c_int),
        "glc_compress": ([vp, c_int, vp, i64, c_int, c_int, i32, pvp, pi64, vp], c_int),
        "glc_partition_variable": ([vp, c_int, vp, i64, c_int, vp, vp, i64, pi64, vp], c_int),
        "glc_partition_v6": ([vp, c_int, vp, i64, c_int, i32, vp, vp, i64, pi64, vp], c_int),
        "glc_column_free": ([vp], c_int),
        "glc_column_get_info": ([vp, ctypes.POINTER(ColumnInfo)], c_int),
        "glc_decompress_full": ([vp, vp, c_int, vp, c_int, vp], c_int),
        "glc_decompress_range": ([vp, vp, c_int, i64, i64, vp, c_int, vp], c_int),
        "glc_random_access": ([vp, vp, c_int, vp, i64, vp, c_int, i32, vp], c_int),
        "glc_preunpack": ([vp, vp, c_int, vp], c_int),
        "glc_blob_size": ([vp, pu64], c_int),
        "glc_serialize": ([vp, vp, vp, u64, c_int, c_int, pu64, vp], c_int),
        "glc_deserialize": ([vp, c_int, vp, u64, c_int, c_int, c_int, pvp, vp], c_int),
        "glc_decompress_range_noalloc": ([vp, i64, i64, vp, vp], c_int),
        "glc_attach_blob": ([vp, c_int, vp, u64, c_int, c_int, pvp, vp], c_int),
        "glc_decode_blob_to_host": ([vp, c_int, vp, u64, c_int, vp, pvp, vp], c_int),
        "glc_batch_create": ([vp, vp, i32, pvp], c_int),
        "glc_batch_compress": ([vp, vp, vp, vp, i32, i32, pvp, pi64, vp], c_int),
        "glc_batch_column": ([vp, i32, pvp], c_int),
        "glc_batch_decompress": ([vp, vp, vp, c_int, vp], c_int),
        "glc_batch_recompress": ([vp, vp, vp, c_int, vp], c_int),
        "glc_batch_sync": ([vp, vp, vp, pi64], c_int),
        "glc_batch_free": ([vp], c_int),
        "glc_server_create": ([vp, ctypes.POINTER(ServerConfig), pvp], c_int),
        "glc_server_destroy": ([vp], c_int),
        "glc_server_admit": ([vp, vp, ctypes.POINTER(i32)], c_int),
        "glc_server_admit_blob": ([vp, c_int, vp, u64, c_int, ctypes.POINTER(i32), vp], c_int),
        "glc_server_evict": ([vp, i32], c_int),
        "glc_server_submit": ([vp, vp, i32], c_int),
        "glc_server_poll": ([vp, vp, i32, ctypes.POINTER(i32)], c_int),
        "glc_server_drain": ([vp, i64], c_int),
        "glc_server_get_stats": ([vp, ctypes.POINTER(ServerStats)], c_int),
        "glc_server_now_ns": ([], i64),
        "glc_server_columns": ([vp, vp, i32, ctypes.POINTER(i32)], c_int),
        "glc_autotune": ([vp, ctypes.c_char_p, i32], c_int),
        "glc_tune_get": ([vp, c_int, i32, i32, ctypes.POINTER(TuneEntry)], c_int),
        "glc_tune_set": ([vp, c_int, i32, i32, ctypes.POINTER(TuneEntry)], c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """A glc context on one device (the reference's LeCoGPU constructor, api/G-LeCo.cuh:103)."""

    def __init__(self, device: int = -1):
        self.lib = load()
        h = ctypes.c_void_p()
        st = self.lib.glc_create(ctypes.byref(h), device)
        if st != OK:
            raise GlcError(st, "glc_create failed (no CUDA device?)")
        self.handle = h

    def check(self, st: int):
        if st != OK:
            raise GlcError(st, self.lib.glc_last_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            self.lib.glc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self, stream: int = 0):
        self.check(self.lib.glc_sync(self.handle, ctypes.c_void_p(stream)))


def autotune(ctx: "Context", cache_path: Optional[str] = None, force: bool = False):
    """Measure and keep the fastest launch shapes per element type and field width (glc_autotune)."""
    ctx.check(ctx.lib.glc_autotune(ctx.handle, cache_path.encode() if cache_path else None,
                                   TUNE_FORCE if force else 0))


def tune_get(ctx: "Context", dtype: int, field_bits: int, preunpacked: bool = False) -> TuneEntry:
    e = TuneEntry()
    ctx.check(ctx.lib.glc_tune_get(ctx.handle, dtype, field_bits, 1 if preunpacked else 0, ctypes.byref(e)))
    return e


def tune_set(ctx: "Context", dtype: int, field_bits: int, preunpacked: bool, stages: int, unroll: int, ra_shape: int,
             cap_words: int = 0, warps: int = 0, partition_len: int = 0):
    e = TuneEntry(stages, unroll, ra_shape, 0, cap_words, warps, 0.0, 0.0, partition_len, 0)
    ctx.check(ctx.lib.glc_tune_set(ctx.handle, dtype, field_bits, 1 if preunpacked else 0, ctypes.byref(e)))


class Column:
    """An owned compressed column (CompressedData<T>, api/G-LeCo_Types.cuh:18-42)."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p):
        self.ctx = ctx
        self.handle = handle

    def info(self) -> ColumnInfo:
        inf = ColumnInfo()
        self.ctx.check(self.ctx.lib.glc_column_get_info(self.handle, ctypes.byref(inf)))
        return inf

    @property
    def dtype(self) -> int:
        return self.info().dtype

    @property
    def total_values(self) -> int:
        return self.info().total_values

    @property
    def num_partitions(self) -> int:
        return self.info().num_partitions

    def free(self):
        if self.handle:
            self.ctx.lib.glc_column_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---- device-pointer level ----------------------------------------------------------------
def compress_device(ctx: Context, dtype: int, dptr: int, n: int, mode: int, fixed_len: int = TILE_SIZE,
                    stream: int = 0, host: bool = False) -> Column:
    h = ctypes.c_void_p()
    size = ctypes.c_int64()
    st = ctx.lib.glc_compress(ctx.handle, dtype, ctypes.c_void_p(dptr), n, HOST_IN if host else 0, mode, fixed_len,
                              ctypes.byref(h), ctypes.byref(size), ctypes.c_void_p(stream))
    ctx.check(st)
    return Column(ctx, h)


def decompress_into(ctx: Context, col: Column, out_ptr: int, source: int = SRC_AUTO, stream: int = 0,
                    host_out: bool = False):
    ctx.check(ctx.lib.glc_decompress_full(ctx.handle, col.handle, source, ctypes.c_void_p(out_ptr),
                                          HOST_OUT if host_out else 0, ctypes.c_void_p(stream)))


def decompress_range_into(ctx: Context, col: Column, first: int, count: int, out_ptr: int, source: int = SRC_AUTO,
                          stream: int = 0, host_out: bool = False):
    ctx.check(ctx.lib.glc_decompress_range(ctx.handle, col.handle, source, first, count, ctypes.c_void_p(out_ptr),
                                           HOST_OUT if host_out else 0, ctypes.c_void_p(stream)))


def decompress_range_noalloc(col: Column, first: int, count: int, out: np.ndarray, stream: int = 0) -> int:
    """glc_decompress_range_noalloc: values [first, first+count) into the host array ``out``
    without any allocation; returns the glc status (the caller checks it).  ``out`` must be a
    C-contiguous array of the column's element size holding at least ``count`` elements
    (ValueError otherwise: the C call would write past a shorter buffer)."""
    if not isinstance(out, np.ndarray) or not out.flags.c_contiguous:
        raise ValueError("out must be a C-contiguous numpy array")
    if out.itemsize != np.dtype(NP_DTYPE[col.dtype]).itemsize:
        raise ValueError("out's element size differs from the column's")
    if count > 0 and out.size < count:
        raise ValueError("out holds fewer than count elements")
    return col.ctx.lib.glc_decompress_range_noalloc(col.handle, first, count, ctypes.c_void_p(out.ctypes.data),
                                                    ctypes.c_void_p(stream))


def random_access_into(ctx: Context, col: Column, pos_ptr: int, q: int, out_ptr: int, source: int = SRC_AUTO,
                       fixed_len: int = 0, stream: int = 0, host_in: bool = False, host_out: bool = False):
    flags = (HOST_IN if host_in else 0) | (HOST_OUT if host_out else 0)
    ctx.check(ctx.lib.glc_random_access(ctx.handle, col.handle, source, ctypes.c_void_p(pos_ptr), q,
                                        ctypes.c_void_p(out_ptr), flags, fixed_len, ctypes.c_void_p(stream)))


def preunpack(ctx: Context, col: Column, drop_packed: bool = False, stream: int = 0):
    ctx.check(ctx.lib.glc_preunpack(ctx.handle, col.handle, 1 if drop_packed else 0, ctypes.c_void_p(stream)))


def partition_v6(ctx: Context, values: np.ndarray, base: int = 2048):
    """The reference's GPU partitioner boundaries on the device (glc_partition_v6)."""
    v = np.ascontiguousarray(values)
    cap = len(v) // max(1, base // 2) + 64
    s = np.zeros(cap, np.int32)
    e = np.zeros(cap, np.int32)
    P = ctypes.c_int64()
    ctx.check(ctx.lib.glc_partition_v6(ctx.handle, DTYPE_OF[v.dtype], _ptr(v), len(v), HOST_IN | HOST_OUT, base,
                                       _ptr(s), _ptr(e), cap, ctypes.byref(P), None))
    return s[:P.value].copy(), e[:P.value].copy()


def partition_variable(ctx: Context, values: np.ndarray):
    """Start/end arrays of the device partitioner for host values."""
    values = np.ascontiguousarray(values)
    cap = max(16, len(values) // 128 + 16)
    s = np.zeros(cap, np.int32)
    e = np.zeros(cap, np.int32)
    P = ctypes.c_int64()
    st = ctx.lib.glc_partition_variable(ctx.handle, DTYPE_OF[values.dtype], _ptr(values), len(values),
                                        HOST_IN | HOST_OUT, _ptr(s), _ptr(e), cap, ctypes.byref(P), None)
    ctx.check(st)
    return s[:P.value].copy(), e[:P.value].copy()


def serialize_host(ctx: Context, col: Column, crc32c: bool = False) -> bytes:
    size = ctypes.c_uint64()
    ctx.check(ctx.lib.glc_blob_size(col.handle, ctypes.byref(size)))
    buf = np.zeros(size.value, np.uint8)
    written = ctypes.c_uint64()
    ctx.check(ctx.lib.glc_serialize(ctx.handle, col.handle, _ptr(buf), size.value, HOST_OUT, 1 if crc32c else 0,
                                    ctypes.byref(written), None))
    return buf.tobytes()


def decode_blob_to_host(ctx: Context, dtype: int, blob_ptr: int, size: int, out_ptr: int, keep: bool = False,
                        stream: int = 0) -> Optional[Column]:
    """Streaming host blob -> host values (glc_decode_blob_to_host); with keep, the column."""
    h = ctypes.c_void_p()
    ctx.check(ctx.lib.glc_decode_blob_to_host(ctx.handle, dtype, ctypes.c_void_p(blob_ptr), size, 0,
                                              ctypes.c_void_p(out_ptr) if out_ptr else None,
                                              ctypes.byref(h) if keep else None, ctypes.c_void_p(stream)))
    return Column(ctx, h) if keep else None


def deserialize_host(ctx: Context, dtype: int, blob: bytes, pre_unpack: bool = False, crc32c: bool = False) -> Optional[Column]:
    b = np.frombuffer(blob, np.uint8)
    h = ctypes.c_void_p()
    st = ctx.lib.glc_deserialize(ctx.handle, dtype, _ptr(b) if len(b) else None, len(b), HOST_IN, 1 if crc32c else 0,
                                 1 if pre_unpack else 0, ctypes.byref(h), None)
    if st == ERR_BAD_BLOB:
        return None
    ctx.check(st)
    return Column(ctx, h)


def attach_blob(ctx: Context, dtype: int, blob_ptr: int, size: int, host: bool = False, crc32c: bool = False,
                stream: int = 0) -> Optional[Column]:
    """glc_attach_blob: a column that reads a serialized blob in place (a host blob is copied to the
    device once; a device blob is borrowed and must outlive the column).  None for a rejected blob."""
    h = ctypes.c_void_p()
    st = ctx.lib.glc_attach_blob(ctx.handle, dtype, ctypes.c_void_p(blob_ptr), size, HOST_IN if host else 0,
                                 1 if crc32c else 0, ctypes.byref(h), ctypes.c_void_p(stream))
    if st == ERR_BAD_BLOB:
        return None
    ctx.check(st)
    return Column(ctx, h)


class DirectAccessHandle:
    """The reference's DirectAccessHandle<T> (api/G-LeCo_Types.cuh:75-107): the host blob it was
    made from, and the device column that reads the blob's copy in place."""

    def __init__(self, blob: bytes, column: Column):
        self.data_blob_host = blob
        self.data_blob_size = len(blob)
        self.column = column


class BorrowedColumn(Column):
    """A column owned by a batch: freed with the batch, never on its own."""

    def free(self):
        self.handle = None


class _BatchColumns:
    """The columns of a compressed batch, as BorrowedColumn handles fetched on first access (a batch
    of thousands of columns is not walked on every compress)."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p, n: int):
        self._ctx, self._handle, self._n = ctx, handle, n
        self._cache = {}

    def __len__(self):
        return self._n

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[k] for k in range(*i.indices(self._n))]
        if i < 0:
            i += self._n
        if not 0 <= i < self._n:
            raise IndexError(i)
        c = self._cache.get(i)
        if c is None:
            h = ctypes.c_void_p()
            self._ctx.check(self._ctx.lib.glc_batch_column(self._handle, i, ctypes.byref(h)))
            c = self._cache[i] = BorrowedColumn(self._ctx, h)
        return c

    def __iter__(self):
        return (self[i] for i in range(self._n))


class Batch:
    """Many columns per launch: batched compress and one-launch decode (glc_batch_*)."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p, columns):
        self.ctx = ctx
        self.handle = handle
        self.columns = columns

    @classmethod
    def compress(cls, ctx: Context, dtypes, dptrs, ns, fixed_len: int = 0, stream: int = 0):
        n = len(dtypes)
        dt = np.ascontiguousarray(dtypes, dtype=np.int32)
        vp = np.ascontiguousarray(dptrs, dtype=np.uint64)
        nn = np.ascontiguousarray(ns, dtype=np.int64)
        h = ctypes.c_void_p()
        size = ctypes.c_int64()
        ctx.check(ctx.lib.glc_batch_compress(ctx.handle, dt.ctypes.data, vp.ctypes.data, nn.ctypes.data, n, fixed_len,
                                             ctypes.byref(h), ctypes.byref(size), ctypes.c_void_p(stream)))
        b = cls(ctx, h, _BatchColumns(ctx, h, n))
        b.compressed_size = size.value
        return b

    @classmethod
    def of(cls, ctx: Context, columns):
        n = len(columns)
        arr = (ctypes.c_void_p * n)(*[c.handle.value for c in columns])
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.glc_batch_create(ctx.handle, arr, n, ctypes.byref(h)))
        return cls(ctx, h, list(columns))

    def decompress(self, out_ptrs, use_graph: bool = False, stream: int = 0):
        arr = np.ascontiguousarray(out_ptrs, dtype=np.uint64)
        assert len(arr) == len(self.columns)
        self.ctx.check(self.ctx.lib.glc_batch_decompress(self.ctx.handle, self.handle, arr.ctypes.data,
                                                         1 if use_graph else 0, ctypes.c_void_p(stream)))

    def recompress(self, dptrs, use_graph: bool = False, stream: int = 0):
        """glc_batch_recompress: new values for the same columns, each at the length chosen before."""
        vp = np.ascontiguousarray(dptrs, dtype=np.uint64)
        assert len(vp) == len(self.columns)
        self.ctx.check(self.ctx.lib.glc_batch_recompress(self.ctx.handle, self.handle, vp.ctypes.data,
                                                         1 if use_graph else 0, ctypes.c_void_p(stream)))

    def sync(self, stream: int = 0) -> int:
        """glc_batch_sync: the columns' sizes after recompress; returns the total compressed size."""
        size = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.glc_batch_sync(self.ctx.handle, self.handle, ctypes.c_void_p(stream),
                                                   ctypes.byref(size)))
        self.compressed_size = size.value
        return size.value

    def free(self):
        if self.handle:
            self.ctx.lib.glc_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Resident columns and continuously batched requests (glc_server_*)."""

    def __init__(self, ctx: Context, budget_bytes: int, slots: int = 0, max_requests: int = 0, max_lookups: int = 0,
                 max_range_values: int = 0, reserve: bool = False):
        self.ctx = ctx
        cfg = ServerConfig(budget_bytes, slots, max_requests, max_lookups, max_range_values,
                           SERVER_RESERVE if reserve else 0, 0)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.glc_server_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h

    def admit(self, column: "Column") -> int:
        """Make a column resident; the server owns it afterwards."""
        i = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.glc_server_admit(self.handle, column.handle, ctypes.byref(i)))
        column.handle = None
        return i.value

    def admit_blob(self, dtype: int, blob_ptr: int, size: int, host: bool = False, stream: int = 0) -> int:
        i = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.glc_server_admit_blob(self.handle, dtype, ctypes.c_void_p(blob_ptr), size,
                                                          HOST_IN if host else 0, ctypes.byref(i),
                                                          ctypes.c_void_p(stream)))
        return i.value

    def evict(self, column_id: int):
        self.ctx.check(self.ctx.lib.glc_server_evict(self.handle, column_id))

    def submit(self, requests: np.ndarray):
        """requests: a REQUEST_DTYPE array."""
        r = np.ascontiguousarray(requests, REQUEST_DTYPE)
        self.ctx.check(self.ctx.lib.glc_server_submit(self.handle, ctypes.c_void_p(r.ctypes.data), len(r)))

    def poll(self, max_records: int = 1 << 16) -> np.ndarray:
        out = np.zeros(max_records, COMPLETION_DTYPE)
        got = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.glc_server_poll(self.handle, ctypes.c_void_p(out.ctypes.data), max_records,
                                                    ctypes.byref(got)))
        return out[: got.value]

    def drain(self, timeout_ms: int = -1):
        self.ctx.check(self.ctx.lib.glc_server_drain(self.handle, timeout_ms))

    def stats(self) -> ServerStats:
        s = ServerStats()
        self.ctx.check(self.ctx.lib.glc_server_get_stats(self.handle, ctypes.byref(s)))
        return s

    def now_ns(self) -> int:
        return self.ctx.lib.glc_server_now_ns()

    def columns(self) -> list:
        """Ids of the columns that accept requests."""
        n = 1 << 16
        ids = np.zeros(n, np.int32)
        got = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.glc_server_columns(self.handle, ctypes.c_void_p(ids.ctypes.data), n,
                                                       ctypes.byref(got)))
        return ids[: got.value].tolist()

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.glc_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def requests(n: int) -> np.ndarray:
    """An empty array of n requests (REQUEST_DTYPE)."""
    return np.zeros(n, REQUEST_DTYPE)


# ---- the reference's class API -------------------------------------------------------------
class LeCoGPU:
    """Drop-in mirror of ``template<typename T> class LeCoGPU`` (api/G-LeCo.cuh:39).

    Host numpy arrays in and out, as the reference's std::vector arguments; every call runs the
    CUDA kernels of libglc through the C ABI.
    """

    def __init__(self, dtype=np.int32, device: int = -1):
        self.np_dtype = np.dtype(dtype)
        self.code = DTYPE_OF[self.np_dtype]
        self.ctx = Context(device)

    # api/G-LeCo.cuh:349-614
    def compress(self, values: np.ndarray, use_variable_partitioning: bool, use_gpu_partitioning: bool = False,
                 dataset_name: str = "", fixed_partition_size: int = TILE_SIZE):
        """Returns (column, compressed_size_bytes).  Every partitioning runs on the GPU here;
        ``use_gpu_partitioning`` selects the reference's GPU partitioner's boundaries."""
        v = np.ascontiguousarray(values, self.np_dtype)
        h = ctypes.c_void_p()
        size = ctypes.c_int64()
        mode = (VARIABLE_V6 if use_gpu_partitioning else VARIABLE) if use_variable_partitioning else FIXED
        st = self.ctx.lib.glc_compress(self.ctx.handle, self.code, _ptr(v) if len(v) else None, len(v), HOST_IN,
                                       mode, fixed_partition_size, ctypes.byref(h), ctypes.byref(size), None)
        self.ctx.check(st)
        return Column(self.ctx, h), size.value

    def _full(self, col: Column, source: int) -> np.ndarray:
        n = col.total_values
        out = np.empty(n, self.np_dtype)
        if n:
            decompress_into(self.ctx, col, out.ctypes.data, source=source, host_out=True)
        return out

    # api/G-LeCo.cuh:680-693 and variants
    def decompressFullFile(self, col: Column) -> np.ndarray:
        return self._full(col, SRC_AUTO)

    def decompressFullFile_BitPacked(self, col: Column) -> np.ndarray:
        return self._full(col, SRC_PACKED)

    def decompressFullFile_PreUnpacked(self, col: Column) -> np.ndarray:
        return self._full(col, SRC_PREUNPACKED)

    decompressFullFile_WorkStealing = decompressFullFile_BitPacked
    decompressFullFile_WorkStealingAdvanced = decompressFullFile_BitPacked
    decompressFullFile_OnTheFly_Optimized_V2 = decompressFullFile

    def decompressFullFile_Fix(self, col: Column, partition_size: int) -> np.ndarray:
        inf = col.info()
        if inf.fixed_partition_len != partition_size and not (inf.num_partitions == 1 and
                                                              inf.total_values <= partition_size):
            raise GlcError(ERR_INVALID_ARG, "column is not partitioned with that fixed length")
        return self._full(col, SRC_AUTO)

    def _ra(self, col: Column, positions, source: int, fixed: int) -> np.ndarray:
        pos = np.ascontiguousarray(positions, np.int32)
        out = np.empty(len(pos), self.np_dtype)
        if len(pos):
            random_access_into(self.ctx, col, pos.ctypes.data, len(pos), out.ctypes.data, source=source,
                               fixed_len=fixed, host_in=True, host_out=True)
        return out

    # api/G-LeCo.cuh:615-678 (random access)
    def decompress(self, col: Column, positions) -> np.ndarray:
        return self._ra(col, positions, SRC_AUTO, 0)

    def randomAccessPreUnpacked(self, col: Column, positions) -> np.ndarray:
        return self._ra(col, positions, SRC_PREUNPACKED, 0)

    def randomAccessFixed(self, col: Column, positions, fixed_partition_size: int) -> np.ndarray:
        return self._ra(col, positions, SRC_PACKED, fixed_partition_size)

    def randomAccessFixedPreUnpacked(self, col: Column, positions, fixed_partition_size: int) -> np.ndarray:
        return self._ra(col, positions, SRC_PREUNPACKED, fixed_partition_size)

    # api/G-LeCo.cuh:826, :1999
    def serialize(self, col: Column, crc32c: bool = False) -> bytes:
        return serialize_host(self.ctx, col, crc32c)

    serializeGPU = serialize

    # api/G-LeCo.cuh:1019, :2157 -- None where the reference returns nullptr
    def deserialize(self, blob: bytes, crc32c: bool = False) -> Optional[Column]:
        return deserialize_host(self.ctx, self.code, blob, False, crc32c)

    def deserializeGPU(self, blob: bytes, preUnpackDeltas: bool = False, crc32c: bool = False) -> Optional[Column]:
        return deserialize_host(self.ctx, self.code, blob, preUnpackDeltas, crc32c)

    # api/G-LeCo.cuh:793-821
    def cleanup(self, col: Column):
        col.free()

    # api/G-LeCo.cuh:1157-1255 -- None where the reference returns nullptr
    def createDirectAccessHandle(self, blob: bytes, copy_to_device: bool = True) -> Optional[DirectAccessHandle]:
        b = np.frombuffer(blob, np.uint8)
        if len(b) == 0:
            return None
        col = attach_blob(self.ctx, self.code, b.ctypes.data, len(b), host=True)
        return DirectAccessHandle(blob, col) if col is not None else None

    # api/G-LeCo.cuh:1257-1334: the lookups read the device copy of the blob in place
    def directRandomAccessGPU(self, handle: DirectAccessHandle, positions) -> np.ndarray:
        return self._ra(handle.column, positions, SRC_PACKED, 0)

    # api/G-LeCo.cuh:1337-1672: this library has no host decoder; the same values come from the device
    directRandomAccessCPU = directRandomAccessGPU

    # api/G-LeCo.cuh:1674-1681
    def destroyDirectAccessHandle(self, handle: DirectAccessHandle):
        handle.column.free()
