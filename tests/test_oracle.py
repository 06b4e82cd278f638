"""CPU tests of the oracle itself: arithmetic primitives, format rules and round trips."""
import random
import struct

import numpy as np
import pytest

from glc import workloads as W


def _split128(v: int):
    u = v & ((1 << 128) - 1)
    hi = u >> 64
    if hi >= 1 << 63:
        hi -= 1 << 64
    return hi, u & ((1 << 64) - 1)


def test_i128_to_double_is_correctly_rounded(oracle):
    rng = random.Random(1)
    cases = [0, 1, -1, 2 ** 53 + 1, 2 ** 64, 2 ** 64 + 2 ** 11, 2 ** 64 + 2 ** 11 + 1, 2 ** 64 + 3 * 2 ** 11,
             -(2 ** 100) - 12345, 2 ** 126 - 1, -(2 ** 127)]
    cases += [rng.randrange(-(2 ** 127), 2 ** 127) for _ in range(2000)]
    cases += [rng.randrange(-(2 ** 70), 2 ** 70) for _ in range(2000)]
    for v in cases:
        hi, lo = _split128(v)
        assert oracle.lib().orc_i128_to_double(hi, lo) == float(v), v  # Python rounds ints half-even


def test_solve_line_recovers_exact_lines(oracle):
    import ctypes
    for n in (2, 3, 17, 1000, 4096, 50_000):
        x = np.arange(n, dtype=object)
        y = 7 + 3 * x
        sy, sxy = int(sum(y)), int(sum(x * y))
        t0, t1 = ctypes.c_double(), ctypes.c_double()
        oracle.lib().orc_solve_line(n, *_split128(sy), *_split128(sxy), ctypes.byref(t0), ctypes.byref(t1))
        assert t1.value == 3.0 and t0.value == 7.0


def _rotate_add(data: bytes) -> int:
    c = 0
    for b in data:
        c = (c + b) & 0xFFFFFFFF
        c = ((c << 1) | (c >> 31)) & 0xFFFFFFFF
    return c


def _crc32c_table(data: bytes, init: int = 0) -> int:
    table = []
    for i in range(256):
        c = i
        for _ in range(8):
            c = (c >> 1) ^ (0x82F63B78 if c & 1 else 0)
        table.append(c)
    c = init
    for b in data:
        c = table[(c ^ b) & 0xFF] ^ (c >> 8)
    return c


def test_header_checksums(oracle):
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 120, 1000):
        data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert oracle.checksum(data) == _rotate_add(data)
        assert oracle.checksum(data, crc32c=True) == _crc32c_table(data)
    # standard CRC-32C check value (init and final xor 0xFFFFFFFF) of "123456789" is 0xE3069283
    assert _crc32c_table(b"123456789", 0xFFFFFFFF) ^ 0xFFFFFFFF == 0xE3069283


def _cases():
    rng = np.random.default_rng(7)
    i = np.arange(30_000, dtype=np.int64)
    yield "i32", (1000 * i[:20_000] + rng.integers(0, 256, 20_000)).astype(np.int32)
    yield "i32neg", (-37 * i[:9_000] + rng.integers(-5000, 5000, 9_000)).astype(np.int32)
    yield "i64walk", np.cumsum(rng.integers(-1000, 100000, 30_000), dtype=np.int64)
    ext = rng.integers(-(2 ** 62), 2 ** 62, 5_000, dtype=np.int64)
    ext[::7] = np.iinfo(np.int64).max
    ext[3::11] = np.iinfo(np.int64).min
    yield "i64ext", ext
    yield "u64pw", W.piecewise_linear(40_000, seed=3, mean_segment=3_000)
    big = (np.uint64(1) << np.uint64(60)) + rng.integers(0, 1000, 7_000).astype(np.uint64)
    big[:3000] = np.arange(3000, dtype=np.uint64) * np.uint64(5)
    yield "u64big", big
    yield "u32", (i[:12_345] * 50 + rng.integers(0, 1 << 12, 12_345)).astype(np.uint32)
    yield "u32const", np.full(5000, 4_000_000_000, np.uint32)
    yield "one", np.array([42], np.int64)


@pytest.mark.parametrize("name,values", list(_cases()))
@pytest.mark.parametrize("mode,L", [("fixed", 1024), ("fixed", 4096), ("fixed", 7), ("variable", 0)])
def test_oracle_round_trips(oracle, name, values, mode, L):
    col = oracle.compress(values, mode, L or 4096)
    assert np.array_equal(oracle.decode_full(col), values)
    pos = np.random.default_rng(1).integers(0, len(values), 3000).astype(np.int32)
    assert np.array_equal(oracle.random_access(col, pos), values[pos])
    plain = oracle.unpack_deltas(col)
    assert np.array_equal(oracle.decode_preunpacked(col, plain), values)
    blob = oracle.serialize(col)
    back = oracle.deserialize(blob, col.dtype)
    assert np.array_equal(oracle.decode_full(back), values)
    assert oracle.serialize(back) == blob
    # partitions cover [0, n) contiguously; offsets are the prefix of len*bits
    assert col.starts[0] == 0 and col.ends[-1] == len(values)
    assert np.array_equal(col.starts[1:], col.ends[:-1])
    w = (col.ends - col.starts).astype(np.int64) * col.bits
    assert np.array_equal(col.offsets, np.concatenate([[0], np.cumsum(w)[:-1]]))


def test_direct_copy_rule(oracle):
    v = np.array([1 << 53, (1 << 53) + 1, 5], np.uint64)
    col = oracle.compress(v, "fixed", 2)
    assert col.types.tolist() == [oracle.MODEL_DIRECT_COPY, oracle.MODEL_LINEAR]  # only > 2^53 overflows
    assert col.bits[0] == 64 and col.params[0] == 0.0 and col.params[1] == 0.0


def test_llong_min_residual_gets_a_full_width_field(oracle):
    v = np.array([0, 0, np.iinfo(np.int64).min, 0], np.int64)
    col = oracle.column_with_lines(v, [0], [4], [(0.0, 0.0)])
    assert col.bits[0] == 64
    assert np.array_equal(oracle.decode_full(col), v)


def test_ties_round_half_away_from_zero(oracle):
    n = 1000
    v = (np.arange(n) + 1).astype(np.int64)  # round(i + 0.5) = i + 1: zero residuals
    col = oracle.column_with_lines(v, [0], [n], [(0.5, 1.0)])
    assert col.bits[0] == 0
    assert np.array_equal(oracle.decode_full(col), v)
    v2 = (np.arange(n) - 1).astype(np.int64)  # round(i - 0.5): -1 at i=0 (away from zero), then i
    col2 = oracle.column_with_lines(v2, [0], [n], [(-0.5, 1.0)])
    assert np.array_equal(oracle.decode_full(col2), v2)
    assert col2.bits[0] == 2  # residual -1 at i >= 1, 0 at i = 0


def test_blob_layout(oracle):
    v = W.plain_small(10_001, seed=5)
    col = oracle.compress(v, "fixed", 1000)
    blob = oracle.serialize(col)
    hdr = struct.unpack("<4I10Q2I3I4x", blob[:120])
    magic, version, total, P = hdr[:4]
    offs = hdr[4:12]
    assert (magic, version, total, P) == (0x4F43454C, 5, 10_001, 11)
    assert all(o % 8 == 0 for o in offs) and list(offs) == sorted(offs)
    assert len(blob) % 8 == 0
    assert hdr[12] == 32 * P and hdr[13] == (col.total_bits + 7) // 8 and hdr[14] == 4
    zeroed = bytearray(blob[:120])
    zeroed[100:104] = b"\0\0\0\0"
    assert hdr[15] == _rotate_add(bytes(zeroed))
    assert len(blob) == oracle.lib().orc_blob_size(P, col.total_bits)


def test_bad_blobs(oracle):
    v = W.plain_small(5000, seed=1)
    blob = oracle.serialize(oracle.compress(v, "fixed", 1024))
    with pytest.raises(oracle.BlobError):
        oracle.deserialize(blob[:119], "i32")
    with pytest.raises(oracle.BlobError):
        oracle.deserialize(blob, "i64")
    for off in (0, 4, 20, 96):
        b = bytearray(blob)
        b[off] ^= 1
        with pytest.raises(oracle.BlobError):
            oracle.deserialize(bytes(b), "i32")
    with pytest.raises(oracle.BlobError):
        oracle.deserialize(blob[:-16], "i32")


def test_split_rule_first_minimum(oracle):
    """Best end of a start follows the reference's size ladder and keeps the first minimum."""
    v = np.arange(10_000, dtype=np.int64) * 3  # exact line: every size costs 0 bits, 80 B model
    # cost per value 80/size is smallest for the largest size 3712
    assert oracle.split_best_end(v, 0) == 3712
    assert oracle.split_best_end(v, 9984) == 10_000  # fewer than 128 left: the rest


def test_variable_partitions_structure(oracle):
    v = W.piecewise_linear(500_000, seed=2, mean_segment=20_000)
    s, e = oracle.partition_variable(v)
    assert s[0] == 0 and e[-1] == len(v) and np.array_equal(s[1:], e[:-1])
    assert np.all(s % 128 == 0)
    assert np.all((e - s)[:-1] >= 128)


@pytest.mark.parametrize("gen", ["c1", "piecewise"])
def test_variable_size_within_one_percent_of_reference_partitioner(oracle, gen):
    v = W.plain_small(1 << 20) if gen == "c1" else W.piecewise_linear(1_000_000, seed=9)
    s, e = oracle.ref_partition_cpu(v)
    ref = oracle.compress(v, starts=s, ends=e).reported_size()
    ours = oracle.compress(v, "variable").reported_size()
    assert ours <= 1.01 * ref, (ours, ref)
    assert ours >= 0.9 * ref, (ours, ref)


def test_half_away_rounding_identity():
    """The device predicts round-half-away(x) as trunc(x + copysign(0.5 - 2^-54, x)) folded into a
    truncating conversion; check the identity against exact rounding (x - trunc(x) is exact)."""
    rng = np.random.default_rng(0)
    bias = np.nextafter(0.5, 0.0)
    ties = rng.integers(-(2 ** 53), 2 ** 53, 500_000) / 2.0
    xs = np.concatenate([rng.standard_normal(500_000) * 10.0 ** rng.integers(-3, 18, 500_000), ties,
                         np.nextafter(ties, np.inf), np.nextafter(ties, -np.inf),
                         [0.5, -0.5, 0.49999999999999994, -0.49999999999999994, 2.4999999999999996,
                          4503599627370495.5, 2.0 ** 53, 2.0 ** 63, -(2.0 ** 63), 0.0, -0.0]])
    t = np.trunc(xs)
    exact = np.where(np.abs(xs - t) >= 0.5, t + np.sign(xs), t)
    assert np.array_equal(np.trunc(xs + np.copysign(bias, xs)), exact)


def test_v6_partitions_follow_sorted_ranks(oracle):
    """The reference's GPU partitioner sizes block i by the i-th SMALLEST block value (it sorts the
    value array in place before the partition kernel reads it): with distinct values the blocks
    get 8192, 4096, 2048, 1024 by position quartile, whatever their own variance; ties (constant
    data) push every block into the 1024 class."""
    rng = np.random.default_rng(4)
    amps = [1 << 20, 1 << 4, 1 << 12, 1 << 8]  # block k's noise amplitude: values all distinct
    v = np.concatenate([rng.integers(0, a, 16_384) for a in amps]).astype(np.int64)
    var = oracle.v6_variances(v, 2048)
    assert len(var) == 4 and len(set(var.tolist())) == 4
    s, e = oracle.partition_v6(v, 2048)
    assert s[0] == 0 and e[-1] == len(v) and np.array_equal(s[1:], e[:-1])
    for b, size in enumerate((8192, 4096, 2048, 1024)):
        inside = (s >= 16_384 * b) & (s < 16_384 * (b + 1))
        assert np.all(e[inside] - s[inside] == size), b
    s, e = oracle.partition_v6(np.full(4 * 16_384, 77, np.int64), 2048)
    assert np.all(e - s == 1024)


@pytest.mark.parametrize("n", [1, 1000, 16_384, 16_385, 50_000, 300_001])
def test_v6_partitions_cover_the_column(oracle, n):
    v = W.piecewise_linear(n, seed=n % 97, mean_segment=5_000)
    s, e = oracle.partition_v6(v, 2048)
    assert s[0] == 0 and e[-1] == n and np.array_equal(s[1:], e[:-1])
    sizes = e - s
    assert np.all(np.isin(sizes[:-1], [1024, 2048, 4096, 8192]) | ((e[:-1] % 16_384) == 0))
    col = oracle.compress(v, starts=s, ends=e)
    assert np.array_equal(oracle.decode_full(col), v)
