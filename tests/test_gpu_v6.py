"""The reference's GPU partitioner mode (GLC_PART_VARIABLE_V6 / glc_partition_v6) on the device:
the same boundaries as the oracle's restatement (and as the compiled reference's own
GPUVariableLengthPartitionerV6 when its harness is built), and blobs byte-identical to the
oracle's compression of those partitions."""
import os
import tempfile

import numpy as np
import pytest

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu

NP = {glc.I32: np.int32, glc.I64: np.int64, glc.U64: np.uint64, glc.U32: np.uint32}


def _cases():
    rng = np.random.default_rng(8)
    out = []
    for n in (1, 1000, 16_384, 16_385, 70_000, 1_000_003):
        out.append((f"u64_pw_{n}", glc.U64, W.piecewise_linear(n, seed=n % 31, mean_segment=7_000)))
    out.append(("i64_ts", glc.I64, W.timestamps(400_000, seed=5)))
    amp = np.repeat(rng.integers(1, 30, 40), 16_384)
    out.append(("i32_blocks", glc.I32, (rng.integers(0, 1 << 30, len(amp)) % (1 << amp)).astype(np.int32)))
    i = np.arange(250_000, dtype=np.int64)
    out.append(("u32_line", glc.U32, (i * 40 + rng.integers(0, 1 << 9, len(i))).astype(np.uint32)))
    big = (np.uint64(1) << np.uint64(60)) + rng.integers(0, 1 << 30, 60_000).astype(np.uint64)
    out.append(("u64_direct", glc.U64, big))
    return out


@pytest.mark.parametrize("name,dt,values", _cases(), ids=[c[0] for c in _cases()])
def test_device_v6_boundaries_and_blob(oracle, name, dt, values):
    ctx = glc.Context(0)
    s, e = glc.partition_v6(ctx, values)
    os_, oe = oracle.partition_v6(values, 2048)
    assert np.array_equal(s, os_) and np.array_equal(e, oe)
    codec = glc.LeCoGPU(NP[dt])
    col, size = codec.compress(values, True, use_gpu_partitioning=True)
    want = oracle.compress(values, starts=os_, ends=oe)
    assert size == want.reported_size()
    assert glc.serialize_host(codec.ctx, col) == oracle.serialize(want)
    assert np.array_equal(codec.decompressFullFile(col), values)
    col.free()


def test_v6_base_sizes(oracle):
    ctx = glc.Context(0)
    v = W.piecewise_linear(300_000, seed=4, mean_segment=3_000)
    for base in (2, 64, 1024, 4096):
        s, e = glc.partition_v6(ctx, v, base)
        os_, oe = oracle.partition_v6(v, base)
        assert np.array_equal(s, os_) and np.array_equal(e, oe), base
    with pytest.raises(glc.GlcError):
        glc.partition_v6(ctx, v, 3)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                     "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built")
@pytest.mark.parametrize("name,dt,values", [c for c in _cases() if len(c[2]) > 16_384],
                         ids=[c[0] for c in _cases() if len(c[2]) > 16_384])
def test_reference_v6_matches_restatement(oracle, name, dt, values):
    """The reference's own GPUVariableLengthPartitionerV6 (compiled from its sources) gives the
    oracle's boundaries.  Its block values are float sums of four warp terms added by atomics in
    completion order, so two blocks whose values differ only in the last float bits could swap
    quartiles; none of these inputs has such a pair."""
    with tempfile.TemporaryDirectory() as td:
        rs, re_ = oracle.ref_partition_v6(values, td)
    os_, oe = oracle.partition_v6(values, 2048)
    assert np.array_equal(rs, os_) and np.array_equal(re_, oe)
