"""Pins of the oracle against the reference implementation itself.

* The reference's VariableLengthPartitioner and its host decoder directRandomAccessCPU,
  compiled from the reference's own sources into oracle/_ref/ref_harness (oracle/Makefile),
  must agree with the oracle's restatements.
* tests/golden/ holds blobs that the reference's stock compress + serialize produced for
  seeded inputs (tests/golden/make_golden.py); the oracle must decode them to the input and
  reproduce their layout.
"""
import json
import os

import numpy as np
import pytest

from glc import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _need_ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness not built (make -C oracle ref)")


def _inputs():
    rng = np.random.default_rng(11)
    i = np.arange(400_000, dtype=np.int64)
    yield "c1", W.plain_small(1 << 20)
    yield "pw", W.piecewise_linear(400_000, seed=4, mean_segment=8_000)
    yield "walk", np.cumsum(rng.integers(-50, 5000, 200_000), dtype=np.int64)
    yield "u32", (i[:150_000] * 9 + rng.integers(0, 300, 150_000)).astype(np.uint32)
    yield "ts", W.timestamps(100_000, seed=8)
    yield "short", (3 * i[:300]).astype(np.int32)
    yield "tiny", np.array([5, 9, 13], np.int64)


@pytest.mark.parametrize("name,values", list(_inputs()))
def test_reference_partitioner_matches_restatement(oracle, tmp_path, name, values):
    _need_ref(oracle)
    rs, re_, rb = oracle.ref_partition(values, str(tmp_path))
    s, e = oracle.ref_partition_cpu(values)
    assert np.array_equal(rs, s) and np.array_equal(re_, e)


@pytest.mark.parametrize("name,values", list(_inputs()))
@pytest.mark.parametrize("mode", ["fixed", "variable"])
def test_reference_host_decoder_reads_oracle_blobs(oracle, tmp_path, name, values, mode):
    _need_ref(oracle)
    col = oracle.compress(values, mode, 1024)
    blob = oracle.serialize(col)
    pos = np.arange(len(values), dtype=np.int32)
    out, _ = oracle.ref_hostdecode(blob, col.dtype, pos, str(tmp_path))
    # the reference's host decoder computes theta0 + theta1*i without fma, so where the two
    # predictions round to different integers (a .5 tie on one side) it returns a value that
    # differs from the input by one.  The oracle's restatement of that decoder must give its
    # output exactly, so every mismatch is one the oracle predicts.
    assert np.array_equal(out, oracle.decode_variant(col, pos, oracle.PRED_HOST))
    mism = np.flatnonzero(out != values)
    predicted = np.flatnonzero(oracle.decode_variant(col, pos, oracle.PRED_HOST)
                               != oracle.decode_variant(col, pos, oracle.PRED_CONTRACT))
    assert np.array_equal(mism, predicted)


def test_reference_host_decoder_direct_copy(oracle, tmp_path):
    _need_ref(oracle)
    v = (np.uint64(1) << np.uint64(60)) + np.arange(5000, dtype=np.uint64) * np.uint64(7)
    v[:2000] = np.arange(2000, dtype=np.uint64)
    col = oracle.compress(v, "fixed", 1000)
    out, _ = oracle.ref_hostdecode(oracle.serialize(col), "u64", np.arange(5000, dtype=np.int32), str(tmp_path))
    assert np.array_equal(out, v)


def _golden():
    path = os.path.join(GOLDEN, "manifest.json")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        man = json.load(f)
    return sorted(man.items())


@pytest.mark.parametrize("name,meta", _golden() or [pytest.param("none", {}, marks=pytest.mark.skip("no fixtures"))])
def test_golden_reference_blobs(oracle, name, meta):
    values = np.load(os.path.join(GOLDEN, f"{name}.values.npy"))
    with open(os.path.join(GOLDEN, f"{name}.blob"), "rb") as f:
        blob = f.read()
    col = oracle.deserialize(blob, meta["dtype"])
    # (1) the oracle decodes the reference's blob to the input, bit for bit
    assert np.array_equal(oracle.decode_full(col), values)
    # (2) the blob layout is the oracle's: same header and byte size for the same P and bits
    assert col.reported_size() == meta["reported_size"]
    # (3) same partitions as the oracle's restatement of the reference's partitioning
    if meta["mode"] == "fixed":
        s, e = oracle.partition_fixed(len(values), 4096)
    elif meta["mode"] == "v6":  # the reference's GPU partitioner (compress, use_gpu_partitioning)
        s, e = oracle.partition_v6(values, 2048)
    else:
        s, e = oracle.ref_partition_cpu(values)
    assert np.array_equal(col.starts, s) and np.array_equal(col.ends, e)
    # (4) compressing the same partitions with the oracle's fit gives the same layout and a size
    #     within 1% (theta is a summation-order artefact, so bit widths may differ by one)
    mine = oracle.compress(values, starts=s, ends=e)
    assert np.array_equal(mine.types, col.types)
    assert np.mean(mine.bits == col.bits) >= 0.95
    assert abs(mine.reported_size() - meta["reported_size"]) <= 0.01 * meta["reported_size"]
    assert oracle.serialize(col) == blob
