"""glc_decompress_range_noalloc: the allocation-free range decode into host memory.

For callers that cannot allocate device memory while they run (fixed device-memory budgets,
code that must not block on the allocator).  The entry point keeps the decode kernel's scratch
and the staging of the values in one static device array, so this test checks, through the C
ABI, that its output equals the regular glc_decompress_range with a host output, on two calls
in a row (the second call must not see the first call's scratch), that the device's free memory
does not change across those calls, and that a range larger than the array is refused.  Results
are integers, so the comparison is exact.
"""
import numpy as np
import pytest
import torch

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu


def _reference_range(codec, col, first, count, dtype):
    out = np.empty(count, dtype)
    glc.decompress_range_into(codec.ctx, col, first, count, out.ctypes.data, glc.SRC_PACKED, host_out=True)
    return out


@pytest.mark.parametrize("dtype", [np.uint64, np.int32])
def test_noalloc_range_decode_matches_regular_entry_point(dtype):
    n = 2_000_000
    v = W.piecewise_linear(n, seed=21) if dtype == np.uint64 else W.plain_small(n, seed=21)
    codec = glc.LeCoGPU(dtype, device=0)
    col, _ = codec.compress(v, True)
    max_count = glc.NOALLOC_MAX_OUTPUT_BYTES // np.dtype(dtype).itemsize
    # a first call looks up the static array and loads the kernel; after it, the device's free
    # memory must not change across further calls (nothing is allocated)
    assert glc.decompress_range_noalloc(col, 0, 1000, np.zeros(1000, dtype)) == glc.OK
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    # two calls in a row: a large range, then a smaller one at an odd offset
    calls = [(123_457, max_count), (1_500_001, 777)]
    got = [np.full(count, 7, dtype) for _, count in calls]
    for (first, count), g in zip(calls, got):
        assert glc.decompress_range_noalloc(col, first, count, g) == glc.OK
    assert torch.cuda.mem_get_info(0)[0] == free_before
    for (first, count), g in zip(calls, got):
        want = _reference_range(codec, col, first, count, dtype)
        assert np.array_equal(g, want)
        assert np.array_equal(g, v[first:first + count])
    # a caller's buffer that is too short or of the wrong element size is refused before the call
    with pytest.raises(ValueError):
        glc.decompress_range_noalloc(col, 0, 10, np.zeros(9, dtype))
    with pytest.raises(ValueError):
        glc.decompress_range_noalloc(col, 0, 10, np.zeros(10, np.int16))
    # larger than the static array: refused with a clear status, nothing written
    big = np.zeros(max_count + 1, dtype)
    assert glc.decompress_range_noalloc(col, 0, max_count + 1, big) == glc.ERR_INVALID_ARG
    assert not big.any()
    # out of range and empty requests
    assert glc.decompress_range_noalloc(col, n - 5, 10, np.zeros(10, dtype)) == glc.ERR_INVALID_ARG
    assert glc.decompress_range_noalloc(col, 5, 0, np.zeros(1, dtype)) == glc.OK
