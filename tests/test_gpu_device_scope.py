"""Every entry point leaves the calling thread's current device as it found it.

A host thread that drives several GPUs keeps its own current device across calls into the
library, whichever device the context, column, batch or server lives on.  The calls run from a
fresh host thread whose current device is set to one index while the context lives on another
(the last device; with a single GPU both are device 0, and the test then checks that nothing
moves the thread off it).
"""
import threading

import numpy as np
import pytest
import torch

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu


def test_entry_points_restore_the_callers_device():
    ndev = torch.cuda.device_count()
    ctx_dev, caller_dev = ndev - 1, 0
    errors = []

    def body():
        try:
            torch.cuda.set_device(caller_dev)
            codec = glc.LeCoGPU(np.uint64, device=ctx_dev)
            ctx = codec.ctx
            assert torch.cuda.current_device() == caller_dev
            v = W.piecewise_linear(300_000, seed=2)
            col, _ = codec.compress(v, True)
            assert torch.cuda.current_device() == caller_dev
            assert np.array_equal(codec.decompressFullFile(col), v)
            pos = np.arange(0, len(v), 997, dtype=np.int32)
            assert np.array_equal(codec.decompress(col, pos), v[pos])
            blob = codec.serialize(col)
            col2 = codec.deserializeGPU(blob, True)
            ctx.sync()
            out = np.zeros(1000, np.uint64)
            assert glc.decompress_range_noalloc(col, 5, 1000, out) == glc.OK and np.array_equal(out, v[5:1005])
            assert torch.cuda.current_device() == caller_dev
            col2.free()
            col.free()
            ctx.close()
            assert torch.cuda.current_device() == caller_dev
        except Exception as ex:  # reported to the test's thread
            errors.append(ex)

    t = threading.Thread(target=body)
    t.start()
    t.join()
    assert not errors, errors
