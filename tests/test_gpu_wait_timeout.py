"""A bounded device-side wait that runs out is reported, and the context stays usable.

With GLC_TEST_EXPIRE_FIRST_WAIT=1 when a context is created, the consumers of that context's
next decode launch give up their first wait on a stage at once (on a healthy copy), so the launch
ends early and the error word reports a timeout.  The consumers still wait, fully bounded, for the
copy they gave up on, and the producer exits only after its own wait for a free stage runs out,
so no CTA leaves with a bulk copy in flight.  glc_sync must return GLC_ERR_TIMEOUT, and the next
decode on the same context must be bit-exact.
"""
import numpy as np
import pytest
import torch

import glc
from glc import workloads as W

pytestmark = pytest.mark.gpu


def test_run_out_wait_is_reported_and_next_decode_is_exact(monkeypatch):
    monkeypatch.setenv("GLC_TEST_EXPIRE_FIRST_WAIT", "1")
    ctx = glc.Context(0)
    monkeypatch.delenv("GLC_TEST_EXPIRE_FIRST_WAIT")
    v = W.piecewise_linear(3_000_000, seed=19, mean_segment=20_000)
    col = glc.compress_device(ctx, glc.U64, v.ctypes.data, len(v), glc.VARIABLE, host=True)
    out = torch.zeros(len(v), dtype=torch.int64, device="cuda:0")
    torch.cuda.synchronize()
    glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED)
    with pytest.raises(glc.GlcError) as err:
        ctx.sync()
    assert err.value.status == glc.ERR_TIMEOUT
    # the same context, the next launch: every value exact, no error left behind
    out.zero_()
    torch.cuda.synchronize()
    glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED)
    ctx.sync()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), v)
    pos = np.arange(0, len(v), 3, dtype=np.int32)
    got = np.zeros(len(pos), np.uint64)
    glc.random_access_into(ctx, col, pos.ctypes.data, len(pos), got.ctypes.data, host_in=True, host_out=True)
    assert np.array_equal(got, v[pos])
    col.free()
    ctx.close()
