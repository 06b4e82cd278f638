"""The C-ABI library loads and exports exactly what include/glc.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

import glc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "glc.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"GLC_API\s+[\w\s\*]+?\b(glc_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = _declared()
    assert names == sorted(glc.EXPORTS), names


def test_library_loads_and_exports_every_symbol():
    lib = glc.load()
    for name in _declared():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value


def test_status_strings_without_a_device():
    lib = glc.load()
    assert lib.glc_status_string(glc.OK) == b"ok"
    assert lib.glc_status_string(glc.ERR_BAD_BLOB) == b"bad blob"
    assert lib.glc_last_error(None) == b"no context"


def test_null_arguments_are_rejected_without_touching_the_device():
    lib = glc.load()
    assert lib.glc_create(None, 0) == glc.ERR_INVALID_ARG
    assert lib.glc_column_free(None) == glc.ERR_INVALID_ARG
    assert lib.glc_compress(None, 0, None, 0, 0, 0, 0, None, None, None) == glc.ERR_INVALID_ARG


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(glc.GlcError):
        glc.Context(0)


def test_server_entry_points_reject_null_arguments():
    lib = glc.load()
    assert lib.glc_server_create(None, None, None) == glc.ERR_INVALID_ARG
    assert lib.glc_server_submit(None, None, 1) == glc.ERR_INVALID_ARG
    assert lib.glc_server_destroy(None) == glc.ERR_INVALID_ARG
    assert lib.glc_server_drain(None, 0) == glc.ERR_INVALID_ARG
    t0 = lib.glc_server_now_ns()
    assert lib.glc_server_now_ns() >= t0 > 0


def test_tuning_entry_points_reject_null_arguments():
    lib = glc.load()
    assert lib.glc_autotune(None, None, 0) == glc.ERR_INVALID_ARG
    assert lib.glc_tune_get(None, 0, 8, 0, None) == glc.ERR_INVALID_ARG
    assert lib.glc_tune_set(None, 0, 8, 0, None) == glc.ERR_INVALID_ARG
