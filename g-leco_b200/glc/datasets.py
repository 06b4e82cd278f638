"""Dataset readers (host only): the reference benchmark driver's text and raw-binary readers
(app/BenchmarkUtils.cuh:26-104) and the SOSD binary layout of its datasets (a uint64 count, then
the values; data/download_data.sh).  Each returns a numpy array of the requested integer type,
or None where the reference's reader returns false."""
from __future__ import annotations

import os
from typing import Optional

import numpy as np


def read_text_file(path: str, dtype=np.int64) -> Optional[np.ndarray]:
    """One integer per line; whitespace around it ignored; blank and unparsable lines skipped."""
    try:
        f = open(path, "r")
    except OSError:
        return None
    out = []
    with f:
        for line in f:
            tok = line.strip()
            if not tok:
                continue
            try:
                out.append(int(tok, 10))
            except ValueError:
                continue
    info = np.iinfo(np.dtype(dtype))
    # the reference converts with a cast (wraps); keep the low bits the same way
    wrapped = [(x - info.min) % (1 << (8 * np.dtype(dtype).itemsize)) + info.min for x in out]
    return np.array(wrapped, dtype=dtype)


def read_binary_file(path: str, dtype=np.int64) -> Optional[np.ndarray]:
    """A raw little-endian array of dtype; None if its size is not a multiple of the element."""
    try:
        size = os.path.getsize(path)
    except OSError:
        return None
    if size % np.dtype(dtype).itemsize:
        return None
    return np.fromfile(path, dtype=np.dtype(dtype).newbyteorder("<")).astype(dtype, copy=False)


def read_sosd_file(path: str, dtype=np.uint64) -> Optional[np.ndarray]:
    """SOSD layout: uint64 count, then count values."""
    try:
        size = os.path.getsize(path)
    except OSError:
        return None
    if size < 8:
        return None
    with open(path, "rb") as f:
        count = int(np.frombuffer(f.read(8), "<u8")[0])
        if size - 8 != count * np.dtype(dtype).itemsize:
            return None
        return np.frombuffer(f.read(), dtype=np.dtype(dtype).newbyteorder("<")).astype(dtype)


def write_sosd_file(path: str, values: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(np.array([len(values)], "<u8").tobytes())
        f.write(np.ascontiguousarray(values).tobytes())
