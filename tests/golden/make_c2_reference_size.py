"""Record the compressed size that the reference's own compress reports for the 200M-value
piecewise uint64 column (seed 42: the decode benchmark's column).

Runs on a machine with a CUDA GPU and the reference harness built (``make -C oracle ref``):
the reference's stock ``LeCoGPU<uint64>::compress(values, true, &size, false)`` -- its CPU
partitioner, then its GPU fit and pack (api/G-LeCo.cuh:349-614) -- and writes

    <outdir>/c2_reference_size.json   workload, values, seed, reference_compressed_bytes

    python tests/golden/make_c2_reference_size.py [outdir]
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "g-leco_b200"))
import oracle  # noqa: E402
from glc import workloads as W  # noqa: E402

N, SEED = 200_000_000, 42


def main(outdir: str = HERE) -> None:
    if not oracle.ref_available():
        raise SystemExit("reference harness not built: make -C oracle ref")
    values = W.piecewise_linear(N, seed=SEED)
    with tempfile.TemporaryDirectory() as td:
        vp = os.path.join(td, "c2.values.bin")
        values.tofile(vp)
        t0 = time.perf_counter()
        size = oracle.ref_compress_blob(vp, "u64", "var", os.path.join(td, "c2"))
        secs = time.perf_counter() - t0
    rec = {"workload": "piecewise_u64_200M_variable", "values": N, "seed": SEED,
           "reference_compressed_bytes": size,
           "how": "LeCoGPU<unsigned long long>::compress(values, true, &size, false) from the reference's sources",
           "seconds": round(secs, 1)}
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, "c2_reference_size.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
