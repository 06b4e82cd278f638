"""Record the oracle's blobs for the 200M-value piecewise uint64 column (seed 42: the decode
benchmark's column), as SHA-256 digests: variable partitions (the oracle's restatement of the
device split/merge partitioner) and fixed partitions of 4096 values.

Runs on the CPU (about 90 s, most of it the oracle's partitioner) and writes

    <outdir>/c2_oracle_blobs.json   per mode: partitions, reported size, blob bytes, blob SHA-256

    python tests/golden/make_c2_oracle_blobs.py [outdir]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "g-leco_b200"))
import oracle  # noqa: E402
from glc import workloads as W  # noqa: E402

N, SEED = 200_000_000, 42


def main(outdir: str = HERE) -> None:
    values = W.piecewise_linear(N, seed=SEED)
    rec = {"workload": "piecewise_u64_200M", "values": N, "seed": SEED}
    for mode in ("variable", "fixed4096"):
        t0 = time.perf_counter()
        if mode == "variable":
            s, e = oracle.partition_variable(values)
            col = oracle.compress(values, starts=s, ends=e)
        else:
            col = oracle.compress(values, "fixed", 4096)
        blob = oracle.serialize(col)
        rec[mode] = {"partitions": int(col.num_partitions),
                     "reported_size": col.reported_size(), "blob_bytes": len(blob),
                     "blob_sha256": hashlib.sha256(blob).hexdigest(),
                     "seconds": round(time.perf_counter() - t0, 1)}
        del blob, col
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, "c2_oracle_blobs.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
