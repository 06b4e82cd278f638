"""Generate golden vectors from the reference implementation itself.

Runs on a machine with a CUDA GPU and the reference harness built (``make -C oracle ref``,
which compiles the reference's own headers into oracle/_ref/ref_harness).  For each seeded
input below it runs the reference's stock ``LeCoGPU<T>::compress`` (fixed TILE_SIZE = 4096
partitions, its CPU VariableLengthPartitioner, or its GPU partitioner V6 with
``use_gpu_partitioning = true``) followed by its CPU ``serialize``
(api/G-LeCo.cuh:349, :826), and stores

    tests/golden/<name>.values.npy   the input
    tests/golden/<name>.blob         the reference's version-5 blob
    tests/golden/manifest.json       dtype, mode and the compressed size the reference reported

Only the reference's compression kernels run on the GPU; none of its decoders does.

    python tests/golden/make_golden.py [outdir] [--missing]

``--missing`` generates only the cases that have no blob yet and keeps the others.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
sys.path.insert(0, os.path.join(ROOT, "g-leco_b200"))
from glc import workloads as W  # noqa: E402


def cases():
    rng = np.random.default_rng(20251203)
    i = np.arange(200_000, dtype=np.int64)
    out = []
    out.append(("c1_formula_fixed", "i32", W.plain_small(65_536, seed=42), "fixed"))
    out.append(("c1_formula_var", "i32", W.plain_small(65_536, seed=43), "var"))
    out.append(("i64_walk_fixed", "i64", np.cumsum(rng.integers(-1000, 100_000, 40_000), dtype=np.int64), "fixed"))
    out.append(("u64_piecewise_var", "u64", W.piecewise_linear(48_000, seed=7, mean_segment=6_000), "var"))
    big = (np.uint64(1) << np.uint64(40)) + i[:20_000].astype(np.uint64) * np.uint64(3)
    big[4096:8192] = (np.uint64(1) << np.uint64(60)) + rng.integers(0, 1 << 20, 4096).astype(np.uint64)
    out.append(("u64_direct_copy_fixed", "u64", big, "fixed"))
    out.append(("u32_noise_var", "u32", (i[:30_000] * 50 + rng.integers(0, 1 << 12, 30_000)).astype(np.uint32), "var"))
    out.append(("i32_short_fixed", "i32", (7 * i[:1000] - 3000 + rng.integers(0, 16, 1000)).astype(np.int32), "fixed"))
    out.append(("i64_one_fixed", "i64", np.array([-123456789012], np.int64), "fixed"))
    out.append(("i64_ts_var", "i64", W.timestamps(25_000, seed=3), "var"))
    # the GPU partitioner: sizes of 16,384-value blocks by quartile of a per-block variance
    out.append(("u64_piecewise_v6", "u64", W.piecewise_linear(120_000, seed=11, mean_segment=9_000), "v6"))
    out.append(("i64_ts_v6", "i64", W.timestamps(98_304, seed=12), "v6"))
    amp = np.repeat(np.array([1 << 4, 1 << 12, 1 << 8, 1 << 20, 1 << 2, 1 << 16]), 16_384)
    noisy = (i[:len(amp)] * 11 + rng.integers(0, 1 << 30, len(amp)) % amp).astype(np.uint32)
    out.append(("u32_blocks_v6", "u32", noisy, "v6"))
    return out


def main(outdir: str = HERE, missing_only: bool = False) -> None:
    if not os.path.exists(HARNESS):
        raise SystemExit("reference harness not built: make -C oracle ref")
    os.makedirs(outdir, exist_ok=True)
    manifest = {}
    mpath = os.path.join(outdir, "manifest.json")
    if missing_only and os.path.exists(mpath):
        with open(mpath) as f:
            manifest = json.load(f)
    for name, dt, values, mode in cases():
        if missing_only and name in manifest and os.path.exists(os.path.join(outdir, f"{name}.blob")):
            continue
        vpath = os.path.join(outdir, f"{name}.values.npy")
        np.save(vpath, values)
        raw = os.path.join(outdir, f"{name}.values.bin")
        values.tofile(raw)
        prefix = os.path.join(outdir, name)
        r = subprocess.run([HARNESS, "golden", dt, raw, prefix, mode], capture_output=True, text=True)
        os.remove(raw)
        if r.returncode != 0:
            raise SystemExit(f"{name}: reference harness failed: {r.stderr[-2000:]}")
        size = int(r.stdout.strip().splitlines()[-1])
        manifest[name] = {"dtype": dt, "mode": mode, "n": int(len(values)), "reported_size": size}
        print(name, dt, mode, len(values), size, flush=True)
    with open(os.path.join(outdir, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    main(args[0] if args else HERE, "--missing" in sys.argv)
