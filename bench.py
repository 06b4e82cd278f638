"""Headline benchmark: full decode of a variable-partitioned 200M uint64 piecewise-linear column.

One step = one full decode of the column (persistent work-stealing kernel, TMA-staged input).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl glc|reference] [--n VALUES]

Workload (``config.workload``): 200,000,000 uint64 values, piecewise linear with segment
lengths ~ Poisson(50,000), slope U{1..10^6}, intercept jump U{0..2^40}, noise U[0, 2^b) with
b in {0,4,8,16,24} (seeded synthetic data standing in for the reference's SOSD datasets),
compressed with the device split/merge partitioner.  The compressed column and the output are
both larger than L2 (126 MB), so no L2 flush is needed between steps.

``value`` = decoded bytes (8 B x values, the reference's decode GB/s definition, app/Main.cu)
/ device time, inputs resident in HBM.  ``e2e`` = the same through the public C ABI with host
buffers: every step deserializes the host (pinned) blob onto the device and decodes into pinned
host memory.  ``roofline`` = algorithmic bytes (compressed bytes read + decoded bytes written)
per decode launch / its CUDA-event duration, against the measured HBM copy bandwidth.

With N > 1 (torchrun, one process per GPU) every rank decodes its own column (columns are
independent; no data-path collective): weak scaling, value = all ranks' bytes / max rank time.

``--impl reference`` times the reference's own CPU decoder (directRandomAccessCPU, compiled from
the reference sources into oracle/_ref; the CPU oracle when that is absent) on this host's cores
over bounded samples of the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "g-leco_b200"))

METRIC = "decode GB/s"
UNIT = "GB/s"
WORKLOAD = "piecewise_u64_200M_variable"
DEFAULT_N = 200_000_000
PROFILE_NOTE = os.path.join(ROOT, "profiles", "decode_piecewise_u64_200M.md")


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic_per_value():
    """DRAM bytes per decoded value from the committed ncu summary (one capture), or None."""
    try:
        with open(PROFILE_NOTE) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_value:"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


_SAMPLER = r"""
import sys, time, pynvml
pynvml.nvmlInit()
uuid, index = sys.argv[1], int(sys.argv[2])
try:
    h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
except Exception:
    h = pynvml.nvmlDeviceGetHandleByIndex(index)
get = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
print("max", pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM), flush=True)
while True:
    print(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), int(get(h)), flush=True)
    time.sleep(0.002)
"""


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of the benchmarked GPU, sampled through NVML
    every 2 ms by a separate process while the timed region runs (reads only; no GPU setting is
    changed)."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device):
        self.dev = torch_device
        self.proc = None

    def start(self):
        import torch
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            uuid = ""
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        idx = self.dev.index or 0
        if vis and vis.split(",")[0].strip().isdigit():
            idx = int(vis.split(",")[idx])
        self.proc = subprocess.Popen([sys.executable, "-c", _SAMPLER, uuid, str(idx)], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True)
        self.max_line = self.proc.stdout.readline()  # the sampler is up before the timed region starts

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": "sampler not started"}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, reasons = [], set()
        for ln in out.splitlines():
            parts = ln.split()
            if len(parts) != 2:
                continue
            sm.append(float(parts[0]))
            for bit, name in self.REASONS.items():
                if int(parts[1]) & bit:
                    reasons.add(name)
        try:
            smax = float(self.max_line.split()[1])
        except Exception:
            smax = None
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "NVML every 2 ms (separate process)"}


def make_values(n: int, rank: int) -> np.ndarray:
    from glc import workloads as W
    return W.piecewise_linear(n, seed=42 + rank)


def cpu_baseline_decode(values: np.ndarray, blob_maker, threads: int, budget_s: float = 20.0):
    """Time the reference's host decoder on a bounded prefix sample; returns a dict."""
    import oracle
    sample_n = min(len(values), 16_000_000)
    sample = np.ascontiguousarray(values[:sample_n])
    blob = blob_maker(sample)
    pos = np.arange(sample_n, dtype=np.int32)
    kind = "reference" if oracle.ref_available() else "port"
    with tempfile.TemporaryDirectory() as td:
        if kind == "reference":
            chunks = np.array_split(pos, threads)
            paths = []
            for k, ch in enumerate(chunks):
                pp = os.path.join(td, f"pos{k}.bin")
                ch.tofile(pp)
                paths.append(pp)
            bp = os.path.join(td, "blob.bin")
            with open(bp, "wb") as f:
                f.write(blob)
            env = dict(os.environ, GLC_REF_CPU_ONLY="1")
            t0 = time.perf_counter()
            procs = [subprocess.Popen([oracle.REF_HARNESS, "hostdecode", "u64", bp, paths[k],
                                       os.path.join(td, f"out{k}.bin"), "1"], stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, env=env) for k in range(len(paths))]
            for p in procs:
                p.wait()
            wall = time.perf_counter() - t0
            secs = max(float(p.stdout.read().decode().strip().splitlines()[-1]) for p in procs)
            out = np.concatenate([np.fromfile(os.path.join(td, f"out{k}.bin"), np.uint64) for k in range(len(paths))])
            mism = int(np.count_nonzero(out != sample))
        else:
            col = oracle.deserialize(blob, "u64")
            t0 = time.perf_counter()
            out = oracle.decode_full(col)
            secs = time.perf_counter() - t0
            wall = secs
            mism = int(np.count_nonzero(out != sample))
            threads = 1
    gbs = sample_n * 8 / secs / 1e9
    return {"value": round(gbs, 4), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"full decode of the first {sample_n:,} values of the workload (all positions, "
                      f"{'directRandomAccessCPU' if kind == 'reference' else 'oracle decode'}), "
                      f"{threads} process(es); wall {wall:.2f} s; values differing from the input: {mism} "
                      f"(the reference's host decoder predicts without fma)"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    n = min(args.n, 200_000_000)
    threads = os.cpu_count() or 1
    values = make_values(min(n, 16_000_000), 0)
    # blob of the sample: the reference's own CPU partitioner (restated) and the format's fit
    def make_blob(sample):
        s, e = oracle.ref_partition_cpu(sample)
        return oracle.serialize(oracle.compress(sample, starts=s, ends=e))
    blob = make_blob(values)
    maker = lambda sample: blob  # noqa: E731
    results = []
    for step in range(args.warmup + args.steps):
        r = cpu_baseline_decode(values, maker, threads)
        if step >= args.warmup:
            results.append(r)
    val = float(np.median([r["value"] for r in results]))
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "values": n, "sample_values": len(values)},
            "cpu_baseline": {**results[-1], "value": val},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_random_access(args):
    """Random access: 64M int64 timestamps (cumulative exponential gaps, mean 1000), fixed
    partitions of 4096, 100M positions (half uniform, half Zipf(1.1) over partitions).  One step
    = one launch answering all positions; value = lookups per second.  Roofline bytes per lookup:
    4 B position + 8 B value + one 32 B DRAM sector holding the field (44 B)."""
    import torch

    import glc
    from glc import workloads as W

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = glc.Context(local)
    n = min(args.n, 64 * 1024 * 1024) if args.n != DEFAULT_N else 64 * 1024 * 1024
    q = args.queries
    L = 4096
    values = W.timestamps(n, seed=42)
    pos = W.lookup_positions(n, q, L, seed=42)
    d_vals = torch.from_numpy(values).to(dev)
    col = glc.compress_device(ctx, glc.I64, d_vals.data_ptr(), n, glc.FIXED, fixed_len=L, stream=sh)
    src = glc.SRC_PACKED
    if args.mode == "preunpacked":
        glc.preunpack(ctx, col, stream=sh)
        src = glc.SRC_PREUNPACKED
    info = col.info()
    d_pos = torch.from_numpy(pos).to(dev)
    out = torch.empty(q, dtype=torch.int64, device=dev)

    def step():
        glc.random_access_into(ctx, col, d_pos.data_ptr(), q, out.data_ptr(), source=src, fixed_len=L, stream=sh)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ok = bool(torch.equal(out, d_vals[d_pos.long()]))
    clocks = ClockSampler(dev)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    lookups_s = q / (ms / 1e3)
    per_lookup = 4 + 8 + 32
    peak, peak_kind = measured_peak()
    achieved = per_lookup * lookups_s / 1e9
    # end to end: pinned host positions in, pinned host values out, through the C ABI
    h_pos = torch.from_numpy(pos).pin_memory()
    h_out = torch.empty(q, dtype=torch.int64).pin_memory()

    def e2e_step():
        glc.random_access_into(ctx, col, h_pos.data_ptr(), q, h_out.data_ptr(), source=src, fixed_len=L,
                               stream=sh, host_in=True, host_out=True)

    e2e_step()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
    e2e_ok = bool(np.array_equal(h_out.numpy(), values[pos]))
    cpu = None
    if not args.no_cpu_baseline:
        import oracle
        try:
            blob = glc.serialize_host(ctx, col) if args.mode == "packed" else None
            if blob is None:
                raise RuntimeError("pre-unpacked columns have no host decoder in the reference")
            sample = pos[:2_000_000]
            with tempfile.TemporaryDirectory() as td:
                got, secs = oracle.ref_hostdecode(blob, "i64", sample, td)
            cpu = {"value": round(len(sample) / secs, 1), "unit": "lookups/s", "cores": 1,
                   "kind": "reference" if oracle.ref_available() else "port",
                   "sample": f"{len(sample):,} of the positions through directRandomAccessCPU; "
                             f"mismatches vs input: {int(np.count_nonzero(got != values[sample]))}"}
        except Exception as ex:
            cpu = {"value": None, "unit": "lookups/s", "cores": 1, "kind": "reference", "sample": f"skipped: {ex}"}
    line = {
        "metric": "random lookups/s", "value": round(lookups_s, 1), "unit": "lookups/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": f"timestamps_i64_64M_fixed4096_lookups100M_{args.mode}", "values": n, "lookups": q,
                   "partitions": info.num_partitions, "bits_per_value": round(info.total_bits / n, 3),
                   "position_mix": "50% uniform, 50% Zipf(1.1) over partitions", "bit_exact": ok and e2e_ok,
                   "l2": "positions and outputs larger than L2 (no flush)"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "bytes_per_lookup": per_lookup},
        "e2e": {"value": round(q / (e2e_ms / 1e3), 1), "unit": "lookups/s", "h2d_bytes_per_step": 4 * q,
                "d2h_bytes_per_step": 8 * q},
        "gpu_launches": args.steps, "clocks": clk, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    col.free()
    ctx.close()
    return 0


def batch_columns(ncols: int, total_bytes: float, seed: int = 42):
    """Column specs of the batched workload: log-normal lengths (median 256K before scaling,
    sigma 1.0, clipped to [1K, 16M]) scaled so the raw total is about total_bytes; dtype uniform
    over int32/int64/uint64; values intercept + slope*i + noise, slope U[0, 10^4] (int32 columns:
    capped so the column stays inside int32), noise U[0, 2^w) with w U{0..20}."""
    rng = np.random.default_rng(seed)
    lens = np.clip(rng.lognormal(np.log(262_144), 1.0, ncols), 1024, 16_777_216)
    dts = rng.integers(0, 3, ncols)  # 0 int32, 1 int64, 2 uint64
    size = np.where(dts == 0, 4, 8)
    lens = np.clip((lens * total_bytes / float(np.sum(lens * size))).astype(np.int64), 1024, 16_777_216)
    specs = []
    for c in range(ncols):
        n = int(lens[c])
        slope = int(rng.integers(0, 10_001))
        if dts[c] == 0:
            slope = min(slope, (2 ** 30) // max(n, 1))
        specs.append((int(dts[c]), n, slope, int(rng.integers(0, 1 << 20)), int(rng.integers(0, 21)), 42 + c))
    return specs


def run_batch(args):
    """Batched multi-column: compress and fully decode thousands of columns of mixed dtype in one
    persistent launch (replayed from a CUDA graph), against a per-column launch loop."""
    import torch

    import glc

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = glc.Context(local)
    code = {0: glc.I32, 1: glc.I64, 2: glc.U64}
    specs = batch_columns(args.columns, 2.5e9 if args.n == DEFAULT_N else float(args.n))
    gen = torch.Generator(device=dev)
    cols, raw_bytes = [], 0
    for dt, n, slope, icpt, w, seed in specs:
        gen.manual_seed(seed)
        i = torch.arange(n, device=dev, dtype=torch.int64)
        v = icpt + slope * i
        if w:
            v = v + torch.randint(0, 1 << w, (n,), device=dev, generator=gen, dtype=torch.int64)
        v = v.to(torch.int32) if dt == 0 else v
        cols.append(v)
        raw_bytes += v.numel() * v.element_size()
    dtypes = [code[dt] for dt, *_ in specs]
    ns = [n for _, n, *_ in specs]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # batched compress (partition length picked per column) vs a per-column compress loop
    torch.cuda.synchronize(dev)
    e0.record(stream)
    batch = glc.Batch.compress(ctx, dtypes, [c.data_ptr() for c in cols], ns, fixed_len=0, stream=sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    batch_compress_ms = e0.elapsed_time(e1)
    e0.record(stream)
    singles = [glc.compress_device(ctx, d, c.data_ptr(), n, glc.FIXED, fixed_len=4096, stream=sh)
               for d, c, n in zip(dtypes, cols, ns)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    loop_compress_ms = e0.elapsed_time(e1)
    comp_bytes = batch.compressed_size
    # outputs: one buffer, 16-byte aligned slices
    offs, o = [], 0
    for c in cols:
        offs.append(o)
        o += (c.numel() * c.element_size() + 255) // 256 * 256
    out = torch.empty(o, dtype=torch.uint8, device=dev)
    ptrs = [out.data_ptr() + x for x in offs]

    def step():
        batch.decompress(ptrs, use_graph=True, stream=sh)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ok = all(torch.equal(out[x:x + c.numel() * c.element_size()], c.view(torch.uint8)) for x, c in zip(offs, cols))
    clocks = ClockSampler(dev)
    clocks.start()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    # the same decode as a per-column launch loop (same kernels, one launch chain per column)
    def loop():
        for col, p in zip(singles, ptrs):
            glc.decompress_into(ctx, col, p, glc.SRC_PACKED, stream=sh)
    loop()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    reps = max(1, min(args.steps, 5))
    for _ in range(reps):
        loop()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    loop_ms = e0.elapsed_time(e1) / reps
    # end to end: batched decode + one device-to-host copy of every column into pinned memory
    h_out = torch.empty(o, dtype=torch.uint8).pin_memory()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        step()
        h_out.copy_(out, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
    peak, peak_kind = measured_peak()
    achieved = (comp_bytes + raw_bytes) / (ms / 1e3) / 1e9
    line = {
        "metric": "batched decode GB/s", "value": round(raw_bytes / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "mixed int32/int64/uint64",
        "data": "synthetic",
        "config": {"workload": f"batch_{args.columns}_columns_mixed", "columns": args.columns,
                   "raw_bytes": raw_bytes, "compressed_bytes": comp_bytes,
                   "compression_ratio": round(raw_bytes / comp_bytes, 3),
                   "per_column_loop_ms": round(loop_ms, 3), "per_column_loop_gbs": round(raw_bytes / loop_ms / 1e6, 2),
                   "speedup_vs_per_column_loop": round(loop_ms / ms, 2),
                   "batch_compress_ms": round(batch_compress_ms, 2), "per_column_compress_loop_ms": round(loop_compress_ms, 2),
                   "partition_lengths": {str(L): sum(1 for c in batch.columns if c.info().fixed_partition_len == L)
                                         for L in (1024, 2048, 4096)},
                   "graph": "one persistent launch captured in a CUDA graph and replayed", "bit_exact": ok},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": None},
        "e2e": {"value": round(raw_bytes / (e2e_ms / 1e3) / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": raw_bytes},
        "gpu_launches": args.steps, "clocks": clk, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    for sgl in singles:
        sgl.free()
    batch.free()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="glc", choices=["glc", "reference"])
    ap.add_argument("--n", type=int, default=DEFAULT_N)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--columns", type=int, default=4096, help="c4 batch: number of columns")
    ap.add_argument("--workload", default="c2_decode", choices=["c2_decode", "c3_random_access", "c4_batch"],
                    help="c2_decode (headline): full decode of the 200M piecewise uint64 column; "
                         "c3_random_access: 100M lookups into a 64M int64 timestamp column")
    ap.add_argument("--mode", default="packed", choices=["packed", "preunpacked"], help="c3 residual source")
    ap.add_argument("--queries", type=int, default=100_000_000, help="c3 lookups per step")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "c3_random_access":
        return run_random_access(args)
    if args.workload == "c4_batch":
        return run_batch(args)

    import torch
    import torch.distributed as dist

    import glc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)  # every launch and both events on this stream
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = glc.Context(local)

    n = args.n
    values = make_values(n, rank)
    d_in = torch.from_numpy(values.view(np.int64)).to(dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    col = glc.compress_device(ctx, glc.U64, d_in.data_ptr(), n, glc.VARIABLE, stream=sh)
    torch.cuda.synchronize(dev)
    compress_s = time.perf_counter() - t0
    info = col.info()
    del d_in
    out = torch.empty(n, dtype=torch.int64, device=dev)

    def step():
        glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED, stream=sh)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ok = bool(np.array_equal(out.cpu().numpy().view(np.uint64), values))

    clocks = ClockSampler(dev)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    t_max = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_max = float(t_max.item())
    ms_per_step = ms_max / args.steps
    decoded_bytes = n * 8
    value = decoded_bytes * world / (ms_per_step / 1e3) / 1e9

    # roofline of the decode kernel (one launch per step)
    algo_bytes = info.compressed_size_bytes + decoded_bytes
    achieved = algo_bytes / (ms / args.steps / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    tpv = profiled_traffic_per_value()

    # end to end through the C ABI with host buffers: host blob -> device -> decode -> host
    blob = glc.serialize_host(ctx, col)
    h_blob = torch.from_numpy(np.frombuffer(blob, np.uint8).copy()).pin_memory()
    h_out = torch.empty(n, dtype=torch.int64).pin_memory()
    lib = ctx.lib
    import ctypes

    def e2e_step():
        h = ctypes.c_void_p()
        ctx.check(lib.glc_deserialize(ctx.handle, glc.U64, ctypes.c_void_p(h_blob.data_ptr()), len(blob), glc.HOST_IN,
                                      0, 0, ctypes.byref(h), ctypes.c_void_p(sh)))
        c2 = glc.Column(ctx, h)
        glc.decompress_into(ctx, c2, h_out.data_ptr(), glc.SRC_PACKED, stream=sh, host_out=True)
        c2.free()

    e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = torch.tensor([e0.elapsed_time(e1) / args.e2e_steps], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_ok = bool(np.array_equal(h_out.numpy().view(np.uint64), values))
    e2e_value = decoded_bytes * world / (float(e2e_ms.item()) / 1e3) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = 1
            cpu = cpu_baseline_decode(values, lambda s: glc.serialize_host(
                ctx, glc.compress_device(ctx, glc.U64, s.ctypes.data, len(s), glc.VARIABLE, host=True)), threads)
        except Exception as ex:  # reported, never fatal
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "values": n, "partitions": info.num_partitions,
                       "bits_per_value": round(info.total_bits / n, 3),
                       "compressed_bytes": info.compressed_size_bytes,
                       "compression_ratio": round(decoded_bytes / info.compressed_size_bytes, 3),
                       "l2": "inputs and output larger than L2 (no flush)", "parallelism": f"replicas{world}",
                       "compress_s": round(compress_s, 3), "bit_exact": ok and e2e_ok},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "traffic": (round(tpv * n) if tpv else None),
                         "algorithmic_bytes": algo_bytes},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": len(blob),
                    "d2h_bytes_per_step": decoded_bytes},
            "gpu_launches": args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    col.free()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
