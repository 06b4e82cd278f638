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
buffers: every step decodes the host (pinned) blob into pinned host memory with
glc_decode_blob_to_host, which checks the blob, uploads its bitstream, decodes and downloads the
values in chunks overlapped on three streams.  ``roofline`` = algorithmic bytes (compressed bytes read + decoded bytes written)
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
TRAFFIC_JSON = os.path.join(ROOT, "profiles", "decode_piecewise_u64_200M.traffic.json")
# launch shapes measured once per device by glc_autotune (built files, not committed)
TUNE_CACHE = os.path.join(ROOT, "g-leco_b200", "_build", "tune_cache.txt")


def tuned_context(glc, device: int):
    """A context whose launch shapes come from the autotuner (measured on first use, ~1 s)."""
    ctx = glc.Context(device)
    os.makedirs(os.path.dirname(TUNE_CACHE), exist_ok=True)
    glc.autotune(ctx, TUNE_CACHE)
    return ctx


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(n: int):
    """DRAM bytes (read + write) of one decode launch over n values, from the ncu capture that the
    profiling step writes as JSON beside its summary (one launch of the full-size workload),
    scaled by the values decoded; None when there is no capture."""
    try:
        with open(TRAFFIC_JSON) as f:
            t = json.load(f)
        return round((t["dram_bytes_read"] + t["dram_bytes_write"]) * n / t["values"])
    except (OSError, KeyError, ValueError):
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
    print(time.monotonic_ns(), pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), int(get(h)), flush=True)
    time.sleep(0.0002)
"""


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of the benchmarked GPU, sampled through NVML
    about every 0.3 ms by a separate process (reads only; no GPU setting is changed).  begin() and
    end() mark the timed region on the host's monotonic clock (both sides synchronised with the
    device); the summary keeps the samples inside it, or the nearest one on each side when the
    region is shorter than the sampling interval."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device):
        self.dev = torch_device
        self.proc = None
        self.t_begin = self.t_end = None

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
        self.max_line = self.proc.stdout.readline()
        self.first_line = self.proc.stdout.readline()  # sampling runs before the timed region starts

    def begin(self):
        self.t_begin = time.monotonic_ns()

    def end(self):
        self.t_end = time.monotonic_ns()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": "sampler not started"}
        if self.t_end is not None:
            time.sleep(0.002)  # a sample after the region
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = []
        for ln in [self.first_line] + out.splitlines():
            parts = ln.split()
            if len(parts) == 3:
                rows.append((int(parts[0]), float(parts[1]), int(parts[2])))
        picked = rows
        if self.t_begin is not None and self.t_end is not None and rows:
            inside = [r for r in rows if self.t_begin <= r[0] <= self.t_end]
            if inside:
                picked = inside
            else:  # the region is shorter than the interval: the nearest sample on each side
                before = [r for r in rows if r[0] < self.t_begin][-1:]
                after = [r for r in rows if r[0] > self.t_end][:1]
                picked = before + after
        reasons = set()
        for _, _, bits in picked:
            for bit, name in self.REASONS.items():
                if bits & bit:
                    reasons.add(name)
        try:
            smax = float(self.max_line.split()[1])
        except Exception:
            smax = None
        inside_n = sum(1 for r in rows if self.t_begin is not None and self.t_end is not None
                       and self.t_begin <= r[0] <= self.t_end)
        return {"sm_mhz": float(np.median([r[1] for r in picked])) if picked else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(picked), "samples_in_region": inside_n,
                "source": "NVML every ~0.3 ms (separate process)"}


def make_values(n: int, rank: int) -> np.ndarray:
    from glc import workloads as W
    return W.piecewise_linear(n, seed=42 + rank)


REF_CACHE = os.path.join(ROOT, "g-leco_b200", "_build", "reference_arm")


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline_decode(blob: bytes, values: np.ndarray, threads: int, passes: int = 3):
    """The reference's host decoder (directRandomAccessCPU, compiled from the reference's sources)
    over EVERY position of ``blob`` on ``threads`` host threads; returns a cpu_baseline dict.
    Without the compiled reference, the oracle's decode (one thread) stands in ("port")."""
    import oracle
    n = len(values)
    if oracle.ref_available():
        with tempfile.TemporaryDirectory() as td:
            bp, vp, mp = (os.path.join(td, f) for f in ("blob.bin", "values.bin", "mism.bin"))
            with open(bp, "wb") as f:
                f.write(blob)
            values.tofile(vp)
            secs, mism = oracle.ref_hostdecode_all(bp, vp, "u64", threads, passes, mp)
            where = np.fromfile(mp, np.int64).astype(np.int32)
        col = oracle.deserialize(blob, "u64")
        # every value the reference's host decoder gets wrong is one where its prediction without
        # fma rounds differently from the format's fma prediction (the oracle restates both)
        explained = bool(np.all(oracle.decode_variant(col, where, oracle.PRED_HOST)
                                != oracle.decode_variant(col, where, oracle.PRED_CONTRACT)))
        best = min(secs)
        kind, how = "reference", "directRandomAccessCPU (the reference's host decoder, compiled from its sources)"
    else:
        col = oracle.deserialize(blob, "u64")
        t0 = time.perf_counter()
        out = oracle.decode_full(col)
        best = time.perf_counter() - t0
        mism, explained, threads, passes = int(np.count_nonzero(out != values)), True, 1, 1
        kind, how = "port", "the oracle's decode (the reference harness is not built)"
    return {"value": round(n * 8 / best / 1e9, 4), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"full decode of all {n:,} values of the workload's blob by {how} on {threads} host "
                      f"thread(s), best of {passes} passes ({best:.3f} s); values differing from the input: "
                      f"{mism}, all at positions where that decoder's prediction without fma rounds "
                      f"differently: {explained}"}


def reference_blob(n: int, seed: int):
    """The workload column compressed by the reference's own stock compress with its CPU
    partitioner (use_variable_partitioning = true, api/G-LeCo.cuh:349-614) and serialize (:826),
    run from the compiled reference on this host's GPU; cached under _build/.  Returns
    (values, blob path, values path, reported compressed size, how)."""
    import oracle
    os.makedirs(REF_CACHE, exist_ok=True)
    stem = os.path.join(REF_CACHE, f"piecewise_u64_{n}_seed{seed}")
    meta_p, vp, bp = stem + ".json", stem + ".values.bin", stem + ".blob"
    values = make_values(n, seed - 42)
    if os.path.exists(meta_p) and os.path.exists(bp) and os.path.exists(vp):
        with open(meta_p) as f:
            meta = json.load(f)
        return values, bp, vp, meta["size"], meta["how"]
    values.tofile(vp)
    t0 = time.perf_counter()
    try:
        size = oracle.ref_compress_blob(vp, "u64", "var", stem)
        how = (f"the reference's own compress (CPU partitioner) + serialize, "
               f"{time.perf_counter() - t0:.1f} s")
    except Exception as ex:  # no GPU or no harness: the oracle's restatement of the same path
        s, e = oracle.ref_partition_cpu(values)
        col = oracle.compress(values, starts=s, ends=e)
        with open(bp, "wb") as f:
            f.write(oracle.serialize(col))
        size = col.reported_size()
        how = f"the oracle's restatement of the reference's CPU partitioner and fit ({str(ex)[:80]})"
    with open(meta_p, "w") as f:
        json.dump({"size": size, "how": how}, f)
    return values, bp, vp, size, how


def run_reference_arm(args):
    """The reference's own CPU path on this host: its host decoder directRandomAccessCPU
    (api/G-LeCo.cuh:1337-1672), the only decoder it runs on host cores, over every position of
    the same 200M-value column, on all host threads; one step = one pass over the column."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    n = args.n
    threads = host_threads()
    values, bp, vp, ref_size, how = reference_blob(n, 42)
    if oracle.ref_available():
        secs, mism = oracle.ref_hostdecode_all(bp, vp, "u64", threads, args.warmup + args.steps)
        kind = "reference"
    else:  # the oracle port, one thread
        with open(bp, "rb") as f:
            col = oracle.deserialize(f.read(), "u64")
        secs = []
        for _ in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            out = oracle.decode_full(col)
            secs.append(time.perf_counter() - t0)
        mism, threads, kind = int(np.count_nonzero(out != values)), 1, "port"
    timed = secs[args.warmup:]
    step_s = float(np.mean(timed))
    val = n * 8 / step_s / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_s * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "values": n, "ref_compressed_bytes": ref_size, "blob": how,
                       "l2": "host decode; column larger than the host caches"},
            "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"every step decodes all {n:,} values (directRandomAccessCPU over every "
                                       f"position, {threads} host threads, wall clock per pass); values "
                                       f"differing from the input: {mism}"},
            "e2e": {"value": round(val, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    ctx = tuned_context(glc, local)
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
    # the ceiling of this access pattern: a plain 8-byte gather (torch.index_select) of the same
    # positions from the raw values, an array as large as the pre-unpacked residuals (512 MB)
    d_pos64 = d_pos.long()
    gout = torch.empty(q, dtype=torch.int64, device=dev)
    for _ in range(3):
        torch.index_select(d_vals, 0, d_pos64, out=gout)
    e0.record(stream)
    for _ in range(args.steps):
        torch.index_select(d_vals, 0, d_pos64, out=gout)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    gather_s = q / (e0.elapsed_time(e1) / args.steps / 1e3)
    del d_pos64, gout
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
                   "gather_ceiling": {"value": round(gather_s, 1), "unit": "lookups/s",
                                      "what": "torch.index_select of the same positions from the raw 512 MB int64 "
                                              "values (8 B random gather, no decoding)",
                                      "frac": round(lookups_s / gather_s, 4)},
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


def run_decode_i32(args):
    """Full decode of an int32 column: n values 1000 + 3 i + U[0, 2^w) (w = --noise-bits), fixed
    partitions of 4096, generated and compressed on the device.  One step = one full decode;
    value = decoded GB/s.  Roofline bytes: compressed bytes read + 4 B per value written."""
    import torch

    import glc

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = tuned_context(glc, local)
    n = args.n if args.n != DEFAULT_N else 100_000_000
    w = args.noise_bits
    i = torch.arange(n, device=dev, dtype=torch.int64)
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    v = (1000 + 3 * i + torch.randint(0, 1 << w, (n,), device=dev, generator=g)).to(torch.int32)
    del i
    col = glc.compress_device(ctx, glc.I32, v.data_ptr(), n, glc.FIXED, fixed_len=4096, stream=sh)
    info = col.info()
    out = torch.empty_like(v)

    def step():
        glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED, stream=sh)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    ok = bool(torch.equal(out, v))
    clocks = ClockSampler(dev)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    peak, peak_kind = measured_peak()
    algo = info.compressed_size_bytes + 4 * n
    line = {
        "metric": "decoded GB/s", "value": round(4 * n / (ms / 1e3) / 1e9, 2), "unit": "GB/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"linear_i32_{n // 1_000_000}M_noise{w}_fixed4096", "values": n,
                   "bits_per_value": round(info.total_bits / n, 3), "values_per_s": round(n / (ms / 1e3), 1),
                   "bit_exact": ok, "l2": "output larger than L2 (no flush)"},
        "roofline": {"bound": "hbm", "achieved": round(algo / (ms / 1e3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(algo / (ms / 1e3) / 1e9 / peak, 4), "peak_kind": peak_kind, "traffic": None},
        "e2e": None, "gpu_launches": args.steps, "clocks": clk, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    col.free()
    ctx.close()
    return 0


def run_c1(args):
    """The plain small workload: 1,048,576 int32 v[i] = 1000 i + U{0..255} (seed 42), fixed
    partitions of 1024.  One step = compress from device memory + full decode + 10,000 uniform
    lookups, each step's column freed outside the timed region; value = raw input GB/s of the step
    (4 MiB / step time).  Roofline bytes: input read + compressed written (compress), compressed read +
    4 B per value written (decode), 4 + 4 + 32 B per lookup.  cpu_baseline: the reference's host code
    for the same step -- its CPU partitioner (one thread, as the reference runs it), then
    directRandomAccessCPU over all values and over the 10,000 positions (the reference has no host
    fit or pack)."""
    import torch

    import glc
    from glc import workloads as W

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = tuned_context(glc, local)
    n, L, q = 1 << 20, 1024, 10_000
    values = W.plain_small(n, seed=42)
    pos = np.random.default_rng(42).integers(0, n, q).astype(np.int32)
    d_in = torch.from_numpy(values).to(dev)
    d_pos = torch.from_numpy(pos).to(dev)
    out = torch.empty(n, dtype=torch.int32, device=dev)
    look = torch.empty(q, dtype=torch.int32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def step():
        ev[0].record(stream)
        col = glc.compress_device(ctx, glc.I32, d_in.data_ptr(), n, glc.FIXED, fixed_len=L, stream=sh)
        ev[1].record(stream)
        glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED, stream=sh)
        ev[2].record(stream)
        glc.random_access_into(ctx, col, d_pos.data_ptr(), q, look.data_ptr(), source=glc.SRC_PACKED, fixed_len=L,
                               stream=sh)
        ev[3].record(stream)
        torch.cuda.synchronize(dev)
        t = [ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3])]
        return col, t

    for _ in range(args.warmup):
        step()[0].free()
    ok = bool(torch.equal(out, d_in)) and bool(torch.equal(look, d_in[d_pos.long()]))
    clocks = ClockSampler(dev)
    clocks.start()
    parts = []
    for _ in range(args.steps):
        col, t = step()
        parts.append(t)
        info = col.info()
        col.free()
    clk = clocks.stop()
    parts = np.array(parts)
    ms = float(parts.sum(axis=1).mean())
    comp = info.compressed_size_bytes
    algo = (4 * n + comp) + (comp + 4 * n) + 40 * q
    peak, peak_kind = measured_peak()
    # end to end through the reference-facing API: host values in, host values out
    codec = glc.LeCoGPU(np.int32, device=local)
    e2e = []
    for k in range(args.e2e_steps + 1):
        t0 = time.perf_counter()
        c, _ = codec.compress(values, False, fixed_partition_size=L)
        full = codec.decompressFullFile(c)
        got = codec.randomAccessFixed(c, pos, L)
        e2e.append(time.perf_counter() - t0)
        c.free()
    e2e_ok = bool(np.array_equal(full, values)) and bool(np.array_equal(got, values[pos]))
    e2e_s = float(np.mean(e2e[1:]))
    cpu = None
    if not args.no_cpu_baseline:
        import oracle
        try:
            with tempfile.TemporaryDirectory() as td:
                t0 = time.perf_counter()
                oracle.ref_partition(values, td)
                part_s = time.perf_counter() - t0
                blob = glc.serialize_host(ctx, glc.compress_device(ctx, glc.I32, values.ctypes.data, n, glc.FIXED,
                                                                   fixed_len=L, host=True))
                _, full_s = oracle.ref_hostdecode(blob, "i32", np.arange(n, dtype=np.int32), td, repeat=3)
                _, ra_s = oracle.ref_hostdecode(blob, "i32", pos, td, repeat=3)
            tot = part_s + full_s + ra_s
            cpu = {"value": round(4 * n / tot / 1e9, 4), "unit": "GB/s", "cores": 1, "kind": "reference",
                   "sample": f"the whole step on the reference's host code, one thread: CPU partitioner "
                             f"{part_s * 1e3:.1f} ms (process run), directRandomAccessCPU over all values "
                             f"{full_s * 1e3:.1f} ms and over the 10,000 positions {ra_s * 1e3:.2f} ms; the "
                             f"reference has no host fit or pack"}
        except Exception as ex:
            cpu = {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}
    line = {
        "metric": "C1 round trip GB/s (input)", "value": round(4 * n / (ms / 1e3) / 1e9, 3), "unit": "GB/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "plain_i32_1M_fixed1024_compress_decode_10k_lookups", "values": n, "lookups": q,
                   "partitions": info.num_partitions, "compressed_bytes": comp,
                   "compress_ms": round(float(parts[:, 0].mean()), 4), "decode_ms": round(float(parts[:, 1].mean()), 4),
                   "lookups_ms": round(float(parts[:, 2].mean()), 4), "bit_exact": ok and e2e_ok,
                   "l2": "4 MiB column: L2-resident; the step is launch-latency bound"},
        "roofline": {"bound": "hbm", "achieved": round(algo / (ms / 1e3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(algo / (ms / 1e3) / 1e9 / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes": algo},
        "e2e": {"value": round(4 * n / e2e_s / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": 4 * n + 4 * q,
                "d2h_bytes_per_step": 4 * n + 4 * q + 8},
        "gpu_launches": (COMPRESS_LAUNCHES["fixed"] + 2) * args.steps, "clocks": clk, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


COMPRESS_LAUNCHES = {"fixed": 5, "v6": 29}  # kernels launched by one compress call (fixed: compress, 3 scan, place)


def run_compress(args):
    """Compress: the 200M piecewise uint64 column of the decode workload, from device memory, with
    fixed partitions of 4096 (--partitioning fixed), the reference's GPU partitioner (v6) or the
    split/merge partitioner (variable).  One step = one glc_compress call (partition, fit, offsets,
    pack) timed alone with CUDA events; the column is freed between steps outside the timed region.
    value = input GB/s.  Roofline bytes: the input read once + the compressed bytes written."""
    import torch

    import glc

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = tuned_context(glc, local)
    n = args.n
    values = make_values(n, 0)
    d_in = torch.from_numpy(values.view(np.int64)).to(dev)
    mode = {"fixed": glc.FIXED, "v6": glc.VARIABLE_V6, "variable": glc.VARIABLE}[args.partitioning]

    def step():
        return glc.compress_device(ctx, glc.U64, d_in.data_ptr(), n, mode, fixed_len=4096, stream=sh)

    for _ in range(args.warmup):
        step().free()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dev)
    clocks.start()
    times = []
    col = None
    for _ in range(args.steps):
        if col is not None:
            col.free()
        e0.record(stream)
        col = step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        times.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    ms = sum(times) / len(times)
    info = col.info()
    comp = info.compressed_size_bytes
    out = torch.empty(n, dtype=torch.int64, device=dev)
    glc.decompress_into(ctx, col, out.data_ptr(), glc.SRC_PACKED, stream=sh)
    torch.cuda.synchronize(dev)
    ok = bool(torch.equal(out, d_in))
    del out
    col.free()
    in_bytes = 8 * n
    peak, peak_kind = measured_peak()
    achieved = (in_bytes + comp) / (ms / 1e3) / 1e9
    # end to end: pinned host values in (uploaded inside the call), the compressed size read back
    h_in = torch.from_numpy(values.view(np.int64)).pin_memory()
    e2e = []
    for k in range(args.e2e_steps + 1):
        e0.record(stream)
        c = glc.compress_device(ctx, glc.U64, h_in.data_ptr(), n, mode, fixed_len=4096, stream=sh, host=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if k:
            e2e.append(e0.elapsed_time(e1))
        c.free()
    e2e_ms = sum(e2e) / len(e2e)
    cpu = None
    if not args.no_cpu_baseline and args.partitioning == "fixed":
        import oracle
        sample = np.ascontiguousarray(values[:4_000_000])
        t0 = time.perf_counter()
        oc = oracle.compress(sample, "fixed", 4096)
        secs = time.perf_counter() - t0
        cpu = {"value": round(8 * len(sample) / secs / 1e9, 3), "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": f"{len(sample):,} values through the oracle's compress (fixed 4096); "
                         f"size {oc.reported_size()} B"}
    line = {
        "metric": "compress GB/s (input)", "value": round(in_bytes / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint64", "data": "synthetic",
        "config": {"workload": f"piecewise_u64_{n // 1_000_000}M_compress_{args.partitioning}", "values": n,
                   "partitions": info.num_partitions, "compressed_bytes": comp,
                   "compression_ratio": round(in_bytes / comp, 3), "best_ms": round(min(times), 4),
                   "round_trip_exact": ok, "l2": "input larger than L2 (no flush)"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes": in_bytes + comp},
        "e2e": {"value": round(in_bytes / (e2e_ms / 1e3) / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": 8},
        "gpu_launches": COMPRESS_LAUNCHES[args.partitioning] * args.steps if args.partitioning in COMPRESS_LAUNCHES else None,
        "clocks": clk, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
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
    ctx = tuned_context(glc, local)
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
    # batched compress (partition length picked per column) vs a per-column compress loop; best of
    # 3 calls each (the first call also grows the context's memory pool)
    batch_compress_ms, loop_compress_ms, batch, singles = 1e30, 1e30, None, None
    col_ptrs = np.array([c.data_ptr() for c in cols], dtype=np.uint64)
    for rep in range(3):
        if batch is not None:
            batch.free()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        batch = glc.Batch.compress(ctx, dtypes, col_ptrs, ns, fixed_len=0, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        batch_compress_ms = min(batch_compress_ms, e0.elapsed_time(e1))
    for rep in range(0 if args.no_loops else 3):
        if singles is not None:
            for sgl in singles:
                sgl.free()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        singles = [glc.compress_device(ctx, d, c.data_ptr(), n, glc.FIXED, fixed_len=4096, stream=sh)
                   for d, c, n in zip(dtypes, cols, ns)]
        e1.record(stream)
        torch.cuda.synchronize(dev)
        loop_compress_ms = min(loop_compress_ms, e0.elapsed_time(e1))
    comp_bytes = batch.compressed_size
    # the same columns recompressed in place (lengths kept, nothing read back), replayed from a CUDA
    # graph: the repeated-call form of the batched compress
    batch.recompress([c.data_ptr() for c in cols], use_graph=True, stream=sh)
    batch.sync(stream=sh)
    recompress_ms = 1e30
    for rep in range(5):
        torch.cuda.synchronize(dev)
        e0.record(stream)
        batch.recompress(col_ptrs, use_graph=True, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        recompress_ms = min(recompress_ms, e0.elapsed_time(e1))
    assert batch.sync(stream=sh) == comp_bytes
    # outputs: one buffer, 16-byte aligned slices
    offs, o = [], 0
    for c in cols:
        offs.append(o)
        o += (c.numel() * c.element_size() + 255) // 256 * 256
    out = torch.empty(o, dtype=torch.uint8, device=dev)
    ptrs = np.array([out.data_ptr() + x for x in offs], dtype=np.uint64)

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
        for col, p in zip(singles, ptrs.tolist()):
            glc.decompress_into(ctx, col, p, glc.SRC_PACKED, stream=sh)
    loop_ms = float("nan")
    if not args.no_loops:
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
                   "per_column_loop_ms": None if args.no_loops else round(loop_ms, 3),
                   "per_column_loop_gbs": None if args.no_loops else round(raw_bytes / loop_ms / 1e6, 2),
                   "speedup_vs_per_column_loop": None if args.no_loops else round(loop_ms / ms, 2),
                   "batch_compress_ms": round(batch_compress_ms, 2),
                   "per_column_compress_loop_ms": None if args.no_loops else round(loop_compress_ms, 2),
                   "batch_recompress_graph_ms": round(recompress_ms, 3),
                   "batch_recompress_gbs": round((raw_bytes + comp_bytes) / recompress_ms / 1e6, 1),
                   "compress_timing": "best of 3 calls each (CUDA events on the calling stream)",
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
    for sgl in singles or []:
        sgl.free()
    batch.free()
    ctx.close()
    return 0


def device_piecewise_u64(n: int, seed: int, dev):
    """The piecewise-linear uint64 distribution of glc.workloads.piecewise_linear, generated on the
    device: segment lengths ~ Poisson(50,000), slope U{1..10^6}, intercept jump U{0..2^40}, noise
    U[0, 2^b) with b in {0,4,8,16,24}.  Values stay below 2^63 (returned as int64 bit patterns)."""
    import torch
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    S = n // 50_000 * 2 + 64
    lens = torch.poisson(torch.full((S,), 50_000.0, device=dev), generator=g).clamp_min(1).to(torch.int64)
    ends = torch.cumsum(lens, 0)
    S = int(torch.searchsorted(ends, torch.tensor([n], device=dev)).item()) + 1
    lens = lens[:S].clone()
    lens[-1] -= int(ends[S - 1].item()) - n
    starts = torch.cumsum(lens, 0) - lens
    slope = torch.randint(1, 1_000_001, (S,), device=dev, generator=g, dtype=torch.int64)
    jump = torch.randint(0, (1 << 40) + 1, (S,), device=dev, generator=g, dtype=torch.int64)
    bsel = torch.tensor([0, 4, 8, 16, 24], device=dev)[torch.randint(0, 5, (S,), device=dev, generator=g)]
    span = slope * (lens - 1)
    base = torch.cumsum(jump, 0) + torch.cumsum(span, 0) - span
    seg = torch.repeat_interleave(torch.arange(S, device=dev), lens)
    j = torch.arange(n, device=dev, dtype=torch.int64) - starts[seg]
    v = base[seg] + slope[seg] * j
    del j
    noise = torch.randint(0, 1 << 24, (n,), device=dev, generator=g, dtype=torch.int64)
    v += noise & ((torch.ones_like(noise) << bsel[seg]) - 1)
    return v


def device_timestamps_i64(n: int, seed: int, dev):
    """Cumulative sums of exponential gaps (mean 1000) rounded to integers, starting at 0."""
    import torch
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    gaps = torch.empty(n, device=dev, dtype=torch.float64).exponential_(1.0 / 1000.0, generator=g)
    gaps = torch.round(gaps).to(torch.int64)
    gaps[0] = 0
    return torch.cumsum(gaps, 0)


def device_linear_i32(n: int, seed: int, dev):
    """intercept + slope * i + noise with slope U[0, 10^4] capped to stay inside int32, noise
    U[0, 2^w) with w U{0..20} (one column of the batched workload's distribution)."""
    import torch
    rng = np.random.default_rng(seed)
    slope = min(int(rng.integers(0, 10_001)), (2 ** 30) // n)
    w = int(rng.integers(0, 21))
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    v = int(rng.integers(0, 1 << 20)) + slope * torch.arange(n, device=dev, dtype=torch.int64)
    if w:
        v += torch.randint(0, 1 << w, (n,), device=dev, generator=g, dtype=torch.int64)
    return v.to(torch.int32)


# Serving column sources: (name, dtype code, values, partitioning, fixed length, columns admitted)
SERVE_SOURCES = [("piecewise_u64_600M_variable", "U64", 600_000_000, "VARIABLE", 0, 32),
                 ("timestamps_i64_256M_fixed4096", "I64", 256_000_000, "FIXED", 4096, 16),
                 ("linear_i32_16M_fixed2048", "I32", 16_000_000, "FIXED", 2048, 16)]


def _pct(a, q):
    return float(np.percentile(a, q)) if len(a) else None


def run_serving(args):
    """Serving: 64 resident compressed columns (32 piecewise uint64 of 600M values, 16 int64
    timestamp columns of 256M, 16 int32 linear+noise columns of 16M; about 40 GB resident under a
    60 GB admission budget), driven by open-loop Poisson request streams at swept rates.  A request
    is a lookup of floor(exp(U[0, ln 65,536])) positions (uniform over the column) or a range
    decode of floor(exp(U[ln 1,024, ln 16M])) values, 50/50; during every rate point new columns
    are admitted and the least recently used idle ones evicted.  Latency = completion seen by the
    server minus the request's scheduled arrival.  The comparison is the plain per-call form:
    one glc_random_access call per lookup request on one stream, back to back."""
    import ctypes

    import torch

    import glc

    from glc.sharding import gather_objects, merge_serving_points

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:  # whole columns per GPU: every rank serves its own columns; no data-path collective
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    ctx = tuned_context(glc, local)
    scale = args.serve_scale
    gens = {"U64": device_piecewise_u64, "I64": device_timestamps_i64, "I32": device_linear_i32}
    sources = []
    t_build = time.perf_counter()
    for k, (name, dt, n, mode, L, copies) in enumerate(SERVE_SOURCES):
        n = max(8192, int(n * scale))
        v = gens[dt](n, 42 + k + 1000 * rank, dev)
        code = getattr(glc, dt)
        col = glc.compress_device(ctx, code, v.data_ptr(), n, getattr(glc, mode), fixed_len=L or 4096, stream=sh)
        size = ctypes.c_uint64()
        ctx.check(ctx.lib.glc_blob_size(col.handle, ctypes.byref(size)))
        blob = torch.empty(int(size.value), dtype=torch.uint8, device=dev)
        wrote = ctypes.c_uint64()
        ctx.check(ctx.lib.glc_serialize(ctx.handle, col.handle, ctypes.c_void_p(blob.data_ptr()), size.value, 0, 0,
                                        ctypes.byref(wrote), ctypes.c_void_p(sh)))
        pool = torch.randint(0, n, (1 << 24,), device=dev, dtype=torch.int32)
        # a few known values to check the served results against
        sources.append(dict(name=name, code=code, n=n, col=col, blob=blob, pool=pool, copies=copies,
                            esize=4 if dt == "I32" else 8, check=v[:1 << 20].clone(),
                            bits=col.info().total_bits / n))
        del v
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    budget = int(60e9 * scale) if scale < 1 else int(60e9)
    server = glc.Server(ctx, budget_bytes=budget, slots=args.slots, max_range_values=args.max_range_values,
                        reserve=True)
    ids, src_of = [], {}
    t0 = time.perf_counter()
    for si, s in enumerate(sources):
        for _ in range(s["copies"]):
            cid = server.admit_blob(s["code"], s["blob"].data_ptr(), s["blob"].numel(), stream=sh)
            ids.append(cid)
            src_of[cid] = si
    admit_s = time.perf_counter() - t0
    st = server.stats()
    resident_gb = st.resident_bytes / 1e9
    build_s = time.perf_counter() - t_build
    lk_arena = torch.empty(1 << 28, dtype=torch.uint8, device=dev)
    rg_arena = torch.empty(4 << 30, dtype=torch.uint8, device=dev)

    def make_stream(rate, lookup_frac, nreq, seed, resident):
        rng = np.random.default_rng(seed)
        req = glc.requests(nreq)
        hot = rng.choice(np.array(resident), min(48, len(resident)), replace=False)
        col = hot[rng.integers(0, len(hot), nreq)]
        is_lk = rng.random(nreq) < lookup_frac
        si = np.array([src_of[int(c)] for c in col])
        n_of = np.array([s["n"] for s in sources])[si]
        es = np.array([s["esize"] for s in sources])[si]
        cnt_l = np.clip(np.floor(np.exp(rng.uniform(0, np.log(65536), nreq))), 1, 65536).astype(np.int64)
        cnt_r = np.floor(np.exp(rng.uniform(np.log(1024), np.log(16 << 20), nreq))).astype(np.int64)
        cnt_r = np.minimum(cnt_r, n_of)
        cnt = np.where(is_lk, cnt_l, cnt_r)
        first = np.where(is_lk, 0, (rng.random(nreq) * (n_of - cnt + 1)).astype(np.int64))
        pool_base = np.array([s["pool"].data_ptr() for s in sources], np.uint64)[si]
        pool_off = (rng.random(nreq) * ((1 << 24) - cnt_l)).astype(np.uint64) * np.uint64(4)
        # outputs: consecutive slices of two arenas (wrapping); ranges placed so that
        # out - first * esize is 16-byte aligned (decoded in place)
        nbytes = cnt * es
        lk_off = np.cumsum(np.where(is_lk, (nbytes + 15) // 16 * 16, 0)) % ((1 << 28) - (1 << 20))
        rg_need = np.where(is_lk, 0, (nbytes + 31) // 16 * 16)
        rg_off = (np.cumsum(rg_need) % ((4 << 30) - (256 << 20))) // 16 * 16 + ((first * es) % 16)
        out = np.where(is_lk, np.uint64(lk_arena.data_ptr()) + lk_off.astype(np.uint64),
                       np.uint64(rg_arena.data_ptr()) + rg_off.astype(np.uint64))
        req["kind"] = np.where(is_lk, glc.REQ_LOOKUP, glc.REQ_RANGE)
        req["column"] = col
        req["first"] = first
        req["count"] = cnt
        req["positions"] = np.where(is_lk, pool_base + pool_off, 0)
        req["out"] = out
        req["tag"] = np.arange(nreq)
        gaps = rng.exponential(1e9 / rate, nreq)
        start = server.now_ns() + 50_000_000 + nreq * 300
        req["not_before_ns"] = start + np.cumsum(gaps).astype(np.int64)
        return req, si, es

    def run_point(rate, lookup_frac, seed, admit_during):
        nonlocal ids
        nreq = int(np.clip(rate * args.serve_seconds, 4000, 500_000))
        req, si, es = make_stream(rate, lookup_frac, nreq, seed + 7919 * rank, ids)
        if world > 1:
            torch.distributed.barrier()  # all ranks serve the rate point at the same time
        before = server.stats()
        server.submit(req)
        admitted, refused, adm_t = 0, 0, 0.0
        if admit_during:  # new columns arrive while the stream runs; LRU idle columns make room
            time.sleep(max(0.0, (int(req["not_before_ns"][0]) - server.now_ns()) / 1e9))
            for k in range(admit_during):
                s = sources[0]  # the largest columns
                ta = time.perf_counter()
                try:
                    cid = server.admit_blob(s["code"], s["blob"].data_ptr(), s["blob"].numel(), stream=sh)
                    src_of[cid] = 0
                    admitted += 1
                except glc.GlcError as ex:
                    if ex.status != glc.ERR_BUDGET:
                        raise
                    refused += 1
                adm_t += time.perf_counter() - ta
        server.drain(600_000)
        after = server.stats()
        ids = server.columns()
        recs = []
        while True:
            r = server.poll()
            if len(r) == 0:
                break
            recs.append(r)
        recs = np.concatenate(recs)
        assert len(recs) == nreq and np.all(recs["status"] == glc.OK), "served request failed"
        order = np.argsort(recs["tag"])
        recs = recs[order]
        lat_us = (recs["done_ns"] - recs["arrival_ns"]) / 1e3
        is_lk = req["kind"] == glc.REQ_LOOKUP
        span_s = (recs["done_ns"].max() - recs["arrival_ns"].min()) / 1e9
        lookups = int(req["count"][is_lk].sum())
        rvals = req["count"][~is_lk]
        rbytes = float((rvals * es[~is_lk]).sum())
        return {"rate_req_s": rate, "requests": nreq, "lookup_share": lookup_frac,
                "lookup_p50_us": round(_pct(lat_us[is_lk], 50), 1) if is_lk.any() else None,
                "lookup_p99_us": round(_pct(lat_us[is_lk], 99), 1) if is_lk.any() else None,
                "range_p50_us": round(_pct(lat_us[~is_lk], 50), 1) if (~is_lk).any() else None,
                "range_p99_us": round(_pct(lat_us[~is_lk], 99), 1) if (~is_lk).any() else None,
                "lookups_per_s": round(lookups / span_s, 1), "range_gb_s": round(rbytes / span_s / 1e9, 2),
                "launches": after.launches - before.launches,
                "requests_per_launch": round(nreq / max(1, after.launches - before.launches), 2),
                "span_s": round(span_s, 4), "admitted_during": admitted, "refused_during": refused,
                "admit_s": round(adm_t, 3), "evictions": after.evictions - before.evictions}

    # bit-exactness of served results: one lookup and one range request per source, checked
    chk_ok = True
    for si, s in enumerate(sources):
        cid = [c for c in ids if src_of[c] == si][0]
        pos = torch.randint(0, s["check"].numel(), (4096,), device=dev, dtype=torch.int32)
        lo = torch.zeros(4096, dtype=s["check"].dtype, device=dev)
        ro = torch.zeros(s["check"].numel(), dtype=s["check"].dtype, device=dev)
        r = glc.requests(2)
        r[0] = (glc.REQ_LOOKUP, cid, 0, 4096, pos.data_ptr(), lo.data_ptr(), 0, 0)
        r[1] = (glc.REQ_RANGE, cid, 0, s["check"].numel(), 0, ro.data_ptr(), 1, 0)
        server.submit(r)
        server.drain(60_000)
        server.poll()
        torch.cuda.synchronize(dev)
        chk_ok &= bool(torch.equal(lo, s["check"][pos.long()])) and bool(torch.equal(ro, s["check"]))

    rates = [float(x) for x in args.rates.split(",")]
    ra_rates = [float(x) for x in args.ra_rates.split(",")] if args.ra_rates else []
    clocks = ClockSampler(dev)
    clocks.start()
    sweep = []
    for k, rate in enumerate(rates):
        sweep.append(run_point(rate, 0.5, 100 + k, admit_during=args.admit_during))
    ra_sweep = []
    for k, rate in enumerate(ra_rates):
        ra_sweep.append(run_point(rate, 1.0, 200 + k, admit_during=0))
    clk = clocks.stop()

    # the plain per-call form: the same kind of stream, one libglc call per request from a C++ loop
    pc_lib = ctypes.CDLL(os.path.join(ROOT, "g-leco_b200", "_build", "libglc_percall.so"))
    src_handles = (ctypes.c_void_p * len(sources))(*[s["col"].handle.value for s in sources])
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def per_call(lookup_frac, nreq, seed):
        req, si, es = make_stream(1e6, lookup_frac, nreq, seed, ids)
        arrs = [np.ascontiguousarray(req["kind"]), si.astype(np.int32), np.ascontiguousarray(req["first"]),
                np.ascontiguousarray(req["count"]), np.ascontiguousarray(req["positions"]),
                np.ascontiguousarray(req["out"])]

        def go(k):
            rc = pc_lib.percall_run(ctx.handle, src_handles, ctypes.c_int32(k),
                                    *[ctypes.c_void_p(a.ctypes.data) for a in arrs], ctypes.c_void_p(sh))
            if rc != 0:
                raise RuntimeError(f"per-call loop failed with status {rc}")
        go(min(200, nreq))
        torch.cuda.synchronize(dev)
        e0.record(stream)
        go(nreq)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        secs = e0.elapsed_time(e1) / 1e3
        is_lk = req["kind"] == glc.REQ_LOOKUP
        return {"requests": nreq, "lookup_share": lookup_frac, "seconds": round(secs, 4),
                "requests_per_s": round(nreq / secs, 1),
                "lookups_per_s": round(float(req["count"][is_lk].sum()) / secs, 1),
                "range_gb_s": round(float((req["count"][~is_lk] * es[~is_lk]).sum()) / secs / 1e9, 2)}

    pc_lookups = per_call(1.0, 20_000, 7)
    pc_mix = per_call(0.5, 4_000, 8)
    # merge the ranks' measurements: throughputs add up, percentiles take the worst rank
    all_pc = gather_objects((pc_lookups["lookups_per_s"], pc_mix["requests_per_s"]))
    if world > 1:
        sweep = merge_serving_points(gather_objects(sweep))
        ra_sweep = merge_serving_points(gather_objects(ra_sweep))
        resident_gb = sum(gather_objects(resident_gb))
        chk_ok = all(gather_objects(chk_ok))
    per_call_lps = sum(x[0] for x in all_pc)

    def ok_point(p):
        return p["lookup_p99_us"] is not None and p["lookup_p99_us"] <= 1000.0
    good = [p for p in sweep + ra_sweep if ok_point(p)]
    best = max(good, key=lambda p: p["lookups_per_s"]) if good else None
    value = best["lookups_per_s"] if best else 0.0
    peak, peak_kind = measured_peak()
    if best:
        bpv = {i: sources[i]["bits"] / 8 for i in range(len(sources))}
        alg = best["lookups_per_s"] * 44 + best["range_gb_s"] * 1e9 * (1 + float(np.mean(list(bpv.values()))) / 8)
    else:
        alg = 0.0
    st = server.stats()
    st_all = gather_objects((int(st.evictions), int(st.admissions_refused), int(st.launches)))
    if rank != 0:
        server.close()
        for s in sources:
            s["col"].free()
        ctx.close()
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return 0
    line = {
        "metric": "served lookups/s at lookup p99 <= 1 ms", "value": round(value, 1), "unit": "lookups/s",
        "n_gpus": world, "steps": len(sweep) + len(ra_sweep), "warmup": args.warmup,
        "ms_per_step": round(1e3 * (best["span_s"] if best else 0.0), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "mixed int32/int64/uint64", "data": "synthetic",
        "config": {"workload": "serving_64_columns_poisson", "columns": len(ids) * world,
                   "sharding": "whole columns per GPU: every rank its own server and columns (weak scaling); "
                               "rate points are per GPU, merged by summing throughput and taking the worst "
                               "rank's percentiles" if world > 1 else "one GPU",
                   "resident_gb": round(resident_gb, 2),
                   "budget_gb": round(budget / 1e9, 1), "slots": args.slots,
                   "sources": [f"{s['copies']} x {s['name']}" for s in sources],
                   "lookup_sizes": "floor(exp(U[0, ln 65536])) positions, uniform over the column",
                   "range_sizes": "floor(exp(U[ln 1024, ln 16M])) values",
                   "mix": "50/50 lookup/range (sweep); lookups only (ra_sweep)",
                   "admission_s": round(admit_s, 2), "build_s": round(build_s, 1), "bit_exact": chk_ok,
                   "best_point": best, "sweep": sweep, "ra_sweep": ra_sweep,
                   "per_call_lookups_per_s": round(per_call_lps, 1),
                   "per_call": {"form": "one glc_random_access / glc_decompress_range call per request from a "
                                        "C++ loop, one stream, back to back (device time)",
                                "lookups_only": pc_lookups, "mix_50_50": pc_mix},
                   "served_over_per_call": round(value / per_call_lps, 2) if per_call_lps else None,
                   "evictions_total": sum(x[0] for x in st_all),
                   "admissions_refused_total": sum(x[1] for x in st_all),
                   "l2": "columns, positions and outputs far larger than L2"},
        "roofline": {"bound": "hbm", "achieved": round(alg / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(alg / 1e9 / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "basis": "whole served stream at the best point: 44 B per lookup + range bytes written "
                              "and read, over the stream's span"},
        "e2e": None, "gpu_launches": sum(x[2] for x in st_all), "clocks": clk, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    server.close()
    for s in sources:
        s["col"].free()
    ctx.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
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
    ap.add_argument("--no-loops", action="store_true",
                    help="c4 batch: skip the per-column comparison loops (a short launch list for ncu)")
    ap.add_argument("--workload", default="c2_decode",
                    choices=["c1_plain", "c2_decode", "c3_random_access", "c4_batch", "c5_serving", "compress",
                             "decode_i32"],
                    help="c2_decode (headline): full decode of the 200M piecewise uint64 column; "
                         "c3_random_access: 100M lookups into a 64M int64 timestamp column")
    ap.add_argument("--mode", default="packed", choices=["packed", "preunpacked"], help="c3 residual source")
    ap.add_argument("--noise-bits", type=int, default=6, help="decode_i32: noise bits of the int32 column")
    ap.add_argument("--partitioning", default="fixed", choices=["fixed", "v6", "variable"],
                    help="compress: fixed partitions of 4096, the reference's GPU partitioner, or split/merge")
    ap.add_argument("--queries", type=int, default=100_000_000, help="c3 lookups per step")
    ap.add_argument("--rates", default="10000,30000,100000,300000,1000000", help="c5: request rates (req/s)")
    ap.add_argument("--ra-rates", default="1000000,2000000,4000000,8000000", help="c5: lookup-only request rates")
    ap.add_argument("--serve-seconds", type=float, default=0.5, help="c5: scheduled duration per rate")
    ap.add_argument("--serve-scale", type=float, default=1.0, help="c5: column length scale (1 = full size)")
    ap.add_argument("--slots", type=int, default=4, help="c5: shared launches in flight")
    ap.add_argument("--max-range-values", type=int, default=0, help="c5: range values per launch (0 = server default)")
    ap.add_argument("--admit-during", type=int, default=8, help="c5: columns admitted during each rate point")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "c1_plain":
        return run_c1(args)
    if args.workload == "c3_random_access":
        return run_random_access(args)
    if args.workload == "c4_batch":
        return run_batch(args)
    if args.workload == "c5_serving":
        return run_serving(args)
    if args.workload == "compress":
        return run_compress(args)
    if args.workload == "decode_i32":
        return run_decode_i32(args)

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
    ctx = tuned_context(glc, local)

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
    clocks.begin()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clocks.end()
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
    traffic = profiled_traffic(n)

    # end to end through the C ABI with host buffers: host blob -> device -> decode -> host
    blob = glc.serialize_host(ctx, col)
    h_blob = torch.from_numpy(np.frombuffer(blob, np.uint8).copy()).pin_memory()
    h_out = torch.empty(n, dtype=torch.int64).pin_memory()
    lib = ctx.lib
    import ctypes

    def e2e_step():  # glc_decode_blob_to_host: upload, decode and download overlapped in chunks
        ctx.check(lib.glc_decode_blob_to_host(ctx.handle, glc.U64, ctypes.c_void_p(h_blob.data_ptr()), len(blob), 0,
                                              ctypes.c_void_p(h_out.data_ptr()), None, ctypes.c_void_p(sh)))

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
            cpu = cpu_baseline_decode(blob, values, host_threads())
        except Exception as ex:  # reported, never fatal
            cpu = {"value": None, "unit": UNIT, "cores": host_threads(), "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "values": n, "partitions": info.num_partitions,
                       "tuned_shape": glc.tune_get(ctx, glc.U64, info.max_delta_bits).as_dict(),
                       "bits_per_value": round(info.total_bits / n, 3),
                       "compressed_bytes": info.compressed_size_bytes,
                       "compression_ratio": round(decoded_bytes / info.compressed_size_bytes, 3),
                       "l2": "inputs and output larger than L2 (no flush)", "parallelism": f"replicas{world}",
                       "compress_s": round(compress_s, 3), "bit_exact": ok and e2e_ok},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_source": os.path.relpath(TRAFFIC_JSON, ROOT),
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
