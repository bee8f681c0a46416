"""bench.py - suffix array + BWT construction throughput on B200, and the reference CPU arm.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload genome3g|natural256m|natural64m|uniform8m]
    python bench.py --workload batch4096 | serve | lcp256m    batched, served, LCP array from text + SA
    python bench.py --impl reference ...       the reference's CPU variant on the host cores
    python bench.py --impl reference-gpu ...   the reference's own CUDA build on this GPU

One step = one construction of the SA (uint32) and BWT of the workload's text, produced together.
The default workload is the 3 GiB genome-like text (uint32 SA past the reference's int32 limit).
``value`` is device throughput with the text resident in HBM (CUDA events on the stream the library
launches on, max over ranks); ``e2e`` is the same metric through the host C ABI (sadcs_gpu_build)
from page-locked host memory, with the upload of the text and the download of SA and BWT inside
the timed region. MB/s is MiB/s (the reference's convention, main.cpp:175-177).

Roofline: HBM-bound integer work. ``roofline`` covers the dominant kernel (the final merge), timed
live with CUDA events around its launch; its algorithmic bytes per input byte are 53 (class lists
4, one 44-byte comparison record per element: 16 text bytes + 7 sample ranks, SA write 4, BWT write
1). ``pipeline_roofline`` credits the whole construction with the fixed 82.125 bytes per input byte
of the reference pipeline's named steps (sample ranking 12.375, class lists 11.75, merge 52, SA->BWT
6). Peak = the measured HBM copy bandwidth in MEASURED_PEAKS.json (fallback 6650 GB/s).

Multi-GPU: a single text does not shard, so N ranks build N independent replicas ("replicas",
weak scaling); value = N * n / max-over-ranks time. Without a launcher, --gpus N > 1 starts the N
ranks itself (torch.distributed.run on this node).

Beside the line's own figures: ``cpu_baseline`` (the reference's CPU build on a prefix sample, the
same sample as the --impl reference arm) and, on one GPU, ``reference_gpu`` (the reference's own
CUDA build on this GPU, on the largest prefix its int32 API takes, SA then BWT, next to this
library's construction of the same prefix) and ``batch`` (the batch4096 workload: one batched
construction of 4096 uneven texts against one construction per text on a sample of them, whose
outputs are checked equal).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "input MB/s (bit-exact SA+BWT, % HBM roofline)"
UNIT = "MiB/s"
MIB = float(1 << 20)
PIPELINE_BYTES_PER_INPUT_BYTE = 82.125
MERGE_BYTES_PER_INPUT_BYTE = 53.0
# LCP array (sadcs_gpu_lcp), per position: Phi scatter 4 + 4, irreducible test 4 + 1 + 1 + 4 (the
# character comparisons are not credited), max-scan 4 + 4, gather 4 + 4 + 4.
LCP_BYTES_PER_POSITION = 38.0
FALLBACK_HBM_GBS = 6650.0

BATCH_DESC = ("4096 texts, lengths log-uniform in [1 KiB, 4 MiB], thirds over {A,C,G,T}, a 20-letter protein-like "
              "alphabet with background frequencies, and uniform bytes; seed 4; one batched construction per step")
SERVE_DESC = ("serving stream: Poisson arrivals at offered loads 50/200/800 req/s, lengths log-uniform in "
              "[4 KiB, 64 MiB] plus 1% at 1 GiB, alphabets as the batched config; seed 5")

WORKLOADS = {
    "natural256m": ("256 MiB natural-language-like text: 50k-word lowercase vocabulary (lengths 2-12), "
                    "Zipf(1.1) words, '.\\n' every 10-30 words, 2% capitalised, seed 2",
                    lambda W: W.natural_text(256 << 20, seed=2)),
    "natural64m": ("64 MiB natural-language-like text, as natural256m (the profiling case: its merge reads "
                   "3.4 GB, far above L2, with 0.75 GB on the device)",
                   lambda W: W.natural_text(64 << 20, seed=2)),
    "uniform8m": ("8 MiB i.i.d. uniform bytes, seed 1", lambda W: W.uniform_bytes(8 << 20, seed=1)),
    "genome3g": ("3 GiB {A,C,G,T}: 2 GiB i.i.d. GC 0.41, then 1 GiB of mutated copies of 1 MiB segments "
                 "(1% substitutions, 0.1% indels of 1-10), seed 3", lambda W: W.genome_text(3 << 30, seed=3)),
    "genome256m": ("256 MiB {A,C,G,T} built as genome3g at 1/12 the size (the profiling case: its 235 MB rank "
                   "array exceeds L2, with about 4.5 GB on the device)",
                   lambda W: W.genome_text(256 << 20, seed=3)),
}
# The first k bytes of a workload's text without generating all of it, where the generator allows.
PREFIXES = {"genome3g": lambda W, k: W.genome_text(3 << 30, seed=3, prefix=k)}
WORKLOAD_BYTES = {"natural256m": 256 << 20, "natural64m": 64 << 20, "uniform8m": 8 << 20, "genome3g": 3 << 30,
                  "genome256m": 256 << 20}
DEFAULT_WORKLOAD = "genome3g"
REFERENCE_INT32_LIMIT = (1 << 31) - 1025  # the reference's largest input (src/cpu/dcsort.h:21)


def workload_prefix(name: str, k: int) -> np.ndarray:
    from sadcs_b200 import workloads as W

    if name in PREFIXES and k <= (WORKLOAD_BYTES[name] * 2) // 3:
        return PREFIXES[name](W, k)
    return np.ascontiguousarray(WORKLOADS[name][1](W)[:k])


def workload_config(name: str, n: int, world: int) -> dict:
    """The line's `config`, the same in this library's arm and the reference arm."""
    return {"workload": name, "description": WORKLOADS[name][0], "text_bytes": n,
            "outputs": "SA + BWT of the text", "l2": "inputs larger than L2 (text %d MiB)" % (n >> 20),
            "parallelism": "replicas" if world > 1 else "single GPU"}


def hbm_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---- clocks -----------------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons for one GPU during the timed region."""

    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={','.join(self.FIELDS)}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        loaded = [v for v in sm if v >= 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- distributed plumbing -----------------------------------------------------------------------

def rank_env():
    """(world, rank, local rank) from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_setup(gpus: int):
    """Joins the process group of a multi-GPU run. Ranks are independent replicas (one text, batch
    or request stream each, no data-path collective); the group only carries the barriers around
    the timed region and the max/sum of the per-rank results. NCCL on GPUs; gloo where SADCS_DIST_BACKEND
    says so (the CPU tests of this host logic)."""
    world, rank, local = rank_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        backend = os.environ.get("SADCS_DIST_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _all_reduce(value: float, world: int, op: str) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, world: int) -> float:
    return _all_reduce(value, world, "max")


def sum_over_ranks(value: float, world: int) -> float:
    return _all_reduce(value, world, "sum")


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's own synthetic request stream (weak scaling: each rank its own)."""
    return base + 1000 * rank


def batch_share(count_per_rank: int, world: int, rank: int) -> list[int]:
    """This rank's texts of one batch of count_per_rank * world texts, partitioned across ranks by
    construction footprint (greedy longest-first); no data crosses between GPUs."""
    from sadcs_b200 import workloads as W

    lengths = W.batch_lengths(count_per_rank * world, lo=1 << 10, hi=4 << 20, seed=4)
    return W.partition_by_footprint(lengths, world)[rank]


# ---- CPU baseline (the reference's own CPU variant, or the oracle port) ----------------------------

def cpu_baseline(sample: np.ndarray) -> dict:
    """The reference's CPU build (or the oracle port) on a prefix sample of the workload's text:
    SA then BWT, as the reference's CLI builds them."""
    import oracle

    sample = np.ascontiguousarray(sample)
    if oracle.ref_available():
        L = oracle.ref()
        cores = oracle.host_cores()
        L.ref_set_threads(cores)
        t0 = time.perf_counter()
        oracle.ref_sa(sample)
        t1 = time.perf_counter()
        oracle.ref_bwt(sample)
        t2 = time.perf_counter()
        return {"value": round(len(sample) / MIB / (t2 - t0), 3), "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"first {len(sample) / MIB:.0f} MiB of the workload text: reference CPU buildSuffixArray "
                          f"({t1 - t0:.2f} s) then buildBwt ({t2 - t1:.2f} s), cover 128, {cores} threads"}
    t0 = time.perf_counter()
    sa = oracle.doubling_sa(sample)
    oracle.bwt_from_sa(sample, sa)
    t1 = time.perf_counter()
    return {"value": round(len(sample) / MIB / (t1 - t0), 3), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"first {len(sample) / MIB:.0f} MiB: oracle prefix-doubling SA + BWT, 1 thread"}


def run_reference(args, world, rank) -> None:
    """--impl reference: the reference's CPU implementation on this host's cores, rank 0 only."""
    if rank != 0:
        return
    import oracle
    from sadcs_b200 import workloads as W

    n = WORKLOAD_BYTES[args.workload]
    n_sample = min(n, args.reference_sample_mib << 20)
    sample = workload_prefix(args.workload, n_sample)
    if oracle.ref_available():
        L = oracle.ref()
        cores = oracle.host_cores()
        L.ref_set_threads(cores)
        kind = "reference"

        def step():
            oracle.ref_sa(sample)
            oracle.ref_bwt(sample)
    else:
        cores = 1
        kind = "port"

        def step():
            sa = oracle.dc_sa(sample)
            oracle.bwt_from_sa(sample, sa)
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    mean = sum(times) / len(times)
    value = n_sample / MIB / mean
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload_config(args.workload, n, 1),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"first {n_sample / MIB:.0f} MiB of the workload text per step (of "
                                       f"{n / MIB:.0f} MiB), SA then BWT (two runs), "
                                       f"{'reference CPU build (cover 128)' if kind == 'reference' else 'oracle port'}"},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_reference_gpu(text: np.ndarray, steps: int, warmup: int) -> dict:
    """The reference's own CUDA build (oracle/_ref/libsadcs_ref_gpu.so: its gpusa.cu compiled
    unchanged for sm_100a) on this GPU, as its CLI's `bench --context --pinned` measures it:
    page-locked host buffers, one context, gpuSuffixArray then gpuBwt per step (the reference
    builds SA and BWT in two constructions), host to host; device time from its own GpuStats.
    Returns the figures, or {"unavailable": why}."""
    import oracle

    if not oracle.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libsadcs_ref_gpu.so not built (make -C oracle ref-gpu needs the "
                               "reference sources)"}
    n = int(len(text))
    if n > REFERENCE_INT32_LIMIT:
        return {"unavailable": "the reference's GPU API takes int32 sizes up to 2^31 - 1025 bytes"}
    try:
        ctx = oracle.RefGpuContext(n)
    except RuntimeError as e:
        return {"unavailable": str(e)}
    h_text = oracle.ref_gpu_pinned(n)
    h_sa = oracle.ref_gpu_pinned(4 * n)
    h_bwt = oracle.ref_gpu_pinned(n)
    try:
        if h_text is None or h_sa is None or h_bwt is None:
            return {"unavailable": "the reference's gpuAllocatePinned failed"}
        h_text[:] = text
        sa_view = h_sa.view(np.int32)
        sa_ms, bwt_ms = [], []

        def step():
            _, sa_dev = ctx.suffix_array(h_text, out=sa_view)
            _, primary, bwt_dev = ctx.bwt(h_text, out=h_bwt)
            return sa_dev, bwt_dev

        for _ in range(max(warmup, 0)):
            step()
        host = []
        for _ in range(steps):
            t0 = time.perf_counter()
            a, b = step()
            host.append(time.perf_counter() - t0)
            sa_ms.append(a * 1e3)
            bwt_ms.append(b * 1e3)
        mean_host = sum(host) / len(host)
        mean_dev = (sum(sa_ms) + sum(bwt_ms)) / len(host)
        return {"value": round(n / MIB / mean_host, 3), "unit": UNIT, "ms_per_step": round(mean_host * 1e3, 3),
                "device_value": round(n / MIB / (mean_dev / 1e3), 3), "device_ms_per_step": round(mean_dev, 3),
                "device_ms_sa": round(sum(sa_ms) / len(sa_ms), 3), "device_ms_bwt": round(sum(bwt_ms) / len(bwt_ms), 3),
                "text_bytes": n, "steps": steps, "warmup": warmup,
                "outputs": "SA (int32) by gpuSuffixArray, then BWT by gpuBwt (two constructions)",
                "cover": "mod 32 (the reference's GPU cover)", "build": "reference gpusa.cu, nvcc 12.9, sm_100a",
                "h2d_bytes_per_step": 2 * n, "d2h_bytes_per_step": 5 * n}
    finally:
        ctx.close()
        for a in (h_text, h_sa, h_bwt):
            if a is not None:
                oracle.ref_gpu_free_pinned(a)


def run_reference_gpu(args, world, rank) -> None:
    """--impl reference-gpu: time_reference_gpu on the workload's text (or its largest prefix the
    reference takes). Rank 0 only."""
    if rank != 0:
        return
    n = min(WORKLOAD_BYTES[args.workload], REFERENCE_INT32_LIMIT)
    record = time_reference_gpu(workload_prefix(args.workload, n), args.steps, args.warmup)
    base = {"impl": "reference-gpu", "metric": METRIC, "unit": UNIT}
    if "unavailable" in record:
        print(json.dumps({**base, **record}), flush=True)
        return
    print(json.dumps({
        **base, "value": record["value"], "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": record["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic", "config": workload_config(args.workload, n, 1),
        "device_value": record["device_value"], "device_ms_per_step": record["device_ms_per_step"],
        "e2e": {"value": record["value"], "unit": UNIT, "h2d_bytes_per_step": record["h2d_bytes_per_step"],
                "d2h_bytes_per_step": record["d2h_bytes_per_step"],
                "api": "gpuSuffixArray + gpuBwt with a context and page-locked buffers"},
    }), flush=True)


def reference_gpu_record(args, d_text, ctx, text: np.ndarray, stream) -> dict:
    """The kernel bar: the reference's CUDA build and this library on the same input (the
    workload's text, or its largest prefix the reference's int32 API takes), on this GPU. Ours is
    one construction of SA + BWT, device time by CUDA events; the reference's is its SA and its
    BWT construction, device time by its own stats."""
    import torch

    import sadcs_b200 as sa

    n = min(len(text), REFERENCE_INT32_LIMIT)
    record = time_reference_gpu(np.ascontiguousarray(text[:n]), args.reference_gpu_steps, 1)
    if "unavailable" in record:
        return record
    d_sa = torch.empty(n, dtype=torch.int32, device=d_text.device)
    d_bwt = torch.empty(n, dtype=torch.uint8, device=d_text.device)
    times = []
    for i in range(1 + args.reference_gpu_steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sa.build_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_bwt.data_ptr(), context=ctx,
                        stream=stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        if i > 0:
            times.append(a.elapsed_time(b))
    ours_ms = sum(times) / len(times)
    record["ours_same_input"] = {"device_ms_per_step": round(ours_ms, 3),
                                 "device_value": round(n / MIB / (ours_ms / 1e3), 3),
                                 "outputs": "SA (uint32) + BWT from one construction"}
    record["device_speedup"] = round(record["device_ms_per_step"] / ours_ms, 3)
    record["input"] = "the workload text" if n == len(text) else f"the first {n} bytes of the workload text"
    return record


# ---- our arm --------------------------------------------------------------------------------------

def run_ours(args, world, rank, local) -> None:
    import torch

    import sadcs_b200 as sa
    from sadcs_b200 import workloads as W

    torch.cuda.set_device(local)
    desc, gen = WORKLOADS[args.workload]
    text = gen(W)
    n = int(len(text))
    props = torch.cuda.get_device_properties(local)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else (str(uuid) if uuid else None)

    d_text = torch.from_numpy(text).to(f"cuda:{local}")
    d_sa = torch.empty(n, dtype=torch.int32, device=f"cuda:{local}")
    d_bwt = torch.empty(n, dtype=torch.uint8, device=f"cuda:{local}")
    ctx = sa.Context(n)
    stream = torch.cuda.current_stream()
    handle = stream.cuda_stream
    stats = sa.Stats()

    def step():
        return sa.build_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_bwt.data_ptr(), context=ctx,
                               stream=handle, stats=stats)

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    merge_ms, launches, phases = [], 0, {"ranking": [], "classes": [], "merge": []}
    start.record(stream)
    for _ in range(args.steps):
        primary = step()
        merge_ms.append(stats.merge_kernel_ms)
        launches += int(stats.kernel_launches)
        phases["ranking"].append(stats.ranking_device_ms)
        phases["classes"].append(stats.class_sort_device_ms)
        phases["merge"].append(stats.merge_device_ms)
    stop.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = start.elapsed_time(stop) / args.steps
    ms_max = max_over_ranks(ms, world)
    total_bytes = sum_over_ranks(float(n), world)
    value = total_bytes / MIB / (ms_max / 1e3)

    # Verification of the last step's output (size-independent checks on the device, test-side):
    # SA is a permutation in suffix order by the Burkhardt-Karkkainen neighbour test, BWT = T[SA-1].
    verified = verify_on_device(d_text, d_sa, d_bwt, primary) if args.verify else None

    e2e = run_e2e(args, text, ctx, world) if args.e2e else None

    if rank != 0:
        return
    peak, peak_kind = hbm_peak()
    merge_avg = sum(merge_ms) / len(merge_ms)
    merge_gbs = MERGE_BYTES_PER_INPUT_BYTE * n / (merge_avg / 1e3) / 1e9
    pipe_gbs = PIPELINE_BYTES_PER_INPUT_BYTE * n / (ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "mergeTree<final> (last merge level: tiles of the 7 class lists merged in shared memory, writing SA + BWT)",
                "achieved": round(merge_gbs, 1), "peak": peak, "unit": "GB/s", "frac": round(merge_gbs / peak, 4),
                "traffic": None, "algorithmic_bytes_per_input_byte": MERGE_BYTES_PER_INPUT_BYTE,
                "kernel_ms": round(merge_avg, 3), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    traffic = profile_traffic(args.workload)
    if traffic:
        roofline["traffic"] = round(traffic[0] * n)
        roofline["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the final merge per input "
                                      "byte, captured on %s (profiles/traffic.json), times n%s" % (
                                          traffic[1], "" if traffic[1] == args.workload else
                                          ": scaled to this size, a lower bound (the tie-breaking rank reads hit L2 less)"))
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload_config(args.workload, n, world),
            "construction": {"outputs": "SA (uint32) + BWT from one construction", "cover": "mod 32 (7 of 32)",
                             "working_set_gb": round(sa.required_bytes(n) / 1e9, 2)},
            "roofline": roofline,
            "pipeline_roofline": {"bound": "hbm", "achieved": round(pipe_gbs, 1), "peak": peak, "unit": "GB/s",
                                  "frac": round(pipe_gbs / peak, 4),
                                  "algorithmic_bytes_per_input_byte": PIPELINE_BYTES_PER_INPUT_BYTE},
            "phases_ms": {k: round(sum(v) / len(v), 3) for k, v in phases.items()},
            "character_passes": int(stats.character_passes), "doubling_rounds": int(stats.doubling_rounds),
            "device_bytes_per_input_byte": round(stats.device_bytes / n, 3),
            "clocks": clocks, "gpu_launches": launches, "verified": verified}
    if e2e:
        line["e2e"] = e2e
    if world == 1 and args.cpu_sample_mib > 0:
        line["cpu_baseline"] = cpu_baseline(text[:args.cpu_sample_mib << 20])
    if world == 1 and args.reference_gpu_steps > 0:
        line["reference_gpu"] = reference_gpu_record(args, d_text, ctx, text, stream)
    if world == 1 and args.batch_steps > 0:
        # the batched configuration beside the headline (its own workload: 4096 uneven texts)
        ctx.close()
        del d_text, d_sa, d_bwt
        torch.cuda.empty_cache()
        line["batch"] = {"workload": "batch4096", "description": BATCH_DESC,
                         **measure_batch(args, 1, 0, local, args.batch_steps, 2, clocks=False)}
    print(json.dumps(line), flush=True)


def run_e2e(args, text, ctx, world):
    """sadcs_gpu_build from page-locked host memory: upload, construction, SA + BWT download."""
    import ctypes

    import sadcs_b200 as sa

    n = len(text)
    h_text = sa.allocate_pinned(n)
    h_sa = sa.allocate_pinned(4 * n)
    h_bwt = sa.allocate_pinned(n)
    try:
        h_text[:] = text
        primary = ctypes.c_int64(-1)
        L = sa.lib()

        def step():
            status = L.sadcs_gpu_build(ctx.handle, h_text.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n,
                                       ctypes.cast(h_sa.ctypes.data, ctypes.POINTER(ctypes.c_uint32)),
                                       h_bwt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.byref(primary),
                                       None)
            if status != 0:
                raise sa.GpuError(status, sa.last_error())

        step()
        steps = max(1, min(args.steps, args.e2e_steps))
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        seconds = (time.perf_counter() - t0) / steps
        seconds = max_over_ranks(seconds, world)
        total = sum_over_ranks(float(n), world)
        return {"value": round(total / MIB / seconds, 3), "unit": UNIT, "h2d_bytes_per_step": n,
                "d2h_bytes_per_step": 5 * n, "ms_per_step": round(seconds * 1e3, 3),
                "api": "sadcs_gpu_build (host C ABI, page-locked buffers)", "steps": steps}
    finally:
        sa.free_pinned(h_text)
        sa.free_pinned(h_sa)
        sa.free_pinned(h_bwt)


def verify_on_device(d_text, d_sa, d_bwt, primary) -> bool:
    """SA: a permutation in suffix order (Burkhardt-Karkkainen neighbour test); BWT: T[SA - 1] in
    the divsufsort convention. Torch arithmetic up to 1 GiB; above that (its int64 temporaries would
    not fit) the library's device checkers, the restated reference checks."""
    import torch

    n = d_text.numel()
    if n > (1 << 30):
        import sadcs_b200 as sa

        ok_sa, _, _ = sa.check_suffix_array_device(d_text.data_ptr(), n, d_sa.data_ptr())
        ok_bwt, _ = sa.check_bwt_device(d_text.data_ptr(), n, d_bwt.data_ptr(), int(primary))
        return bool(ok_sa and ok_bwt)
    s = d_sa.to(torch.int64)
    isa = torch.empty(n + 1, dtype=torch.int64, device=d_text.device)
    isa[n] = -1
    isa[s] = torch.arange(n, device=d_text.device)
    if not bool((isa[:n][s] == torch.arange(n, device=d_text.device)).all()):
        return False
    t = d_text.to(torch.int64)
    left, right = s[:-1], s[1:]
    tl, tr = t[left], t[right]
    nl, nr = isa[left + 1], isa[right + 1]
    ok = (tl < tr) | ((tl == tr) & (nl < nr))
    if not bool(ok.all()):
        return False
    rows = torch.arange(n, device=d_text.device)
    row0 = int(rows[s == 0].item())
    expected = torch.empty(n, dtype=torch.uint8, device=d_text.device)
    expected[0] = d_text[n - 1]
    keep = s != 0
    idx = torch.where(rows < row0, rows + 1, rows)[keep]
    expected[idx] = d_text[(s[keep] - 1)]
    return bool(primary == row0 + 1 and torch.equal(expected, d_bwt))


def profile_traffic(workload: str):
    """(DRAM bytes per input byte of the final merge kernel, the workload they were captured on),
    from the committed ncu summary (profiles/traffic.json), or None."""
    path = ROOT / "profiles" / "traffic.json"
    try:
        entry = json.loads(path.read_text())[workload]
        return float(entry["merge_dram_bytes_per_input_byte"]), entry.get("scaled_from", workload)
    except Exception:
        return None


def scan_launches(count: int) -> int:
    """Kernels of the library's device-wide scan of count elements (primitives.cuh deviceScan)."""
    if count == 0:
        return 0
    blocks = -(-count // 4096)
    return 1 if blocks == 1 else 2 + scan_launches(blocks)


def run_lcp(args, world, rank, local) -> None:
    """The LCP array of the natural256m text's suffix array (sadcs_gpu_lcp) on device buffers; the
    suffix array is built once, outside the timed region. Each step is one call, its scratch
    allocation (stream-ordered) included."""
    import torch

    import oracle
    import sadcs_b200 as sa
    from sadcs_b200 import workloads as W

    torch.cuda.set_device(local)
    desc, gen = WORKLOADS["natural256m"]
    text = gen(W)
    n = int(len(text))
    props = torch.cuda.get_device_properties(local)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else (str(uuid) if uuid else None)
    device = f"cuda:{local}"
    d_text = torch.from_numpy(text).to(device)
    d_sa = torch.empty(n, dtype=torch.int32, device=device)
    d_lcp = torch.empty(n, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream()
    handle = stream.cuda_stream
    sa.build_device(d_text.data_ptr(), n, d_sa.data_ptr(), None, stream=handle)

    def step():
        sa.lcp_device(d_text.data_ptr(), n, d_sa.data_ptr(), d_lcp.data_ptr(), stream=handle)

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step()
    stop.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = start.elapsed_time(stop) / args.steps
    ms_max = max_over_ranks(ms, world)
    value = sum_over_ranks(float(n), world) / MIB / (ms_max / 1e3)
    verified = None
    if args.verify:
        h_sa = d_sa.cpu().numpy().view(np.uint32)
        verified = bool(np.array_equal(d_lcp.cpu().numpy().view(np.uint32), oracle.lcp(text, h_sa)))
    if rank != 0:
        return
    peak, peak_kind = hbm_peak()
    gbs = LCP_BYTES_PER_POSITION * n / (ms / 1e3) / 1e9
    line = {"metric": "input MB/s (LCP array from text + SA)", "value": round(value, 3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "lcp256m", "description": desc, "text_bytes": n,
                       "outputs": "LCP (uint32) from device text + SA", "l2": "inputs larger than L2",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "kernel": "all LCP passes of one call (Phi, irreducible test, warp "
                         "pass, max-scan, gather)", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "traffic": None,
                         "algorithmic_bytes_per_input_byte": LCP_BYTES_PER_POSITION,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "clocks": clocks, "gpu_launches": args.steps * (4 + scan_launches(n)), "verified": verified}
    print(json.dumps(line), flush=True)


def measure_batch(args, world, rank, local, steps: int, warmup: int, clocks: bool = True) -> dict:
    """Config 4: many uneven texts in one construction (sadcs_gpu_build_batch_device), against one
    construction per text on a bounded sample of the same texts (device-resident both). Every
    sampled text's SA, BWT and primary from the batch are checked against its own construction."""
    import torch

    import sadcs_b200 as sa
    from sadcs_b200 import workloads as W

    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    texts = W.batch_texts(args.batch_count * world, lo=1 << 10, hi=4 << 20, seed=4,
                          indices=batch_share(args.batch_count, world, rank))
    lengths = [len(t) for t in texts]
    offsets = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    total = int(offsets[-1])
    packed = torch.from_numpy(np.concatenate(texts)).to(device)
    d_sa = torch.empty(total, dtype=torch.int32, device=device)
    d_bwt = torch.empty(total, dtype=torch.uint8, device=device)
    ctx = sa.Context(total, max_texts=len(texts))
    stream = torch.cuda.current_stream()
    stats = sa.Stats()
    primaries = []

    def step():
        primaries[:] = sa.build_batch_device(packed.data_ptr(), lengths, d_sa.data_ptr(), d_bwt.data_ptr(),
                                             context=ctx, stream=stream.cuda_stream, stats=stats)

    for _ in range(max(warmup, 0)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(None)
    if clocks:
        sampler.start()
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    start.record(stream)
    for _ in range(steps):
        step()
        launches += int(stats.kernel_launches)
    stop.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clock_record = sampler.stop() if clocks else None
    ms = start.elapsed_time(stop) / steps
    ms_max = max_over_ranks(ms, world)
    value = sum_over_ranks(float(total), world) / MIB / (ms_max / 1e3)
    texts_total = sum_over_ranks(float(len(texts)), world)
    ctx.close()

    # The plain path: one construction per text (a bounded sample of the same texts), device-resident.
    picks = list(range(0, len(texts), max(1, len(texts) // args.plain_sample)))[: args.plain_sample]
    longest = max(lengths[i] for i in picks)
    one = sa.Context(longest)
    p_sa = torch.empty(longest, dtype=torch.int32, device=device)
    p_bwt = torch.empty(longest, dtype=torch.uint8, device=device)
    plain_bytes, plain_ms, same = 0, 0.0, True
    for i in picks:
        lo, hi = int(offsets[i]), int(offsets[i + 1])
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        p = sa.build_device(packed[lo:hi].data_ptr(), lengths[i], p_sa.data_ptr(), p_bwt.data_ptr(), context=one,
                            stream=stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        plain_ms += a.elapsed_time(b)
        plain_bytes += lengths[i]
        same = same and p == primaries[i] and torch.equal(p_sa[:hi - lo], d_sa[lo:hi]) and \
            torch.equal(p_bwt[:hi - lo], d_bwt[lo:hi])
    one.close()
    plain = plain_bytes / MIB / (plain_ms / 1e3)
    return {"value": round(value, 3), "unit": UNIT, "ms_per_step": round(ms_max, 3), "steps": steps,
            "warmup": warmup, "texts": len(texts), "total_bytes": total,
            "texts_per_s": round(texts_total / (ms_max / 1e3), 1),
            "plain_one_text_per_launch": {"value": round(plain, 3), "unit": UNIT, "texts": len(picks),
                                          "texts_per_s": round(len(picks) / (plain_ms / 1e3), 1)},
            "speedup_vs_plain": round(value / world / plain, 2), "gpu_launches": launches,
            "sample_equal_to_plain": bool(same), "clocks": clock_record}


def run_batch(args, world, rank, local) -> None:
    """--workload batch4096: measure_batch as the line's own figures."""
    r = measure_batch(args, world, rank, local, args.steps, args.warmup)
    if rank == 0:
        print(json.dumps({
            "metric": "batched input MB/s (bit-exact SA+BWT per text)", "value": r["value"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "batch4096", "description": BATCH_DESC, "texts": r["texts"],
                       "total_bytes": r["total_bytes"], "l2": "inputs larger than L2",
                       "parallelism": ("one batch of %d texts per GPU, partitioned by footprint (longest first)"
                                       % args.batch_count) if world > 1 else "single GPU"},
            "texts_per_s": r["texts_per_s"], "plain_one_text_per_launch": r["plain_one_text_per_launch"],
            "speedup_vs_plain": r["speedup_vs_plain"], "sample_equal_to_plain": r["sample_equal_to_plain"],
            "clocks": r["clocks"], "gpu_launches": r["gpu_launches"],
        }), flush=True)


def serve_requests(rng, count: int, huge_fraction: float):
    """One request stream's texts: lengths log-uniform in [4 KiB, 64 MiB] plus huge_fraction at
    1 GiB; thirds over DNA, a protein-like alphabet and uniform bytes."""
    from sadcs_b200.workloads import protein_text

    lengths = np.exp(rng.uniform(np.log(4 << 10), np.log(64 << 20), count)).astype(np.int64)
    lengths[rng.random(count) < huge_fraction] = 1 << 30
    kinds = rng.integers(0, 3, count)
    pool, texts = {}, []
    for n, kind in zip(lengths.tolist(), kinds.tolist()):
        key = (n, kind)
        if key not in pool:
            g = np.random.default_rng(n * 3 + kind)
            if kind == 0:
                pool[key] = np.frombuffer(b"ACGT", np.uint8)[g.integers(0, 4, n)]
            elif kind == 1:
                pool[key] = protein_text(g, n)
            else:
                pool[key] = g.integers(0, 256, n, dtype=np.uint8)
        texts.append(pool[key])
    return lengths, texts


class PinnedArena:
    """Page-locked host buffers for a request stream: each request's text, SA and BWT, carved from
    one allocation (as a serving front end would hold them)."""

    def __init__(self, lengths):
        import sadcs_b200 as sa

        total = int(sum(int(n) for n in lengths))
        self.raw = sa.allocate_pinned(max(6 * total + 64 * len(lengths), 1))
        self.views = []
        at = 0
        for n in lengths:
            n = int(n)
            text = self.raw[at:at + n]
            at += (n + 15) // 16 * 16
            out_sa = self.raw[at:at + 4 * n].view(np.uint32)
            at += (4 * n + 15) // 16 * 16
            out_bwt = self.raw[at:at + n]
            at += (n + 15) // 16 * 16
            self.views.append((text, out_sa, out_bwt))

    def close(self):
        import sadcs_b200 as sa

        sa.free_pinned(self.raw)
        self.views = []


def run_serve(args, world, rank, local) -> None:
    """Config 5: Poisson request streams through the server; p50/p99 latency at each offered load,
    against the same requests built one at a time. Host buffers are page-locked in both arms."""
    import ctypes
    import threading

    import torch

    import sadcs_b200 as sa

    torch.cuda.set_device(local)
    rng = np.random.default_rng(rank_seed(5, rank))
    loads = [float(x) for x in args.serve_loads.split(",")]
    results = []
    first = None
    # One server for the whole run, as a service would keep it; a few requests first warm its
    # memory pool and kernels.
    server = sa.Server(workers=args.serve_workers, small_limit=64 << 20, batch_bytes=512 << 20, batch_texts=4096)
    warm = [server.submit(np.frombuffer(bytes(range(256)) * (1 << k), np.uint8)) for k in (4, 12, 16, 18)]
    for ticket in warm:
        server.wait(ticket)
    for load in loads:
        count = args.serve_requests
        lengths, texts = serve_requests(rng, count, args.serve_huge_fraction)
        arena = PinnedArena(lengths)
        for (dst, _, _), t in zip(arena.views, texts):
            dst[:] = t
        arrivals = np.cumsum(rng.exponential(1.0 / load, count))
        constructions0, launches0 = server.counters()
        tickets = [None] * count
        t0 = time.perf_counter()

        def producer():
            for i in range(count):
                delay = arrivals[i] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                text, out_sa, out_bwt = arena.views[i]
                tickets[i] = server.submit(text, sa=out_sa, bwt=out_bwt)

        thread = threading.Thread(target=producer)
        thread.start()
        thread.join()
        latencies, batch_sizes = [], []
        for i in range(count):
            _, _, _, lat, size = server.wait(tickets[i])
            latencies.append(lat[2])
            batch_sizes.append(size)
        elapsed = time.perf_counter() - t0
        constructions, launches = server.counters()
        constructions -= constructions0
        launches -= launches0
        total_bytes = float(lengths.sum())
        lat = np.array(latencies)
        small = lengths <= (64 << 20)

        def pct(mask, q):
            return round(float(np.percentile(lat[mask], q)) * 1e3, 2) if mask.any() else None

        results.append({"offered_req_s": load, "requests": count, "req_s": round(count / elapsed, 2),
                        "mib_s": round(total_bytes / MIB / elapsed, 2),
                        "offered_mib_s": round(total_bytes / MIB / float(arrivals[-1]), 2),
                        "p50_ms": round(float(np.percentile(latencies, 50)) * 1e3, 2),
                        "p99_ms": round(float(np.percentile(latencies, 99)) * 1e3, 2),
                        "up_to_64mib": {"requests": int(small.sum()), "p50_ms": pct(small, 50), "p99_ms": pct(small, 99)},
                        "at_1gib": {"requests": int((~small).sum()), "p50_ms": pct(~small, 50),
                                    "max_ms": round(float(lat[~small].max()) * 1e3, 2) if (~small).any() else None},
                        "mean_batch": round(float(np.mean(batch_sizes)), 2), "constructions": constructions,
                        "gpu_launches": launches})
        if first is None:
            first = (lengths, arena)
        else:
            arena.close()
    server.close()
    # The plain path: the first load's requests built one at a time through sadcs_gpu_build, host to
    # host from the same page-locked buffers.
    lengths, arena = first
    ctx = sa.Context(int(lengths.max()))
    L = sa.lib()
    primary = ctypes.c_int64(-1)
    t0 = time.perf_counter()
    for text, out_sa, out_bwt in arena.views:
        status = L.sadcs_gpu_build(ctx.handle, text.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), len(text),
                                   out_sa.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                   out_bwt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.byref(primary), None)
        if status != 0:
            raise sa.GpuError(status, sa.last_error())
    plain_s = time.perf_counter() - t0
    ctx.close()
    arena.close()
    plain = float(lengths.sum()) / MIB / plain_s
    if rank == 0:
        best = max(results, key=lambda r: r["mib_s"])
        print(json.dumps({
            "metric": "served input MB/s with p50/p99 latency (bit-exact SA+BWT)", "value": best["mib_s"],
            "unit": UNIT, "n_gpus": world, "steps": len(loads), "warmup": 0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": "serve", "description": SERVE_DESC, "workers": args.serve_workers,
                       "host_buffers": "page-locked", "small_limit_bytes": 64 << 20, "batch_bytes": 512 << 20},
            "loads": results,
            "plain_one_at_a_time": {"value": round(plain, 2), "unit": UNIT, "requests": len(lengths),
                                    "seconds": round(plain_s, 3),
                                    "api": "sadcs_gpu_build per request, host to host, same page-locked buffers"},
            "speedup_vs_plain": round(best["mib_s"] / plain, 2),
        }), flush=True)


def launch_ranks(gpus: int) -> None:
    """--gpus N > 1 without a launcher: starts this same command as N ranks on this node
    (torch.distributed.run, rendezvous on 127.0.0.1) and exits with its status."""
    import socket

    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        port = probe.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()), *sys.argv[1:]]
    sys.exit(subprocess.call(cmd))


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours")
    p.add_argument("--workload", choices=sorted(WORKLOADS) + ["batch4096", "serve", "lcp256m"], default=DEFAULT_WORKLOAD)
    p.add_argument("--batch-count", type=int, default=4096)
    p.add_argument("--plain-sample", type=int, default=64)
    p.add_argument("--serve-loads", default="50,200,800")
    p.add_argument("--serve-requests", type=int, default=200)
    p.add_argument("--serve-huge-fraction", type=float, default=0.01)
    p.add_argument("--serve-workers", type=int, default=3)
    p.add_argument("--cpu-sample-mib", type=int, default=64)
    p.add_argument("--reference-sample-mib", type=int, default=64)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--reference-gpu-steps", type=int, default=2,
                   help="steps of the reference CUDA build in the line's reference_gpu record (0: none)")
    p.add_argument("--batch-steps", type=int, default=3,
                   help="steps of the batch4096 record in the default line's `batch` (0: none)")
    p.add_argument("--no-e2e", dest="e2e", action="store_false")
    p.add_argument("--no-verify", dest="verify", action="store_false")
    args = p.parse_args()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        launch_ranks(args.gpus)  # does not return
    if int(os.environ.get("WORLD_SIZE", "1")) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but the launcher started {os.environ.get('WORLD_SIZE')} ranks",
              file=sys.stderr)
        sys.exit(2)
    if args.impl == "reference-gpu":
        world, rank, _ = rank_env()
        run_reference_gpu(args, world, rank)
        return
    if args.impl == "reference":
        # Rank 0 alone times the reference on the host cores; other ranks exit without work (and
        # without joining a process group, so nothing waits on them).
        world, rank, _ = rank_env()
        if args.workload == "lcp256m":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference computes no LCP array"}))
        elif args.workload in ("batch4096", "serve"):
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched or served "
                                  "construction (one text per call); its per-text CPU rate is the natural256m line"}))
        else:
            run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.workload == "batch4096":
            run_batch(args, world, rank, local)
        elif args.workload == "serve":
            run_serve(args, world, rank, local)
        elif args.workload == "lcp256m":
            run_lcp(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
