"""Benchmark of the cgemm3m hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form tf32x3|bf16x6|fp32]

Workload (one step = one cgemm3m call): C <- A*B, complex64, M = N = K = 4096,
column-major, op N/N, alpha = 1, beta = 0, contiguous; Re(A), Re(B) ~ N(0,1),
Im ~ N(0,1)*2^e with an integer e in [-8, 8] drawn per column; seeded
synthetic data (the reference publishes no dataset).  This is the precision
form's configuration as stated: the rounding-correction pass is ON (the
drop-in's default gate admits this shape), for the tensor-core form (value)
and for the plain FP32 drop-in (plain_fp32), both timed with the same steps
and warm-up; the same calls with the pass off are reported beside them.
Metric: c64 TFLOP/s counted as 8*M*N*K per call.  Under torchrun every rank
runs its own independent problem on its own GPU (no data-path collective; weak
scaling) and the value is the whole job's throughput over the max-over-ranks
time.

--impl reference times the reference's CPU algorithm (the oracle's
reference-order cgemm, timing build) on all host cores on a bounded column
sample of the same workload; under torchrun only rank 0 runs it.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "ascend-open-source-contributions_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "c64 TFLOP/s (8MNK) at 4096^3: tensor-core 3M vs FP32 3M, same err vs FP64"
UNIT = "TFLOP/s"
SIZE = 4096
SEED_A, SEED_B = 20261203, 20261204


def l2_note(n):
    """How the step's inputs relate to the 126 MB L2 (no flush between steps)."""
    mib = 3 * n * n * 8 / 2 ** 20
    if mib * 2 ** 20 > 126e6:
        return f"inputs exceed L2: A, B, C {mib:.0f} MiB plus packed planes; no flush needed"
    return f"inputs fit in L2 (A, B, C {mib:.1f} MiB): steps reuse them from L2, a warm-cache figure"


def workload(n):
    return f"cgemm3m {n}x{n}x{n} complex64 NN alpha=1 beta=0, precision-form data"


PASSES = {"fp32": 1, "tf32x3": 3, "bf16x6": 6, "bf16x9": 9}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="bf16x6", choices=["fp32", "tf32x3", "bf16x6", "bf16x9"])
    ap.add_argument("--size", type=int, default=SIZE)
    ap.add_argument("--tc-segment", type=int, default=0)
    ap.add_argument("--rounding", default="auto", choices=["off", "auto"],
                    help="rounding-correction pass for the headline calls (the other setting is reported beside)")
    ap.add_argument("--no-rounding-report", action="store_true", help="skip the calls with the other setting")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batching-report", action="store_true")
    ap.add_argument("--batching-only", action="store_true",
                    help="run only the batching-form measurement (one JSON object; for profiling)")
    ap.add_argument("--pf-cases", action="store_true",
                    help="run only the reference's 200 performance cases against its GPU baseline times")
    ap.add_argument("--pf-forms", default="fp32,bf16x6",
                    help="forms for --pf-cases: fp32 (the drop-in as called), fp32-norounding, cgemm, tf32x3, bf16x6")
    ap.add_argument("--pf-per-case", action="store_true")
    ap.add_argument("--shard-report", action="store_true",
                    help="also time one problem split by output columns over the ranks (always on for N > 1)")
    return ap.parse_args()


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock and clock-event reasons sampled every ~2 ms (NVML, read-only
    queries) while the timed region runs; nvidia-smi at 200 ms if NVML is
    unavailable."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, pci_bus_id=None):
        self.gpu = gpu_index
        self.pci = pci_bus_id
        self.proc = None
        self.thread = None
        self.stop_flag = threading.Event()
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.lines = []
        self.nvml = None

    def start(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            if self.pci:
                dev = pynvml.nvmlDeviceGetHandleByPciBusId(self.pci)
            else:
                dev = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.nvml = (pynvml, dev)
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _poll(self):
        nv, dev = self.nvml
        mx = nv.nvmlDeviceGetMaxClockInfo(dev, nv.NVML_CLOCK_SM)
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(dev, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(dev)
                self.samples.append((float(sm), float(mx), int(rs)))
            except Exception:
                break
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        for s_, m_, r_ in self.samples:
            sm.append(s_)
            mx.append(m_)
            for nm, bit in self.REASONS:
                if r_ & bit:
                    reasons.add(nm)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(nm)
        if self.nvml is not None:
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def pci_bus_id(props):
    try:
        return f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
    except AttributeError:
        return None


# ----------------------------------------------------------------------------- peaks

def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def sgemm_tflops(torch, dev, n=4096, reps=5):
    """cuBLAS FP32 SGEMM (TF32 off) at n^3 on this GPU, timed with CUDA events:
    the measured FP32-pipe peak (2n^3 flop per call)."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(n, n, device=dev)
        b = torch.randn(n, n, device=dev)
        for _ in range(2):
            c = a @ b
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            c = a @ b
        e1.record()
        torch.cuda.synchronize()
        del a, b, c
        return 2.0 * n ** 3 / (e0.elapsed_time(e1) / reps * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def pipe_peak(form, sm_count, sgemm=None):
    pk, src = peaks()
    if form == "fp32":
        if sgemm:
            return sgemm, "measured: cuBLAS FP32 SGEMM 4096^3 (TF32 off) on this GPU, timed in this run"
        mhz = pk.get("sm_max_mhz", 1965.0)
        return sm_count * 128 * 2 * mhz * 1e6 / 1e12, f"nominal: {sm_count} SMs x 128 FP32 lanes x 2 x {mhz:.0f} MHz"
    if form == "tf32x3":
        return pk["bf16_tflops"] / 2.0, f"{src} bf16 burst / 2 (dense TF32 = half of dense BF16)"
    return pk["bf16_tflops"], f"{src} bf16 burst"


# ----------------------------------------------------------------------------- data

def host_operands(n):
    import oracle as O

    a = O.precision_matrix(n, n, SEED_A)
    b = O.precision_matrix(n, n, SEED_B)
    return a, b


def cpu_sample(cols, n, seed_offset=0):
    """Reference-order FP32 cgemm (the oracle's timing build: same bytes as the
    checker) on op(A) (n x n) times the first `cols` columns of B:
    (seconds, flops8)."""
    import numpy as np

    import oracle as O

    a = O.precision_matrix(n, n, SEED_A)
    b = O.precision_matrix(n, n, SEED_B)[: n * cols]
    c = np.zeros(n * cols, np.complex64)
    O.cgemm_timing("N", "N", n, 2, n, 1 + 0j, a, n, b, n, 0j, c, n)  # page in A
    t0 = time.perf_counter()
    O.cgemm_timing("N", "N", n, cols, n, 1 + 0j, a, n, b, n, 0j, c, n)
    dt = time.perf_counter() - t0
    return dt, 8.0 * n * cols * n


def _cpu_worker(args):
    cols, n = args
    return cpu_sample(cols, n)


def cpu_parallel_sample(n, cols_per_worker, steps=1, warmup=0):
    """The oracle on every host core (one spawned process per core, each its
    own column block): per-step wall times and the cores used."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(cores) as pool:
        for step in range(warmup + steps):
            t0 = time.perf_counter()
            pool.map(_cpu_worker, [(cols_per_worker, n)] * cores)
            dt = time.perf_counter() - t0
            if step >= warmup:
                times.append(dt)
    return times, cores


def openblas_cgemm(n):
    """OpenBLAS cgemm (numpy/scipy's bundled build) at full n^3 on all host
    cores: (TFLOP/s at 8n^3, threads, seconds)."""
    import numpy as np

    import oracle as O
    import scipy.linalg.blas as sb

    try:
        from threadpoolctl import threadpool_info

        threads = max((x.get("num_threads", 0) for x in threadpool_info() if x.get("internal_api") == "openblas"),
                      default=0)
    except Exception:
        threads = 0
    a = np.asfortranarray(O.precision_matrix(n, n, SEED_A).reshape(n, n).T)
    b = np.asfortranarray(O.precision_matrix(n, n, SEED_B).reshape(n, n).T)
    sb.cgemm(1.0, a, b)
    t0 = time.perf_counter()
    sb.cgemm(1.0, a, b)
    dt = time.perf_counter() - t0
    return 8.0 * n ** 3 / dt / 1e12, threads or (os.cpu_count() or 1), dt


# ----------------------------------------------------------------------------- reference arm

def run_reference(args, rank):
    if rank != 0:
        return
    n = args.size
    cols_per_worker = 16  # a few hundred ms of vectorised scalar work per step
    times, cores = cpu_parallel_sample(n, cols_per_worker, args.steps, args.warmup)
    flops = 8.0 * n * n * cols_per_worker * cores
    t = statistics.median(times)
    value = flops / t / 1e12
    sample = (f"{n}x{cols_per_worker * cores}x{n} column sample of the {n}^3 workload per step "
              f"({cores} processes, one column block each)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload(args.size), "form": "reference-BLAS order FP32 (oracle port, timing build)",
                   "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- the reference's own data

# The reference's 4096^3 performance row with the rounding pass gated in
# (gpu_baseline.csv:5, op C,N, alpha = 1, beta = 0, RANDOM_NORM_5_5 fills) and
# the NPU time its perf gate implies: GPU baseline 10.8757 ms / worst ratio
# 0.41465 (README.md:54).
REF_ROW_BASELINE_MS = 10.8757
REF_ROW_NPU_BOUND_MS = 10.8757 / 0.41465


def column_shard_report(h, stream, dev, world, rank, A, B, n, form, steps, warmup):
    """One n^3 problem split by output columns over the ranks (no exchange on
    the data path: rank r multiplies all of op(A) by its own block of op(B)).
    op(A) is broadcast once from rank 0 with NCCL before the timed steps (its
    time is reported apart); the value is the whole problem's 8MNK over the
    slowest rank's device time per step.  A column block is not square, so
    the rounding-correction pass's gate leaves it off."""
    import torch
    import torch.distributed as dist
    from cg3m import dist as cdist

    C2 = torch.zeros(n * n, dtype=torch.complex64, device=dev)
    first, cols = cdist.shard_columns(n, world, rank)
    bcast_ms = None
    with torch.cuda.stream(stream):
        if world > 1:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dist.broadcast(torch.view_as_real(A), src=0)
            e1.record(stream)
            torch.cuda.synchronize()
            bcast_ms = cdist.max_over_ranks(e0.elapsed_time(e1), dev)

        def call():
            return cdist.cgemm3m_local_block(h, "N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C2, n, world, rank,
                                             form=form)

        info = None
        for _ in range(warmup):
            info = call()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = cdist.max_over_ranks(e0.elapsed_time(e1) / steps, dev)
    return {"workload": f"one cgemm3m {n}x{n}x{n} NN split by output columns over {world} rank(s), "
                        f"op(A) resident on every rank", "form": form, "value": 8.0 * n ** 3 / (ms * 1e-3) / 1e12,
            "unit": "TFLOP/s", "ms_per_step": ms, "scaling": "strong", "columns_per_rank": cols,
            "rounding": info["rounding"] if info else None, "broadcast_a_ms": bcast_ms,
            "timing": "max over ranks of CUDA-event time on each rank's stream"}


def reference_data_report(h, stream, dev, world, args, timed_fn):
    """The drop-in exactly as called (cg3mCgemm3m arithmetic, rounding pass as
    the reference gates it) on the reference's own fill -- entries uniform in
    [-5, 5] -- at op C,N, n = --size: time with the same steps and warm-up,
    per-kernel times and the rounding pass's counters."""
    import torch

    n = args.size
    gen = torch.Generator(device=dev)
    gen.manual_seed(20262029)
    with torch.cuda.stream(stream):
        A = (torch.rand(2 * n * n, generator=gen, device=dev) * 10 - 5).view(torch.complex64)
        B = (torch.rand(2 * n * n, generator=gen, device=dev) * 10 - 5).view(torch.complex64)
        C = torch.zeros(n * n, dtype=torch.complex64, device=dev)
    import cg3m

    def call(form, rounding):
        return h.cgemm3m("C", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, form=form, rounding=rounding)

    out = {"workload": f"cgemm3m {n}^3 op C,N alpha=1 beta=0, entries uniform in [-5,5] (the reference's fill)"}
    for form in ("fp32", args.form):
        ms, info, stages = timed_fn(form, "auto", args.steps, args.warmup, call=call)
        out[form] = {"value": world * 8.0 * n ** 3 / (ms * 1e-3) / 1e12, "ms_per_step": ms,
                     "stage_names": cg3m.stage_names(info), "stage_ms": stages, "rounding_stats": h.rounding_stats()}
    if n == 4096:
        out["reference_gpu_baseline_ms"] = REF_ROW_BASELINE_MS
        out["reference_npu_bound_ms"] = REF_ROW_NPU_BOUND_MS
    del A, B, C
    torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------------------- batching form

def batching_report(h, stream, dev, world, args):
    """512 heterogeneous problems (m, n, k log-uniform in [16, 1024], 9 op
    pairs, random alpha/beta): one graph-replayed persistent launch of the
    autotuned plan vs 512 separate cg3mCgemm3m calls; metric sum(8mnk)/t."""
    import torch

    from cg3m.workloads import batch_flops, batch_problems

    probs = batch_problems(dev, count=512)
    fl = batch_flops(probs)
    steps = max(5, min(args.steps, 20))

    def timeit(fn, n_steps, warm):
        with torch.cuda.stream(stream):
            for _ in range(warm):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(n_steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n_steps

    with torch.cuda.stream(stream):
        t0 = time.perf_counter()
        plan = h.batch_plan(probs, tune=True)
        torch.cuda.synchronize()
        plan_s = time.perf_counter() - t0
    desc = plan.describe()
    batch_ms = timeit(lambda: plan.execute(use_graph=True), steps, 3)
    direct_ms = timeit(lambda: plan.execute(use_graph=False), steps, 1)

    def separate():
        for (ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc) in probs:
            st = h.cgemm3m(ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc, raw=True)
            if st != 0:
                raise RuntimeError(f"cg3mCgemm3m status {st}")

    sep_ms = timeit(separate, max(2, steps // 4), 1)
    plan.close()
    tiles = {}
    for tm, tn, kp in desc:
        key = f"{tm}x{tn}/k{kp}"
        tiles[key] = tiles.get(key, 0) + 1
    del probs
    torch.cuda.empty_cache()
    return {"workload": "512 cgemm3m, m,n,k log-uniform [16,1024], 9 op pairs, |alpha|,|beta|<=1, plain FP32 3M",
            "flops8": fl, "value": world * fl / (batch_ms * 1e-3) / 1e12, "unit": UNIT, "ms": batch_ms,
            "direct_launch_ms": direct_ms, "separate_calls": {"value": world * fl / (sep_ms * 1e-3) / 1e12,
                                                              "ms": sep_ms, "calls": 512},
            "speedup_vs_separate": sep_ms / batch_ms, "plan_create_s": plan_s, "plan_tiles": tiles}


# ----------------------------------------------------------------------------- reference performance cases

def pf_cases_report(h, stream, dev, forms=("fp32", "bf16x6"), per_case=False):
    """The reference's 200 performance cases (tests/golden/pf_gpu_baseline.json:
    shapes, ops and leading dimensions of its TC_PF rows, alpha = 1, beta = 0,
    entries uniform in [-5, 5] as RANDOM_NORM_5_5), 5 warm-up calls then 10
    timed calls per case, two ways: back to back with CUDA events (host launch
    costs included) and as a replayed CUDA graph of the 10 calls (device time,
    closer to the reference's sum of kernel times).  Per form: the ratio of the
    reference's GPU baseline time to this library's time per case (> 1:
    faster), its minimum, median and mean, and the summed times.  `fp32` is the
    drop-in exactly as called (rounding pass where the reference gates it)."""
    import torch

    with open(os.path.join(ROOT, "tests", "golden", "pf_gpu_baseline.json")) as f:
        cases = json.load(f)["cases"]
    gen = torch.Generator(device=dev)
    gen.manual_seed(20262029)
    out = {}
    for form in forms:
        rows = []
        for cs in cases:
            ta, tb, m, n, k = cs["transa"], cs["transb"], cs["m"], cs["n"], cs["k"]
            a_cols = k if ta == "N" else m
            b_cols = n if tb == "N" else k
            with torch.cuda.stream(stream):
                A = (torch.rand(2 * cs["lda"] * a_cols, generator=gen, device=dev) * 10 - 5).view(torch.complex64)
                B = (torch.rand(2 * cs["ldb"] * b_cols, generator=gen, device=dev) * 10 - 5).view(torch.complex64)
                C = torch.zeros(cs["ldc"] * n, dtype=torch.complex64, device=dev)

                def call():
                    if form == "fp32":
                        st = h.cgemm3m(ta, tb, m, n, k, 1.0, A, cs["lda"], B, cs["ldb"], 0.0, C, cs["ldc"], raw=True)
                        if st != 0:
                            raise RuntimeError(f"cg3mCgemm3m status {st}")
                    elif form == "fp32-norounding":
                        h.cgemm3m(ta, tb, m, n, k, 1.0, A, cs["lda"], B, cs["ldb"], 0.0, C, cs["ldc"], form="fp32",
                                  rounding="off")
                    elif form == "cgemm":
                        st = h.cgemm(ta, tb, m, n, k, 1.0, A, cs["lda"], B, cs["ldb"], 0.0, C, cs["ldc"])
                        if st != 0:
                            raise RuntimeError(f"cg3mCgemm status {st}")
                    else:
                        h.cgemm3m(ta, tb, m, n, k, 1.0, A, cs["lda"], B, cs["ldb"], 0.0, C, cs["ldc"], form=form,
                                  rounding="off")

                for _ in range(5):
                    call()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(10):
                    call()
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / 10
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=stream):
                    for _ in range(10):
                        call()
                g.replay()
                torch.cuda.synchronize()
                e0.record(stream)
                g.replay()
                e1.record(stream)
                torch.cuda.synchronize()
                gms = e0.elapsed_time(e1) / 10
                del g
            rows.append((cs["gpu_ms"] / ms, cs["gpu_ms"] / gms, ms, gms, cs))
            del A, B, C
        def summary(idx, tidx):
            r = sorted(x[idx] for x in rows)
            worst = min(rows, key=lambda x: x[idx])
            return {"ratio_min": r[0], "ratio_median": r[len(r) // 2], "ratio_mean": sum(r) / len(r),
                    "ms_total": sum(x[tidx] for x in rows),
                    "worst": {"ratio": worst[idx], "id": worst[4]["id"],
                              "shape": f"{worst[4]['transa']}{worst[4]['transb']} "
                                       f"{worst[4]['m']}x{worst[4]['n']}x{worst[4]['k']}",
                              "ms": worst[tidx], "baseline_ms": worst[4]["gpu_ms"]}}
        out[form] = {"cases": len(rows), "baseline_ms_total": sum(x[4]["gpu_ms"] for x in rows),
                     "back_to_back": summary(0, 2), "graph_replay": summary(1, 3)}
        if per_case:
            out[form]["per_case"] = [[x[4]["id"], round(x[2], 4), round(x[3], 4)] for x in rows]
    torch.cuda.empty_cache()
    return {"what": "reference GPU baseline time / B200 time per case (its perf gate divides the same baseline by "
                    "its NPU time: min 0.415, mean 0.635)", **out}


# ----------------------------------------------------------------------------- our arm

def kernel_roofline(name, ms, n, form, sm_count, sgemm, stats, mhz):
    """Roofline entry of one kernel of the 4096^3 call from its mean in-loop
    duration: algorithmic work per launch over the time, against the pipe or
    memory peak that bounds it."""
    pk, src = peaks()
    p = PASSES[form]
    if name in ("gemm", "gemm_path", "gemm_form_tiles"):
        # the tensor-core forms' path GEMM is one pass of the four real products
        # (8 n^3 flop) over the leading split planes of re and im; their form
        # products then cover only the tiles the exact recompute does not take
        cover = 1.0
        per = 6.0
        if name == "gemm_path" and form != "fp32":
            p, per = 1, 8.0
        if name == "gemm_form_tiles":
            cover = 1.0 - (float(stats.get("exact_positions", 0)) / float(n * n) if stats else 0.0)
        work = per * n ** 3 * p * cover
        peak, peak_src = pipe_peak(form, sm_count, sgemm)
        return {"bound": "tensor" if form != "fp32" else "fp32-pipe",
                "achieved": work / (ms * 1e-3) / 1e12 if ms > 0 else 0.0,
                "peak": peak, "unit": "TFLOP/s", "work_per_launch": work,
                "work_model": f"{per:.0f}*n^3 real flop x {p} pass(es) x {cover:.3f} of the outputs",
                "peak_source": peak_src}
    if name == "exact_tiles":
        positions = float(stats.get("exact_positions", 0)) if stats else 0.0
        work = 2.0 * 14 * 4 * positions * n  # int8 ops: 14 moduli x 4 real products per output and term
        peak = 2.0 * pk["bf16_tflops"]
        return {"bound": "tensor", "achieved": work / (ms * 1e-3) / 1e12, "peak": peak, "unit": "Top/s",
                "work_per_launch": work,
                "work_model": "2 x 14 moduli x 4 real products x n int8 ops per output position of the tiles run",
                "peak_source": f"{src} bf16 burst x 2 (dense int8 is twice the dense bf16 rate)"}
    if name.startswith("recompute_fp64") or name.startswith("fallback"):
        key = "fallback_outputs" if name.startswith("fallback") else "sparse_outputs"
        outs = float(stats[key]) if stats and stats.get(key) is not None else float(n * n)
        work = 8.0 * outs * n
        peak = sm_count * 64 * 2 * mhz * 1e6 / 1e12
        return {"bound": "fp64-pipe", "achieved": work / (ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                "work_per_launch": work,
                "work_model": f"8 flop (4 DFMA) x n per flagged output it recomputes ({key})",
                "peak_source": f"nominal: {sm_count} SMs x 64 FP64 lanes x 2 x {mhz:.0f} MHz"}
    if name.startswith("replay"):
        key = "dense_outputs" if name.endswith("tiles") else "sparse_outputs"
        outs = float(stats[key]) if stats and stats.get(key) is not None else float(n * n)
        work = 20.0 * outs * n
        peak = sm_count * 128 * mhz * 1e6 / 1e12
        return {"bound": "fp32-pipe", "achieved": work / (ms * 1e-3) / 1e12, "peak": peak, "unit": "Top/s",
                "work_per_launch": work,
                "work_model": f"2 passes x 10 FP32 ops (operand sums, 3 products, term, accumulate) x n per flagged "
                              f"output it recomputes ({key})",
                "peak_source": f"nominal: {sm_count} SMs x 128 FP32 lanes x {mhz:.0f} MHz (one op per lane)"}
    return {"bound": "hbm", "achieved": None, "peak": pk.get("hbm_gbs"), "unit": "GB/s", "work_per_launch": None,
            "work_model": "not modelled", "peak_source": f"{src} copy bandwidth"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    # CPU legs first: the spawned processes must start before CUDA is up.
    cpu = None
    cpu_openblas = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cols = 16
        times, cores = cpu_parallel_sample(args.size, cols, steps=1)
        fl = 8.0 * args.size * args.size * cols * cores
        cpu = {"value": fl / times[0] / 1e12, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.size}x{cols * cores}x{args.size} column sample of the workload, reference-BLAS "
                         f"order FP32 (oracle timing build, bit-identical to the checker), {cores} processes"}
        try:
            tf, threads, dt = openblas_cgemm(args.size)
            cpu_openblas = {"value": tf, "unit": UNIT, "threads": threads, "seconds": dt,
                            "what": f"OpenBLAS cgemm (scipy's bundled build) at full {args.size}^3 on this host"}
        except Exception as e:  # scipy missing on the host: report why
            cpu_openblas = {"unavailable": str(e)[:200]}

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    import cg3m

    if args.pf_cases:
        stream = torch.cuda.Stream(device=dev)
        h = cg3m.Handle(stream=stream.cuda_stream)
        rep = pf_cases_report(h, stream, dev, forms=tuple(args.pf_forms.split(",")), per_case=args.pf_per_case)
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"pf_cases": rep}), flush=True)
        return

    if args.batching_only:
        stream = torch.cuda.Stream(device=dev)
        h = cg3m.Handle(stream=stream.cuda_stream)
        rep = batching_report(h, stream, dev, world, args)
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"batching_form": rep}), flush=True)
        return

    n = args.size
    a_host, b_host = host_operands(n)
    A = torch.from_numpy(a_host).to(dev)
    B = torch.from_numpy(b_host).to(dev)
    C = torch.zeros(n * n, dtype=torch.complex64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    h = cg3m.Handle(stream=stream.cuda_stream)
    props = torch.cuda.get_device_properties(dev)
    sm_count = props.multi_processor_count

    def call(form, rounding):
        return h.cgemm3m("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, form=form, tc_segment=args.tc_segment,
                         rounding=rounding)

    def timed(form, rounding, steps, warmup, call=call):
        """Mean ms per call over `steps` calls after `warmup`, and the mean
        duration of each of the call's kernels from events the library records
        between its launches inside the same timed loop."""
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                info = call(form, rounding)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            nk = info["kernels"]
            evsets = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * nk)] for _ in range(steps)]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(steps):
                h.set_stage_events(evsets[i])
                info = call(form, rounding)
            e1.record(stream)
            h.set_stage_events([])
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        per = [sum(ev[2 * j].elapsed_time(ev[2 * j + 1]) for ev in evsets) / steps for j in range(nk)]
        if world > 1:
            t = torch.tensor([ms] + per, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms, per = float(t[0].item()), [float(x) for x in t[1:].tolist()]
        return ms, info, per

    flops8 = 8.0 * n ** 3
    other = "off" if args.rounding == "auto" else "auto"

    sampler = ClockSampler(local, pci_bus_id(props))
    sampler.start()
    ms, info, stages = timed(args.form, args.rounding, args.steps, args.warmup)
    stats = h.rounding_stats() if info["rounding"] else None
    if args.form != "fp32":
        pms, pinfo, pstages = timed("fp32", args.rounding, args.steps, args.warmup)
        pstats = h.rounding_stats() if pinfo["rounding"] else None
    clocks = sampler.stop()
    value = world * flops8 / (ms * 1e-3) / 1e12
    names = cg3m.stage_names(info)
    mhz = (clocks or {}).get("sm_mhz") or peaks()[0].get("sm_max_mhz", 1965.0)

    sgemm = sgemm_tflops(torch, dev)
    dom = max(range(len(stages)), key=lambda i: stages[i])
    roofline = kernel_roofline(names[dom], stages[dom], n, args.form, sm_count, sgemm, stats, mhz)
    roofline.update({"kernel": names[dom], "kernel_ms": stages[dom], "share_of_step": stages[dom] / ms,
                     "traffic": None})
    roofline["frac"] = (roofline["achieved"] / roofline["peak"]) if roofline.get("achieved") else None
    traffic_file = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            roofline["traffic"] = json.load(f).get(f"{names[dom]}_{args.form}_{n}")

    # End to end through the public host-buffer entry point (cg3mCgemm3mHost):
    # A and B uploaded from page-locked host memory and C read back inside
    # every step (with the rounding pass the call runs as one panel).
    a_pin = torch.from_numpy(a_host).pin_memory()
    b_pin = torch.from_numpy(b_host).pin_memory()
    c_pin = torch.empty(n * n, dtype=torch.complex64).pin_memory()

    def host_call():
        return h.cgemm3m_host("N", "N", n, n, n, 1.0, a_pin, n, b_pin, n, 0.0, c_pin, n, form=args.form,
                              tc_segment=args.tc_segment, rounding=args.rounding)

    with torch.cuda.stream(stream):
        for it in range(args.warmup + args.steps):
            if it == args.warmup:
                torch.cuda.synchronize()
                if world > 1:
                    dist.barrier()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            host_info = host_call()
        e1.record(stream)
        torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": world * flops8 / (e2e_ms * 1e-3) / 1e12, "unit": UNIT, "h2d_bytes_per_step": 2 * n * n * 8,
           "d2h_bytes_per_step": n * n * 8, "ms_per_step": e2e_ms,
           "api": f"cg3mCgemm3mHost (page-locked host A, B, C; rounding {args.rounding})",
           "kernels_per_step": host_info["kernels"]}

    # accuracy vs FP64 (device reference) for every timed call
    out64 = torch.empty(n * n, dtype=torch.complex128, device=dev)
    errors = {}
    with torch.cuda.stream(stream):
        h.zgemm_reference("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, out64)
        for form in sorted({args.form, "fp32"}):
            call(form, args.rounding)
            errors[form] = h.error_report(n, n, C, n, out64)
    plain = None
    if args.form != "fp32":
        plain = {"value": world * flops8 / (pms * 1e-3) / 1e12, "ms_per_step": pms, "rounding": args.rounding,
                 "kernels": pinfo["kernels"], "stage_names": cg3m.stage_names(pinfo), "stage_ms": pstages,
                 "rounding_stats": pstats, "errors_vs_fp64": errors["fp32"],
                 "what": "the plain FP32 drop-in (cg3mCgemm3m arithmetic) on the same call, same steps and warm-up"}
    # the same calls with the pass set the other way (same steps and warm-up)
    other_report = None
    if not args.no_rounding_report:
        other_report = {"rounding": other}
        for form in sorted({args.form, "fp32"}):
            oms, oinfo, ost = timed(form, other, args.steps, args.warmup)
            with torch.cuda.stream(stream):
                call(form, other)
                err = h.error_report(n, n, C, n, out64)
            other_report[form] = {"value": world * flops8 / (oms * 1e-3) / 1e12, "ms_per_step": oms,
                                  "kernels": oinfo["kernels"], "stage_names": cg3m.stage_names(oinfo),
                                  "stage_ms": ost, "errors_vs_fp64": err}
        if args.form != "fp32":
            other_report["tc_over_plain"] = other_report[args.form]["value"] / other_report["fp32"]["value"]
            other_report["fp32"]["sgemm_tflops_measured"] = sgemm
            fp32_names = other_report["fp32"]["stage_names"]
            if "gemm" in fp32_names:
                gms = other_report["fp32"]["stage_ms"][fp32_names.index("gemm")]
                other_report["fp32"]["gemm_fp32_tflops"] = 6.0 * n ** 3 / (gms * 1e-3) / 1e12
                other_report["fp32"]["gemm_frac_of_sgemm"] = other_report["fp32"]["gemm_fp32_tflops"] / sgemm
    del out64
    reference_data = None if args.no_rounding_report else reference_data_report(h, stream, dev, world, args, timed)
    batching = None if args.no_batching_report else batching_report(h, stream, dev, world, args)
    shard = column_shard_report(h, stream, dev, world, rank, A, B, n, args.form, args.steps, args.warmup) \
        if (world > 1 or args.shard_report) else None
    status = h.device_status()

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.form == "fp32" else args.form, "data": "synthetic",
        "config": {"workload": workload(n), "form": args.form, "rounding": args.rounding, "m": n, "n": n, "k": n,
                   "transa": "N", "transb": "N", "alpha": [1, 0], "beta": [0, 0],
                   "parallelism": f"replica x{world} (independent problems)", "l2": l2_note(n),
                   "plan": {k_: info[k_] for k_ in ("tile_m", "tile_n", "k_partitions", "k_span", "rounding",
                                                    "kernels", "workspace_bytes")}},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "cpu_openblas": cpu_openblas,
        "e2e": e2e,
        "gpu_launches": args.steps * info["kernels"],
        "clocks": clocks,
        "stage_names": names,
        "stage_ms": stages,
        "rounding_stats": stats,
        "errors_vs_fp64": errors,
        "plain_fp32": plain,
        "tc_over_plain": (value / plain["value"]) if plain else None,
        "rounding_" + other: other_report,
        "reference_data": reference_data,
        "batching_form": batching,
        "column_shard": shard,
        "device_status": status,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
