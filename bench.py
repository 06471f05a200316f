#!/usr/bin/env python
"""Benchmark of the NMF iteration loop on B200.

A step is one NMF iteration (H update + W update) over the whole V.  The
default is the plain method in f64 (the precision the reference computes
in), lee on the atlas shape 20000 x 200000 rank 20; beside it, as extra keys,
the precision forms (split-bf16 on the tensor cores, f32 on the CUDA cores)
with their relative objective and max|dW| against the f64 run, and brunet
(f64 and split-bf16) at the same shape.

  value    iterations/s with V, W, H already in HBM (nmfcu_run_device),
           K timed iterations in one call, CUDA events on the launch stream,
           max over ranks.  Whole job: N replicas x K iterations / time.
  e2e      iterations/s through the host-pointer C ABI (nmfcu_run, the call
           behind nmf_rs.nmf): host->device copy of V, W0, H0, the K
           iterations and the device->host copy of W, H, all timed.
  roofline achieved HBM GB/s of the dominant V-streaming kernel class,
           algorithmic bytes (one read of V per launch) / average launch time
           from the library's CUDA-event hooks, against MEASURED_PEAKS.json;
           for brunet in f64 also the FP64 TFLOP/s of the ratio pass against
           a cuBLAS f64 GEMM measured in the same run.
  cpu_baseline  the CPU restatement of the reference loop (oracle/, the
           Rust reference cannot be built here; -march=native, OpenMP on all
           host cores) on a column slice of the same V: the difference of a
           3- and a 1-iteration call (so the per-run set-up is not counted as
           iteration time), extrapolated linearly in the column count.

--impl reference times that CPU restatement as the reference arm.

--form serve measures the serving form: a stream of Poisson-arriving
requests (shapes log-uniform 500x1000 .. 5000x50000, rank U{5..30}, methods
lee 40% / brunet 30% / hals 20% / dnmf 10%, 25..200 iterations, FP32 form)
through nmfcu_server_*, reporting p50/p99 latency and aggregate iters/s.

--form nndsvd measures the NNDSVD start (nmf_rs.nndsvd_init, the reference's
nndsvd_init over scikit-learn's randomized_svd) at the atlas shape: one step
= one rank-20 NNDSVD of V with its 16 FP64 passes over V on the device
(nmfcu_v_product_device) and the small factorizations on the device;
cpu_baseline = scikit-learn's randomized_svd (the reference's own call) on a
column slice of the same V.

--form shard measures one solve split by columns of V over the N ranks
(nmf_rs.shard: each rank holds its column block, one NCCL all-reduce of the
W contraction and Grams per iteration): strong scaling, value = iterations
of the whole problem per second.

--form consensus measures the batching form instead: a consensus sweep of
64 brunet restarts x ranks 2..10 (576 solves x 200 iterations) on a
2000 x 5000 V, one step = one whole sweep through nmfcu_run_batch_device
plus the nine consensus matrices and their cophenetic correlation and
dispersion (nmfcu_consensus_stats_device), against the same solves run one
by one through the single-solve engine.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (str(ROOT), str(ROOT / "rust-nmf_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (n, p, k, alpha, rank, default iterations)
    "atlas": (20000, 200000, 20, 0.2, 20, 25),
    # a 20000 x 20000 column slice of the atlas shape (larger than L2; small
    # enough for profiler captures)
    "atlas-slice": (20000, 20000, 20, 0.2, 20, 25),
    "pbmc8k": (2000, 7750, 10, 0.2, 10, 100),
    "pbmc-subset": (1500, 3000, 8, 0.3, 8, 100),
}
ATLAS_WORKLOADS = ("atlas", "atlas-slice")  # the precision form's shapes


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed iterations")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="atlas")
    ap.add_argument("--method", choices=["lee", "brunet", "hals", "dnmf"], default="lee")
    ap.add_argument("--precision", choices=["fp32", "bf16x3", "fp64"], default=None,
                    help="default: fp64 (the reference's precision); fp32 for the consensus "
                         "form (its batched FP32 form)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--form", choices=["iterate", "consensus", "serve", "nndsvd", "shard",
                                       "sparse"],
                    default="iterate")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the stream")
    ap.add_argument("--slots", type=int, default=8, help="serve: server slots")
    ap.add_argument("--load", type=float, default=0.8,
                    help="serve: Poisson arrival rate as a fraction of the measured capacity")
    ap.add_argument("--runs", type=int, default=64, help="consensus restarts per rank")
    ap.add_argument("--seq-runs", type=int, default=None,
                    help="consensus: restarts per rank timed one by one (default: all; 0: skip)")
    ap.add_argument("--iters", type=int, default=200, help="consensus: iterations per solve")
    ap.add_argument("--density", type=float, default=0.1,
                    help="sparse: fraction of V's entries stored")
    args = ap.parse_args()
    if args.precision is None:
        args.precision = "fp32" if args.form == "consensus" else "fp64"
    return args


# ---------------------------------------------------------------------------
# Distributed plumbing (replicas: no data-path collective)
# ---------------------------------------------------------------------------

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# Synthetic V on the device (same generator as nmf_rs.synthetic, torch RNG)
# ---------------------------------------------------------------------------

def device_workload(n, p, k, alpha, rank, seed, device):
    from nmf_rs import synthetic

    return synthetic.device_workload(n, p, k, alpha, rank, seed, device)


def objective_torch(V64, p, W, H, method):
    """f64 objective of (W, H) on the device, column chunks (a check, not
    the product path)."""
    import torch

    total = torch.zeros((), dtype=torch.float64, device=V64.device)
    for c0 in range(0, p, 16384):
        c1 = min(p, c0 + 16384)
        v = V64[:, c0:c1]
        wh = W @ H[:, c0:c1]
        if method == "brunet":
            pos = v > 0
            good = pos & (wh > 0)
            term = torch.where(good, v * torch.log(torch.where(good, v / wh, 1.0)) - v + wh,
                               torch.zeros_like(v))
            term = torch.where(pos, term, wh)
            total += term.sum()
        else:
            total += ((v - wh) ** 2).sum()
    return float(total) * (1.0 if method == "brunet" else 0.5)


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.file is None:
            return {}
        self.file.flush()
        rows = [ln.split(",") for ln in Path(self.file.name).read_text().splitlines() if ln.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, r[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (CPU restatement of the reference loop)
# ---------------------------------------------------------------------------

def _oracle_native():
    """The oracle built -march=native on this host (same bits as the generic
    build; see oracle/Makefile)."""
    import oracle

    oracle.use_native()
    return oracle


def oracle_iteration_seconds(method, V, W0, H0, iters, threads):
    """Seconds per iteration of the CPU restatement on V: one call of 1 + iters
    iterations minus one call of 1 iteration, so the per-run set-up that the
    reference also pays once per run (its V^T copy, lib.rs:1606, and the
    buffers) is not counted as iteration time."""
    oracle = _oracle_native()
    t0 = time.perf_counter()
    oracle.nmf_method(method, V, W0, H0, 1, num_threads=threads)
    t1 = time.perf_counter()
    oracle.nmf_method(method, V, W0, H0, 1 + iters, num_threads=threads)
    t2 = time.perf_counter()
    return max((t2 - t1) - (t1 - t0), 1e-9) / iters, (t1 - t0), (t2 - t1)


def pick_slice(V_host_fn, p, method, seconds, threads):
    """Column count whose single iteration takes about `seconds` / 4."""
    oracle = _oracle_native()
    p_s = min(p, 512)
    while True:
        V_s, W0, H0 = V_host_fn(p_s)
        t0 = time.perf_counter()
        oracle.nmf_method(method, V_s, W0, H0, 1, num_threads=threads)
        dt = time.perf_counter() - t0
        if dt > seconds / 16 or p_s >= p:
            break
        p_s = int(min(p, max(p_s * 2, p_s * (seconds / 4) / max(dt, 1e-3))))
    target = int(min(p, max(64, p_s * (seconds / 4) / max(dt, 1e-3))))
    return (target + 15) // 16 * 16 if target < p else p


def cpu_baseline(V_host_fn, n, p, rank, method, seconds, seed=0):
    """The CPU restatement of the reference loop (oracle/, -march=native,
    OpenMP on all host cores) on a column slice of the workload: 2 timed
    iterations beyond a 1-iteration call, extrapolated linearly in columns
    (every part of an iteration is linear in p)."""
    threads = os.cpu_count() or 1
    p_s = pick_slice(V_host_fn, p, method, seconds, threads)
    V_s, W0, H0 = V_host_fn(p_s)
    per_iter, t_one, t_three = oracle_iteration_seconds(method, V_s, W0, H0, 2, threads)
    t_full = per_iter * p / p_s
    return {
        "value": 1.0 / t_full,
        "unit": "iters/s",
        "cores": threads,
        "kind": "port",
        "sample": (f"{method} on the CPU restatement (oracle/, -march=native, OpenMP, "
                   f"{threads} threads) on all {n} rows x {p_s} of {p} columns: a 1-iteration "
                   f"call took {t_one:.2f} s and a 3-iteration call {t_three:.2f} s; their "
                   f"difference / 2 = {per_iter:.3f} s an iteration, extrapolated linearly "
                   f"in columns to the full V"),
    }


def host_slice_fn(V64, p_full, rank, seed=0):
    """Returns f(p_s) -> (V slice, W0, H0) on the host for the CPU baseline."""
    def f(p_s):
        v = V64[:, :p_s].double().cpu().numpy()
        v = np.ascontiguousarray(v)
        gen = np.random.default_rng(seed)
        top = float(v.max()) if v.size else 1.0
        W0 = gen.uniform(0, top, (v.shape[0], rank))
        H0 = gen.uniform(0, top, (rank, p_s))
        return v, W0, H0
    return f


# DRAM bytes (read + write) per V element of one launch of each streaming
# pass, from an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum)
# of the 20000 x 20000 slice (V larger than L2), rank 20.  Traffic grows with
# the V elements a launch streams, so a launch over n x p moves this times
# n * p bytes.
PASS_DRAM_BYTES_PER_ELEMENT = {
    ("hpass", "fp32"): (1634701568 + 35060736) / 4e8,
    ("wpass", "fp32"): (1637906432 + 33353984) / 4e8,
    # f64: the FP64 tensor-core passes (hpass_dmma / wpass_dmma)
    ("hpass", "fp64"): (3233123072 + 32075008) / 4e8,
    ("wpass", "fp64"): (3237119744 + 31909376) / 4e8,
    # split-bf16 form: the tensor-core passes (H pass streams the split V^T)
    ("hpass", "bf16x3"): (1614820000 + 7405568) / 4e8,
    ("wpass", "bf16x3"): (1614029000 + 9831936) / 4e8,
}


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        d = json.loads(path.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# Reference arm
# ---------------------------------------------------------------------------

def iterate_metric(method, workload):
    """The metric string both arms of the iterate form print."""
    n, p, _, _, r, _ = WORKLOADS[workload]
    return f"{method} iterations/s, {workload} {n}x{p} rank {r}"


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the reference loop on the
    host cores.  A step is one iteration over a column slice of the workload
    (the full f64 V would need ~96 GB of host memory and minutes a step);
    exactly `steps` slice iterations are timed after `warmup` untimed ones,
    in one call (so the per-run V^T copy and buffers are paid once, as in
    the reference), and `value` is full-V iterations per second, the slice
    time scaled by p / slice columns."""
    if rank != 0:
        return
    n, p, k, alpha, r, iters = WORKLOADS[args.workload]
    steps = args.steps or iters
    warm = max(1, args.warmup)
    threads = os.cpu_count() or 1
    from nmf_rs import synthetic

    def V_host_fn(p_s):
        V = synthetic.counts_matrix(n, p_s, k, alpha, seed=0)
        W0, H0 = synthetic.starting_point(V, r, seed=0)
        return V, W0, H0

    # Slice sized so one iteration takes about cpu_seconds / 8 (the whole
    # arm, warm-up and calibration included, stays within a few minutes).
    budget = args.cpu_seconds * max(1.0, 20.0 / max(steps, 1))
    p_s = pick_slice(V_host_fn, p, args.method, budget / 2, threads)
    V_s, W0, H0 = V_host_fn(p_s)
    oracle = _oracle_native()
    t0 = time.perf_counter()
    oracle.nmf_method(args.method, V_s, W0, H0, warm, num_threads=threads)
    t1 = time.perf_counter()
    oracle.nmf_method(args.method, V_s, W0, H0, warm + steps, num_threads=threads)
    t2 = time.perf_counter()
    timed_s = max((t2 - t1) - (t1 - t0), 1e-9)
    ms_step = 1000.0 * timed_s / steps
    value = steps * p_s / p / timed_s
    sample = (f"{steps} {args.method} iterations of the CPU restatement (oracle/, -march=native, "
              f"OpenMP, {threads} threads) on all {n} rows x {p_s} of {p} columns: "
              f"{timed_s:.2f} s beyond a {warm}-iteration call ({t1 - t0:.2f} s); "
              f"value = iterations of the full V per second, scaled by {p}/{p_s} columns")
    line = {
        "impl": "reference",
        "metric": iterate_metric(args.method, args.workload),
        "value": value,
        "unit": "iters/s",
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": warm,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": f"synthetic (seeded generator), {n}x{p_s} column slice of the workload",
        "config": {"workload": args.workload, "n": n, "p": p, "rank": r,
                   "method": args.method, "precision": "fp64", "slice_columns": p_s,
                   "step": f"one iteration over the {n}x{p_s} slice"},
        "cpu_baseline": {"value": value, "unit": "iters/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": ("the Rust reference cannot be built in this image (no cargo/rustc); "
                 "this arm times the C restatement of its loop (oracle/) on host cores; "
                 "ms_per_step is one slice iteration"),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------

def measure_fp64_gemm_tflops(dev):
    """FP64 throughput of cuBLAS (torch.matmul, 8192^3 f64, best of 5, CUDA
    events): the measured FP64 denominator of the ratio passes' FLOP
    roofline."""
    import torch

    a = torch.rand((8192, 8192), dtype=torch.float64, device=dev)
    b = torch.rand((8192, 8192), dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * 8192 ** 3 / (best / 1000.0) / 1e12


def run_ours(args, world, rank, local):
    """The iterate form.  The headline is the precision the reference
    computes in (f64, the plain method); the mixed-precision forms and, at the
    atlas shape, brunet are measured beside it as extra keys."""
    import torch

    from nmf_rs import _native

    n, p, k, alpha, r, iters = WORKLOADS[args.workload]
    steps = args.steps or iters
    warm = max(3, args.warmup)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    V64, ld64, V32, ld32, W0, H0 = device_workload(n, p, k, alpha, r, 1234 + rank, dev)
    atlas = args.workload in ATLAS_WORKLOADS
    if atlas:
        # The atlas shape starts from an NNDSVD start computed in f64 (on the
        # device, outside the timed region); the small workloads from the
        # seeded uniform start above.
        from nmf_rs import nndsvd
        W0, H0 = nndsvd.nndsvd_device(V64[:, :p], r, fill="mean", seed=0)
        W0, H0 = W0.contiguous(), H0.contiguous()
    torch.cuda.synchronize()
    ctx = _native.Context(local)
    stream = torch.cuda.current_stream(dev)
    KCLASSES = (("hstep", _native.KCLASS_HSTEP), ("wstep", _native.KCLASS_WSTEP),
                ("objective", _native.KCLASS_OBJECTIVE), ("other", _native.KCLASS_OTHER),
                ("hstep_refine", _native.KCLASS_HSTEP_REFINE),
                ("wstep_refine", _native.KCLASS_WSTEP_REFINE))

    def options(method, precision, iters_, refine=2):
        o = _native.default_options()
        o.method = _native.parse_method(method)
        o.stop = 0
        o.precision = _native.PRECISIONS[precision]
        o.max_iter = iters_
        o.refine_iters = refine
        o.device = local
        return o

    def device_run(method, precision, iters_, W, H):
        o = options(method, precision, iters_)
        if precision == "fp32":
            return ctx.run(o, n, p, r, V32.data_ptr(), _native.F32, ld32, W.data_ptr(),
                           H.data_ptr(), v64_ptr=V64.data_ptr(), ldv64=ld64,
                           stream=stream.cuda_stream)
        return ctx.run(o, n, p, r, V64.data_ptr(), _native.F64, ld64, W.data_ptr(),
                       H.data_ptr(), stream=stream.cuda_stream)

    def timed(method, precision):
        W = W0.clone()
        H = H0.clone()
        device_run(method, precision, warm, W, H)  # warm-up iterations (untimed)
        W = W0.clone()
        H = H0.clone()
        torch.cuda.synchronize()
        ctx.reset_timing()
        ctx.set_timing(True)
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        device_run(method, precision, steps, W, H)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1)
        launches = ctx.launch_count()
        classes = {name: ctx.kernel_time(kc) for name, kc in KCLASSES}
        ctx.set_timing(False)
        return ms, launches, classes, W, H

    def rate(ms):
        return world * steps / (max_over_ranks(ms, world) / 1000.0)

    peak, peak_kind = measured_peaks()
    fp64_tflops = measure_fp64_gemm_tflops(dev) if args.method == "brunet" or atlas else None

    def kernel_name(method, precision, dom):
        hw = "H step" if dom == "hstep" else "W step"
        ratio = method == "brunet"
        if precision == "bf16x3":
            return (("tcr_pass" if ratio else "tc_pass") + ("<H>" if dom == "hstep" else "<W>") +
                    (" (KL ratio pass, tensor cores, f32 V)" if ratio else
                     " (split-bf16 pass, tensor cores)"))
        if precision == "fp64":
            return (("h" if dom == "hstep" else "w") + "pass_dmma" + ("_ratio" if ratio else "") +
                    f" ({hw}, FP64 tensor cores)")
        return ("hpass" if dom == "hstep" else "wpass") + f" ({hw}, f32 CUDA cores)"

    def roofline(method, precision, classes):
        """Achieved HBM GB/s (and, for the KL ratio passes, FP64 TFLOP/s) of
        the dominant V-streaming pass: algorithmic bytes (one read of V) per
        launch / its average launch time (library CUDA events)."""
        s_main = 8 if precision == "fp64" else 4  # f64 V; f32 V or bf16 hi + lo
        main_iters = steps if precision == "fp64" else max(0, steps - 2)
        dom = max(("hstep", "wstep"), key=lambda name: classes[name][1])
        nl, tot_ms = classes[dom]
        bytes_per_launch = n * p * s_main
        avg_ms = tot_ms / max(nl, 1)
        achieved = bytes_per_launch / (avg_ms / 1000.0) / 1e9
        kname = "hpass" if dom == "hstep" else "wpass"
        traffic = None
        if (atlas and r == 20 and method != "brunet" and
                (kname, precision) in PASS_DRAM_BYTES_PER_ELEMENT):
            traffic = PASS_DRAM_BYTES_PER_ELEMENT[(kname, precision)] * n * p  # per launch
        roof = {
            "bound": "hbm",
            "kernel": kernel_name(method, precision, dom),
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "peak_kind": peak_kind,
            "launches": nl,
            "main_form_iterations": main_iters,
            "avg_launch_ms": avg_ms,
            "traffic": traffic,
            "traffic_note": ("ncu DRAM bytes per launch, measured on the 20000x20000 slice and "
                             "scaled by V elements") if traffic else None,
            "algorithmic_bytes_per_launch": bytes_per_launch,
            "class_ms": {name: classes[name][1] for name, _ in KCLASSES},
        }
        if method == "brunet" and precision == "fp64" and fp64_tflops:
            # A ratio pass recomputes WH (2 n p r) and contracts (2 n p r).
            flops = 4.0 * n * p * r
            tf = flops / (avg_ms / 1000.0) / 1e12
            roof["fp64_flops"] = {"achieved": tf, "peak": fp64_tflops, "unit": "TFLOP/s",
                                  "frac": tf / fp64_tflops,
                                  "peak_kind": "measured cuBLAS f64 GEMM 8192^3, same run",
                                  "flops_per_launch": flops}
        if n * p * 8 <= 126e6:
            roof["regime"] = ("V (f64) fits in the 126 MB L2: the GB/s figure is L2 and HBM "
                              "traffic together, not an HBM roofline")
        return roof

    # Headline: the requested precision (f64 by default), clocks sampled.
    with Clocks(local) as clk:
        ms, launches, classes, W, H = timed(args.method, args.precision)
    clocks = clk.summary()
    ms_max = max_over_ranks(ms, world)
    value = world * steps / (ms_max / 1000.0)
    roof = roofline(args.method, args.precision, classes)

    extra = {}
    if not args.no_fp64_compare:
        # The mixed-precision forms against the f64 run of the same inputs.
        def compare(method, W64, H64, ms64, precisions):
            out = {}
            o_plain = objective_torch(V64, p, W64, H64, method)
            fp64_rate = rate(ms64)
            for prec in precisions:
                ms_m, _, cls_m, Wm, Hm = timed(method, prec)
                o_m = objective_torch(V64, p, Wm, Hm, method)
                rf = roofline(method, prec, cls_m)
                out[prec] = {
                    "iters_per_s": rate(ms_m),
                    "over_fp64": rate(ms_m) / fp64_rate,
                    "rel_objective_vs_fp64": abs(o_m - o_plain) / abs(o_plain),
                    "max_rel_dW_vs_fp64": float((Wm - W64).abs().max() / W64.abs().max()),
                    "dominant_pass": {"kernel": rf["kernel"], "avg_launch_ms": rf["avg_launch_ms"],
                                      "achieved_gbs": rf["achieved"], "frac": rf["frac"]},
                }
            return out

        if args.precision == "fp64":
            extra["mixed"] = {args.method: {"fp64_iters_per_s": value,
                                            **compare(args.method, W, H, ms, ("bf16x3", "fp32"))}}
            if atlas and args.method == "lee":
                # brunet (KL) at the same shape: the plain f64 ratio passes and
                # the split-bf16 tensor-core ratio passes.
                ms_b, _, cls_b, Wb, Hb = timed("brunet", "fp64")
                extra["mixed"]["brunet"] = {
                    "fp64_iters_per_s": rate(ms_b),
                    "fp64_roofline": roofline("brunet", "fp64", cls_b),
                    **compare("brunet", Wb, Hb, ms_b, ("bf16x3",))}
        else:
            ms64, _, _, W64, H64 = timed(args.method, "fp64")
            o_plain = objective_torch(V64, p, W64, H64, args.method)
            o_m = objective_torch(V64, p, W, H, args.method)
            extra["fp64_iters_per_s"] = rate(ms64)
            extra["mixed_over_fp64"] = value / rate(ms64)
            extra["rel_objective_vs_fp64"] = abs(o_m - o_plain) / abs(o_plain)
            extra["max_rel_dW_vs_fp64"] = float((W - W64).abs().max() / W64.abs().max())

    if atlas and not args.no_fp64_compare and args.workload == "atlas":
        # The 2000 x 7750 rank-10 workload (brunet and hals, FP64, 100
        # iterations from the seeded uniform start), measured beside the
        # headline: iterations/s and the fused KL ratio passes' GB/s and
        # FP64 TFLOP/s.
        extra["pbmc8k"] = small_workload_extra(ctx, local, dev, fp64_tflops, world)

    # End to end through the host-pointer C ABI.
    e2e = None
    if not args.no_e2e:
        V_host = torch.empty((n, p), dtype=torch.float64, pin_memory=True)
        V_host.copy_(V64[:, :p])
        W0h = W0.cpu().numpy()
        H0h = H0.cpu().numpy()
        Vh = V_host.numpy()
        del V64, V32
        torch.cuda.empty_cache()
        Wout = np.empty_like(W0h)
        Hout = np.empty_like(H0h)
        import ctypes

        lib = _native.load()
        o = options(args.method, args.precision, steps)
        nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)
        dp = _native._ptr
        # warm-up (allocates the library's workspace)
        ow = options(args.method, args.precision, 1)
        _native.check(lib.nmfcu_run(ctypes.byref(ow), n, p, r, dp(Vh), dp(W0h), dp(H0h), dp(Wout),
                                    dp(Hout), None, 0, ctypes.byref(nd), ctypes.byref(ni)))
        barrier(world)
        t0 = time.perf_counter()
        _native.check(lib.nmfcu_run(ctypes.byref(o), n, p, r, dp(Vh), dp(W0h), dp(H0h), dp(Wout),
                                    dp(Hout), None, 0, ctypes.byref(nd), ctypes.byref(ni)))
        t_e2e = time.perf_counter() - t0
        t_e2e = max_over_ranks(t_e2e, world)
        e2e = {"value": world * steps / t_e2e, "unit": "iters/s",
               "h2d_bytes_per_step": (n * p + n * r + r * p) * 8 / steps,
               "d2h_bytes_per_step": (n * r + r * p) * 8 / steps,
               "note": ("one nmfcu_run call per K steps (the call behind nmf_rs.nmf): V, W0, "
                        "H0 uploaded from pinned host memory once, W, H read back once")}
        del V_host
    else:
        del V64, V32

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from nmf_rs import synthetic

        def V_host_fn(p_s):
            V = synthetic.counts_matrix(n, p_s, k, alpha, seed=0)
            W0s, H0s = synthetic.starting_point(V, r, seed=0)
            return V, W0s, H0s

        cpu = cpu_baseline(V_host_fn, n, p, r, args.method, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": iterate_metric(args.method, args.workload),
            "value": value,
            "unit": "iters/s",
            "n_gpus": world,
            "steps": steps,
            "warmup": warm,
            "ms_per_step": ms_max / steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"fp32": "f32 products, f64 epilogues/objective",
                      "bf16x3": "bf16x3 (split bf16, f32 accumulation), f64 epilogues",
                      "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded single-cell-like generator on the device)",
            "config": {"workload": args.workload, "n": n, "p": p, "rank": r,
                       "method": args.method, "precision": args.precision,
                       "start": ("NNDSVD (mean fill), f64, on the device"
                                 if atlas else "seeded uniform"),
                       "parallelism": f"replicas x{world}",
                       "l2": ("V is larger than L2 (no flush needed)" if n * p * 8 > 126e6 else
                              "V fits in L2 (126 MB): L2-resident regime, no flush")},
            "gpu_launches": launches,
            "clocks": clocks,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            **extra,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def small_workload_extra(ctx, local, dev, fp64_tflops, world):
    """brunet and hals in FP64 on the 2000 x 7750 rank-10 workload, 100
    timed iterations each (after 3 untimed), with the dominant pass's
    achieved GB/s (one f64 read of V a launch; V fits in L2, so this is L2
    and HBM together) and, for brunet's fused ratio passes, FP64 TFLOP/s
    (4 n p r a launch) against a cuBLAS f64 GEMM measured in the same run."""
    import torch

    from nmf_rs import _native

    n, p, k, alpha, r, iters = WORKLOADS["pbmc8k"]
    V64, ld64, _, _, W0, H0 = device_workload(n, p, k, alpha, r, 4321, dev)
    # A stream of its own: the library replays the iterations as a CUDA graph
    # on a capturable stream when its per-kernel timing is off.
    stream = torch.cuda.Stream(dev)
    out = {"n": n, "p": p, "rank": r, "iterations": iters, "precision": "fp64",
           "start": "seeded uniform", "regime": "V (124 MB f64) fits in the 126 MB L2"}
    for method in ("brunet", "hals"):
        o = _native.default_options()
        o.method = _native.parse_method(method)
        o.stop = 0
        o.precision = _native.PRECISIONS["fp64"]
        o.device = local

        def run(iters_, W, H):
            o.max_iter = iters_
            ctx.run(o, n, p, r, V64.data_ptr(), _native.F64, ld64, W.data_ptr(), H.data_ptr(),
                    stream=stream.cuda_stream)

        def once(timing):
            W, H = W0.clone(), H0.clone()
            torch.cuda.synchronize()
            ctx.reset_timing()
            ctx.set_timing(timing)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run(iters, W, H)
            e1.record(stream)
            torch.cuda.synchronize()
            cls = {name: ctx.kernel_time(kc) for name, kc in
                   (("hstep", _native.KCLASS_HSTEP), ("wstep", _native.KCLASS_WSTEP))}
            ctx.set_timing(False)
            return max_over_ranks(e0.elapsed_time(e1), world), cls

        W, H = W0.clone(), H0.clone()
        run(3, W, H)
        ms, _ = once(False)            # the rate: graph-replayed iterations
        ms_t, classes = once(True)     # the passes' times (launched one by one)
        dom = max(classes, key=lambda c: classes[c][1])
        nl, tot = classes[dom]
        avg = tot / max(nl, 1)
        line = {"iters_per_s": world * iters / (ms / 1000.0),
                "iters_per_s_with_kernel_timing": world * iters / (ms_t / 1000.0),
                "dominant_pass": {"kernel": ("h" if dom == "hstep" else "w") + "pass_dmma" +
                                  ("_ratio" if method == "brunet" else ""),
                                  "avg_launch_ms": avg,
                                  "achieved_gbs": n * p * 8 / (avg / 1000.0) / 1e9,
                                  "pass_share_of_step": (classes["hstep"][1] +
                                                         classes["wstep"][1]) / ms_t}}
        if method == "brunet" and fp64_tflops:
            tf = 4.0 * n * p * r / (avg / 1000.0) / 1e12
            line["dominant_pass"]["fp64_tflops"] = tf
            line["dominant_pass"]["fp64_frac"] = tf / fp64_tflops
        out[method] = line
    del V64
    return out


# ---------------------------------------------------------------------------
# Batching form: consensus sweep
# ---------------------------------------------------------------------------

CONSENSUS = {"n": 2000, "p": 5000, "k": 6, "alpha": 0.3, "ranks": list(range(2, 11)),
             "iters": 200}


def consensus_inputs(runs, seed=7):
    from nmf_rs import consensus, synthetic

    c = CONSENSUS
    V = synthetic.counts_matrix(c["n"], c["p"], c["k"], c["alpha"], seed)
    starts = []
    for r in c["ranks"]:
        starts.extend(consensus.restart_starts(V, r, runs))
    return V, starts


def host_linkage_seconds(p, runs=64, k=6, seed=0):
    """One cophenetic correlation on the host the way the reference workflow
    computes it (scipy average linkage + cophenet on 1 - C, p x p)."""
    from nmf_rs import consensus

    gen = np.random.default_rng(seed)
    truth = gen.integers(0, k, p)
    C = np.zeros((p, p), dtype=np.float32)
    for _ in range(runs):
        lab = np.where(gen.random(p) < 0.3, gen.integers(0, k, p), truth)
        C += lab[:, None] == lab[None, :]
    C /= runs
    t0 = time.perf_counter()
    consensus.cophenetic_correlation(C)
    consensus.dispersion_coefficient(C)
    return time.perf_counter() - t0


def consensus_cpu_baseline(V, runs, seconds, iters=200):
    """The reference workflow on the CPU restatement: per rank, one solve's
    set-up (a 1-iteration call minus an iteration) plus `iters` iterations
    (the difference of a 3- and a 1-iteration call, / 2), on a column slice of
    V and scaled to the full V, times `runs` restarts (each restart is its own
    nmf() call in the reference, so each pays the set-up); plus each rank's
    cophenetic correlation and dispersion on the host."""
    from nmf_rs import consensus

    c = CONSENSUS
    threads = os.cpu_count() or 1
    total = 0.0
    samples = []
    for r in c["ranks"]:
        def fn(p_s, r=r):
            v = np.ascontiguousarray(V[:, :p_s])
            W0, H0 = consensus.restart_starts(v, r, 1)[0]
            return v, W0, H0
        p_s = pick_slice(fn, c["p"], "brunet", seconds / len(c["ranks"]), threads)
        v, W0, H0 = fn(p_s)
        per_iter, t_one, _ = oracle_iteration_seconds("brunet", v, W0, H0, 2, threads)
        setup = max(t_one - per_iter, 0.0)
        total += runs * (setup + iters * per_iter) * c["p"] / p_s
        samples.append(f"k={r}: {p_s} cols, {1000 * per_iter:.1f} ms/it + {1000 * setup:.1f} ms")
    t_link = host_linkage_seconds(c["p"])
    total += len(c["ranks"]) * t_link
    return {"value": runs * len(c["ranks"]) / total, "unit": "solves/s",
            "cores": threads, "kind": "port",
            "sample": ("brunet on the CPU restatement (oracle/, -march=native, OpenMP) per rank "
                       "2..10 on a column slice of V (" + "; ".join(samples) + "), "
                       f"scaled to {runs} restarts x {iters} iterations on 2000x5000; "
                       f"plus 9 x {t_link:.2f} s of scipy average linkage + cophenet + "
                       f"dispersion on a {c['p']}x{c['p']} consensus matrix")}


def run_consensus_reference(args, world, rank):
    if rank != 0:
        return
    V, _ = consensus_inputs(1)
    vals, base = [], None
    for _ in range(max(1, min(args.steps or 3, 3))):
        base = consensus_cpu_baseline(V, args.runs, args.cpu_seconds, args.iters)
        vals.append(base["value"])
    value = statistics.median(vals)
    c = CONSENSUS
    print(json.dumps({
        "impl": "reference",
        "metric": f"consensus sweep solves/s ({args.runs} brunet restarts x ranks 2..10, "
                  f"{args.iters} iterations, 2000x5000)",
        "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps or 3,
        "warmup": args.warmup, "ms_per_step": 1000.0 * args.runs * len(c["ranks"]) / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded single-cell-like generator)",
        "config": {"workload": "consensus-sweep", "n": c["n"], "p": c["p"], "ranks": "2..10",
                   "restarts": args.runs, "iters": args.iters},
        "cpu_baseline": {**base, "value": value},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_consensus(args, world, rank, local):
    import ctypes

    import torch

    from nmf_rs import _native, consensus

    c = CONSENSUS
    n, p, iters = c["n"], c["p"], args.iters
    runs = args.runs
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    V, starts = consensus_inputs(runs)
    ranks = np.array([w.shape[1] for w, _ in starts], dtype=np.int32)
    offs = np.concatenate([[0], np.cumsum(ranks)[:-1]]).astype(np.int64)
    nsolves = len(ranks)
    rtot = int(ranks.sum())
    W0 = np.ascontiguousarray(np.concatenate([w for w, _ in starts], axis=1))
    H0 = np.ascontiguousarray(np.concatenate([h for _, h in starts], axis=0))
    del starts
    dV = torch.from_numpy(V).to(dev)
    dW0 = torch.from_numpy(W0).to(dev)
    dH0 = torch.from_numpy(H0).to(dev)
    dW, dH = dW0.clone(), dH0.clone()
    ctx = _native.Context(local)
    lib = _native.load()
    stream = torch.cuda.current_stream(dev)
    prec = _native.PRECISIONS[args.precision]
    i32p = ctypes.POINTER(ctypes.c_int32)
    rp = ranks.ctypes.data_as(i32p)
    cons = torch.empty((len(c["ranks"]), p, p), dtype=torch.float32, device=dev)
    sels = [np.arange(ci * runs, (ci + 1) * runs, dtype=np.int32) for ci in range(len(c["ranks"]))]

    def post():
        """The nine consensus matrices and their statistics (dH: all solves),
        the nine average-linkage trees built concurrently."""
        for ci, sel in enumerate(sels):
            _native.check(lib.nmfcu_consensus_device(
                ctx.handle, p, nsolves, rp, ctypes.c_void_p(dH.data_ptr()), runs,
                sel.ctypes.data_as(i32p), ctypes.c_void_p(cons[ci].data_ptr()),
                ctypes.c_void_p(stream.cuda_stream)))
        consensus.consensus_stats_batch(cons, ctx)  # cophenetic + dispersion, on the GPU

    def batched_sweep():
        dW.copy_(dW0)
        dH.copy_(dH0)
        _native.check(lib.nmfcu_run_batch_device(
            ctx.handle, _native.parse_method("brunet"), prec, iters, n, p,
            ctypes.c_void_p(dV.data_ptr()), p, nsolves, rp, ctypes.c_void_p(dW.data_ptr()),
            ctypes.c_void_p(dH.data_ptr()), ctypes.c_void_p(stream.cuda_stream)))
        post()

    warm = max(3, args.warmup)
    steps = args.steps or 3
    for _ in range(warm):
        batched_sweep()
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    barrier(world)
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            batched_sweep()
        e1.record(stream)
        torch.cuda.synchronize()
    clocks = clk.summary()
    launches = ctx.launch_count() - l0
    ms = max_over_ranks(e0.elapsed_time(e1), world) / steps
    value = world * nsolves / (ms / 1000.0)

    # The same solves one by one through the single-solve engine, on a
    # stream of their own so that each solve replays its iterations as a
    # CUDA graph, as nmf() does (the best single-solve path).
    seq_runs = min(runs, runs if args.seq_runs is None else args.seq_runs)
    seq_value = dh_rel = t_seq_solves = t_post = None
    if seq_runs > 0:
        o = _native.default_options()
        o.method = _native.parse_method("brunet")
        o.stop = 0
        o.precision = prec
        o.max_iter = iters
        o.refine_iters = 0
        o.device = local
        pick = [ci * runs + i for ci in range(len(c["ranks"])) for i in range(seq_runs)]
        side = torch.cuda.Stream(dev)

        side.wait_stream(stream)

        def one(s_):
            a, r = int(offs[s_]), int(ranks[s_])
            with torch.cuda.stream(side):  # the copies and the solve on the side stream
                w = dW0[:, a:a + r].contiguous()
                h = dH0[a:a + r].contiguous()
                ctx.run(o, n, p, r, dV.data_ptr(), _native.F64, p, w.data_ptr(), h.data_ptr(),
                        stream=side.cuda_stream)
            return h

        one(0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s_ in pick:
            h = one(s_)
        torch.cuda.synchronize()
        t_seq = (time.perf_counter() - t0) * runs / seq_runs
        t_seq_solves = t_seq
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        post()  # the same consensus matrices and statistics as the batched step
        torch.cuda.synchronize()
        t_post = time.perf_counter() - t0
        t_seq += t_post
        seq_value = nsolves / t_seq
        a, r = int(offs[pick[-1]]), int(ranks[pick[-1]])
        dh_rel = float((h - dH[a:a + r]).abs().max() / h.abs().max())

    # End to end: host V in, stacked factors and consensus matrices out.
    t0 = time.perf_counter()
    consensus.consensus_sweep(V, c["ranks"], runs, iters, precision=args.precision,
                              device=local, metrics=True)
    t_e2e = time.perf_counter() - t0
    # The consensus statistics alone: device vs the host (scipy) path.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        consensus.consensus_stats(cons[0], ctx)
    stats_ms = (time.perf_counter() - t0) / 3 * 1000.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    consensus.consensus_stats_batch(cons, ctx)
    batch_stats_ms = (time.perf_counter() - t0) * 1000.0
    host_stats_ms = host_linkage_seconds(p) * 1000.0
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = consensus_cpu_baseline(V, runs, args.cpu_seconds, iters)
    if rank == 0:
        print(json.dumps({
            "metric": f"consensus sweep solves/s ({runs} brunet restarts x ranks 2..10, "
                      f"{iters} iterations, 2000x5000)",
            "value": value, "unit": "solves/s", "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32",
            "data": "synthetic (seeded single-cell-like generator)",
            "config": {"workload": "consensus-sweep", "n": n, "p": p, "ranks": "2..10",
                       "restarts": runs, "iters": iters, "solves": nsolves, "sum_rank": rtot,
                       "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": "V (80 MB f64 / 40 MB f32) stays L2-resident by design"},
            "gpu_launches": launches,
            "clocks": clocks,
            "one_by_one_solves_per_s": seq_value,
            "batched_over_one_by_one": value / seq_value if seq_value else None,
            "batched_over_one_by_one_solves_only": (
                t_seq_solves / (ms / 1000.0 - t_post) if seq_value and ms / 1000.0 > t_post
                else None),
            "one_by_one_sample": f"{seq_runs} of {runs} restarts per rank timed, scaled; plus "
                                 "the same consensus matrices and statistics",
            "max_rel_dH_batched_vs_single": dh_rel,
            "batch_shape": {"chosen": consensus.last_batch_shape(),
                            "candidates": consensus.batch_shape_count(),
                            "how": "autotuned: each shape timed on the first run, fastest kept"},
            "consensus_stats_ms_per_rank": stats_ms,
            "consensus_stats_ms_all_ranks_concurrent": batch_stats_ms,
            "host_scipy_stats_ms_per_rank": host_stats_ms,
            "cpu_baseline": cpu,
            "e2e": {"value": world * nsolves / t_e2e, "unit": "solves/s",
                    "h2d_bytes_per_step": V.nbytes + W0.nbytes + H0.nbytes,
                    "d2h_bytes_per_step": W0.nbytes + H0.nbytes + len(c["ranks"]) * p * p * 4,
                    "note": "consensus_sweep: host V/starts in, stacked W/H, 9 consensus "
                            "matrices and their cophenetic/dispersion (on the GPU) out"},
        }), flush=True)
    ctx.close()


# ---------------------------------------------------------------------------
# Serving form: Poisson request stream
# ---------------------------------------------------------------------------

SERVE_METHODS = (("lee", 0.4), ("brunet", 0.3), ("hals", 0.2), ("dnmf", 0.1))
SERVE_MAX = (5000, 50000)


def serve_requests(count, seed=11):
    """The request mix: (n, p, rank, method, iterations) per request."""
    gen = np.random.default_rng(seed)
    names = [m for m, _ in SERVE_METHODS]
    probs = [w for _, w in SERVE_METHODS]
    out = []
    for _ in range(count):
        n = int(round(np.exp(gen.uniform(np.log(500), np.log(5000)))))
        p = int(round(np.exp(gen.uniform(np.log(1000), np.log(50000)))))
        out.append((n, p, int(gen.integers(5, 31)), str(gen.choice(names, p=probs)),
                    int(gen.integers(25, 201))))
    return out


def serve_cpu_rate(V_host, reqs, seconds):
    """Oracle seconds per (row x column x iteration), from 1 iteration of each
    method on a block of V; returns (iters/s for the whole mix, sample)."""
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    n_s, p_s = 1000, 2000
    v = np.ascontiguousarray(V_host[:n_s, :p_s])
    per = {}
    for m, _ in SERVE_METHODS:
        gen = np.random.default_rng(0)
        W0 = gen.uniform(0, 1, (n_s, 15))
        H0 = gen.uniform(0, 1, (15, p_s))
        t0 = time.perf_counter()
        oracle.nmf_method(m, v, W0, H0, 1, num_threads=threads)
        per[m] = (time.perf_counter() - t0) / (n_s * p_s * 15)
    total_s = sum(per[m] * n * p * r * it for n, p, r, m, it in reqs)
    iters = sum(it for *_, it in reqs)
    return iters / total_s, {
        "cores": threads,
        "sample": (f"1 iteration per method of the CPU restatement (oracle/, OpenMP) on a "
                   f"{n_s}x{p_s} rank-15 block, scaled by rows x columns x rank x iterations "
                   f"to the {len(reqs)}-request mix")}


def run_serve_reference(args, world, rank):
    if rank != 0:
        return
    from nmf_rs import synthetic

    reqs = serve_requests(args.requests)
    V = synthetic.counts_matrix(1000, 2000, 12, 0.3, 4321)
    value, info = serve_cpu_rate(V, reqs, args.cpu_seconds)
    iters = sum(it for *_, it in reqs)
    print(json.dumps({
        "impl": "reference",
        "metric": f"served iterations/s ({len(reqs)} Poisson-arriving mixed requests, "
                  f"FP32 form, {args.slots} slots)",
        "value": value, "unit": "iters/s", "n_gpus": args.gpus, "steps": len(reqs),
        "warmup": args.warmup, "ms_per_step": 1000.0 * iters / value / len(reqs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded single-cell-like generator)",
        "config": {"workload": "serve-stream", "requests": len(reqs)},
        "cpu_baseline": {"value": value, "unit": "iters/s", "kind": "port", **info},
        "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference runs requests one after another on the host cores",
    }), flush=True)


def run_serve(args, world, rank, local):
    import ctypes

    import torch

    from nmf_rs import _native

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    reqs = serve_requests(args.requests)
    N, P = SERVE_MAX
    # One pinned host V; request i reads its top-left n x p block (ldv = P).
    V64, ld64, V32, ld32, _, _ = device_workload(N, P, 12, 0.3, 5, 4321 + rank, dev)
    V_host = torch.empty((N, P), dtype=torch.float64, pin_memory=True)
    V_host.copy_(V64[:, :P])
    del V64, V32
    torch.cuda.empty_cache()
    Vh = V_host.numpy()
    lib = _native.load()
    h = ctypes.c_void_p()
    _native.check(lib.nmfcu_server_create(local, args.slots, 0, ctypes.byref(h)))
    gen = np.random.default_rng(5)
    bufs = []
    for n, p, r, m, it in reqs:
        top = 1.0
        W0 = gen.uniform(0, top, (n, r))
        H0 = gen.uniform(0, top, (r, p))
        o = _native.default_options()
        o.method = _native.parse_method(m)
        o.precision = _native.PRECISIONS["fp32"]
        o.max_iter = it
        o.refine_iters = 2
        o.device = local
        bufs.append((o, W0, H0, np.empty((n, r)), np.empty((r, p))))
    dp = _native._ptr

    def submit(i):
        n, p, r, m, it = reqs[i]
        o, W0, H0, W, H = bufs[i]
        rid = ctypes.c_int64(0)
        _native.check(lib.nmfcu_server_submit(
            h, ctypes.byref(o), n, p, r, dp(Vh), P, dp(W0), dp(H0), dp(W), dp(H), None, 0,
            ctypes.byref(rid)))
        return rid.value

    def wait(rid):
        ni, nd = ctypes.c_int64(0), ctypes.c_int64(0)
        _native.check(lib.nmfcu_server_wait(h, rid, -1, ctypes.byref(ni), ctypes.byref(nd)))
        return ni.value

    # Warm-up: the first requests as one burst (untimed).
    warm = list(range(min(len(reqs), max(3, args.warmup) * args.slots)))
    ids = [submit(i) for i in warm]
    for rid in ids:
        wait(rid)
    # Capacity: the whole stream run closed-loop at constant concurrency (a
    # new request is submitted whenever one completes, so the server never
    # has a choice of order): work units (rows x columns x rank x
    # iterations) completed per second until the last submission, over the
    # mean work of a request: requests per second.  The open-loop stream
    # below then arrives at args.load of that.
    def poll(rid):
        state = ctypes.c_int32(0)
        _native.check(lib.nmfcu_server_poll(h, rid, ctypes.byref(state)))
        return state.value

    cal = reqs
    cal_work = [n * p * r * it for n, p, r, _, it in cal]
    t0 = time.perf_counter()
    inflight = {}
    nxt = 0
    work_done = iters_done = 0
    while nxt < len(cal) and len(inflight) < args.slots:
        inflight[submit(nxt)] = nxt
        nxt += 1
    while nxt < len(cal):
        finished = [rid for rid in inflight if poll(rid) == 2]
        if not finished:
            time.sleep(0.0002)
            continue
        for rid in finished:
            iters_done += wait(rid)
            work_done += cal_work[inflight.pop(rid)]
            if nxt < len(cal):
                inflight[submit(nxt)] = nxt
                nxt += 1
    cal_s = time.perf_counter() - t0
    cal_iters = iters_done
    for rid in list(inflight):
        wait(rid)
    units = [n * p * r * it for n, p, r, _, it in reqs]
    rate_cap = work_done / cal_s / float(np.mean(units))
    lam = args.load * rate_cap  # requests per second
    _native.check(lib.nmfcu_server_reset_stats(h))
    arrivals = np.cumsum(np.random.default_rng(17).exponential(1.0 / lam, len(reqs)))
    barrier(world)
    with Clocks(local) as clk:
        t_start = time.perf_counter()
        ids = []
        for i, ta in enumerate(arrivals):
            delay = ta - (time.perf_counter() - t_start)
            if delay > 0:
                time.sleep(delay)
            ids.append(submit(i))
        total_iters = sum(wait(rid) for rid in ids)
        elapsed = time.perf_counter() - t_start
    clocks = clk.summary()
    st = _native.ServerStats()
    _native.check(lib.nmfcu_server_get_stats(h, ctypes.byref(st)))
    lib.nmfcu_server_destroy(h)
    # FP64 objective checks: a few requests again alone in FP64.
    from nmf_rs import _native as nv

    rel = []
    for i in range(min(4, len(reqs))):
        n, p, r, m, it = reqs[i]
        o, W0, H0, W, H = bufs[i]
        Vi = np.ascontiguousarray(Vh[:n, :p])
        ref = nv.py_nmf_run(m, Vi, W0, H0, it, precision="fp64", device=local)
        f = nv.divergence if m == "brunet" else nv.distance
        a, b = f(Vi, W, H), f(Vi, ref["W"], ref["H"])
        rel.append(abs(a - b) / abs(b))
    value = world * total_iters / elapsed
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cv, info = serve_cpu_rate(Vh, reqs, args.cpu_seconds)
        cpu = {"value": cv, "unit": "iters/s", "kind": "port", **info}
    h2d = sum(n * p * 8 + (n * r + r * p) * 8 for n, p, r, _, _ in reqs)
    d2h = sum((n * r + r * p) * 8 for n, p, r, _, _ in reqs)
    if rank == 0:
        print(json.dumps({
            "metric": f"served iterations/s ({len(reqs)} Poisson-arriving mixed requests, "
                      f"FP32 form, {args.slots} slots)",
            "value": value, "unit": "iters/s", "n_gpus": world, "steps": len(reqs),
            "warmup": len(warm), "ms_per_step": 1000.0 * elapsed / len(reqs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded single-cell-like generator; request blocks of one V)",
            "config": {"workload": "serve-stream", "requests": len(reqs), "slots": args.slots,
                       "shapes": "log-uniform 500x1000..5000x50000", "ranks": "5..30",
                       "iters": "25..200", "mix": "lee .4 brunet .3 hals .2 dnmf .1",
                       "arrival_rate_per_s": lam, "load": args.load,
                       "capacity": (f"the {len(cal)} requests run closed-loop with "
                                    f"{args.slots} in flight, measured until the last "
                                    f"submission: {cal_iters / cal_s:.0f} iters/s, "
                                    f"{rate_cap:.2f} requests/s"),
                       "parallelism": f"replicas x{world}"},
            "latency_ms": {"p50": st.p50_ms, "p99": st.p99_ms, "max": st.max_ms,
                           "mean_queue": st.mean_queue_ms},
            "closed_loop_iters_per_s": cal_iters / cal_s,
            "server": {"completed": st.completed, "failed": st.failed,
                       "peak_running": st.peak_running, "peak_bytes": st.peak_bytes,
                       "budget_bytes": st.budget_bytes},
            "rel_objective_vs_fp64_alone": rel,
            "gpu_launches": st.launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": h2d / len(reqs),
                    "d2h_bytes_per_step": d2h / len(reqs),
                    "note": "already end to end: host V/W0/H0 in, host W/H out, per request"},
        }), flush=True)


# ---------------------------------------------------------------------------
# NNDSVD start
# ---------------------------------------------------------------------------

FP64_PEAK_TFLOPS = 37.0  # B200 nominal dense FP64 (CUDA-core FMA and DMMA alike)


def nndsvd_passes(n, p, rank, over=10):
    """Passes over V of one randomized SVD (power iterations x 2, the final
    range product, the projection), and the test-vector count."""
    l = rank + over
    n_iter = 7 if rank < 0.1 * min(n, p) else 4
    return 2 * n_iter + 2, l


def nndsvd_cpu_baseline(n, k, alpha, rank, p_full, seconds, seed=0):
    """scikit-learn's randomized_svd -- the call the reference's nndsvd_init
    makes (python/nmf_rs/__init__.py:172-174) -- on all rows x a column
    slice, extrapolated linearly in columns (each pass over V is linear in
    p); the O((n + p) rank) post-processing is left out of the sample."""
    from sklearn.utils.extmath import randomized_svd

    from nmf_rs import synthetic

    p_s = 1024
    for _ in range(6):
        V = synthetic.counts_matrix(n, p_s, k, alpha, seed=seed)
        t0 = time.perf_counter()
        randomized_svd(V, n_components=rank, n_oversamples=10, random_state=0)
        dt = time.perf_counter() - t0
        if dt > seconds / 4 or p_s >= p_full:
            break
        p_s = int(min(p_full, max(p_s * 2, p_s * (seconds / 2) / max(dt, 1e-3))))
    t_full = dt * p_full / p_s
    return {"value": 1.0 / t_full, "unit": "starts/s", "cores": os.cpu_count() or 1,
            "kind": "reference",
            "sample": (f"scikit-learn {__import__('sklearn').__version__} randomized_svd "
                       f"(rank {rank}, 10 oversamples, numpy BLAS threads) on {n} rows x {p_s} "
                       f"of {p_full} columns took {dt:.2f} s; extrapolated linearly in columns")}


def run_nndsvd_reference(args, world, rank):
    if rank != 0:
        return
    n, p, k, alpha, r, _ = WORKLOADS[args.workload]
    vals = []
    base = None
    for _ in range(max(1, min(args.steps or 2, 3))):
        base = nndsvd_cpu_baseline(n, k, alpha, r, p, args.cpu_seconds / 2)
        vals.append(base["value"])
    value = statistics.median(vals)
    print(json.dumps({
        "impl": "reference",
        "metric": f"NNDSVD starts/s, {args.workload} {n}x{p} rank {r}",
        "value": value, "unit": "starts/s", "n_gpus": args.gpus, "steps": len(vals),
        "warmup": 0, "ms_per_step": 1000.0 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, column slice)",
        "config": {"workload": args.workload, "n": n, "p": p, "rank": r, "form": "nndsvd"},
        "cpu_baseline": {**base, "value": value},
        "e2e": {"value": value, "unit": "starts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_nndsvd(args, world, rank, local):
    import torch

    import nmf_rs
    from nmf_rs import _native, nndsvd

    n, p, k, alpha, r, _ = WORKLOADS[args.workload]
    steps = args.steps or 5
    warm = max(3, args.warmup)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    V64, ld64, V32, ld32, _, _ = device_workload(n, p, k, alpha, r, 1234 + rank, dev)
    del V32
    torch.cuda.empty_cache()
    V = V64[:, :p]
    ctx = nndsvd._context(local)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warm):
        nndsvd.nndsvd_device(V, r, fill="mean", seed=0)
    torch.cuda.synchronize()
    ctx.reset_timing()
    ctx.set_timing(True)
    launches0 = ctx.launch_count()
    barrier(world)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            W, H = nndsvd.nndsvd_device(V, r, fill="mean", seed=0)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    clocks = clk.summary()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    launches = ctx.launch_count() - launches0
    hk = ctx.kernel_time(_native.KCLASS_HSTEP)
    wk = ctx.kernel_time(_native.KCLASS_WSTEP)
    ctx.set_timing(False)
    value = world * steps / (ms / 1000.0)
    passes, l = nndsvd_passes(n, p, r)
    peak, peak_kind = measured_peaks()
    nl = hk[0] + wk[0]
    avg_ms = (hk[1] + wk[1]) / max(nl, 1)
    bytes_launch = n * p * 8
    achieved = bytes_launch / (avg_ms / 1000.0) / 1e9
    flops_launch = 2.0 * n * p * l
    roof = {
        "bound": "hbm", "kernel": "hpass/wpass (FP64, V product)", "achieved": achieved,
        "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
        "traffic": PASS_DRAM_BYTES_PER_ELEMENT[("hpass", "fp64")] * n * p
        if args.workload in ("atlas", "atlas-slice") else None,
        "traffic_note": "the FP64 H pass's ncu DRAM bytes per V element (rank-20 capture), "
                        "scaled to n x p",
        "launches": nl, "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": bytes_launch,
        "passes_per_step": passes, "test_vectors": l,
        "fp64_flops_per_launch": flops_launch,
        "fp64_tflops": flops_launch / (avg_ms / 1000.0) / 1e12,
        "fp64_frac_of_nominal": flops_launch / (avg_ms / 1000.0) / 1e12 / FP64_PEAK_TFLOPS,
        "pass_ms_of_step": (hk[1] + wk[1]) / steps,
    }
    e2e = None
    if not args.no_e2e:
        V_host = torch.empty((n, p), dtype=torch.float64, pin_memory=True)
        V_host.copy_(V)
        Vh = V_host.numpy()
        del V64, V
        torch.cuda.empty_cache()
        nmf_rs.nndsvd_init(Vh[:, :256], r, fill="mean", seed=0, device=local)  # warm-up
        barrier(world)
        t0 = time.perf_counter()
        Wh, Hh = nmf_rs.nndsvd_init(Vh, r, fill="mean", seed=0, device=local)
        t_e2e = max_over_ranks(time.perf_counter() - t0, world)
        e2e = {"value": world / t_e2e, "unit": "starts/s", "h2d_bytes_per_step": n * p * 8,
               "d2h_bytes_per_step": (n + p) * r * 8,
               "note": "nmf_rs.nndsvd_init on a host V: upload, the start, W0/H0 read back"}
        del V_host
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = nndsvd_cpu_baseline(n, k, alpha, r, p, args.cpu_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": f"NNDSVD starts/s, {args.workload} {n}x{p} rank {r}",
            "value": value, "unit": "starts/s", "n_gpus": world, "steps": steps,
            "warmup": warm, "ms_per_step": ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded single-cell-like generator on the device)",
            "config": {"workload": args.workload, "n": n, "p": p, "rank": r, "form": "nndsvd",
                       "fill": "mean", "n_oversamples": 10,
                       "parallelism": f"replicas x{world}",
                       "l2": "V is larger than L2 (no flush needed)"},
            "gpu_launches": launches, "clocks": clocks, "roofline": roof,
            "cpu_baseline": cpu, "e2e": e2e,
        }), flush=True)


# ---------------------------------------------------------------------------
# Column-sharded single solve (strong scaling)
# ---------------------------------------------------------------------------

def run_shard_bench(args, world, rank, local):
    import torch

    from nmf_rs import _native, shard

    n, p, k, alpha, r, iters = WORKLOADS[args.workload]
    steps = args.steps or iters
    warm = max(3, args.warmup)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c0, c1 = shard.split_columns(p, world, rank)
    # This rank's column block of the workload (its own generator stream),
    # W0 the same on every rank.
    V64, ld64, V32, _, _, H0 = device_workload(n, c1 - c0, k, alpha, r, 1234 + rank, dev)
    del V32
    torch.cuda.empty_cache()
    g = torch.Generator(device=dev)
    g.manual_seed(77)
    W0 = torch.rand((n, r), generator=g, device=dev, dtype=torch.float64) * 3.0
    V = V64[:, : c1 - c0]
    stream = torch.cuda.current_stream(dev)
    reduce = shard.torch_reduce()

    def options(iters_):
        o = _native.default_options()
        o.method = _native.parse_method(args.method)
        o.precision = _native.PRECISIONS[args.precision]
        o.max_iter = iters_
        o.device = local
        return o

    sh = shard.DeviceShard(V, W0, H0, options(warm))
    shard.run_shard(sh, reduce, warm, False)
    sh.status()
    sh.close()
    sh = shard.DeviceShard(V, W0, H0, options(steps))
    sh.ctx.set_timing(True)
    torch.cuda.synchronize()
    barrier(world)
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n_iter, _ = shard.run_shard(sh, reduce, steps, False)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    classes = {kc: sh.ctx.kernel_time(kc) for kc in (_native.KCLASS_HSTEP, _native.KCLASS_WSTEP)}
    launches = sh.ctx.launch_count()
    sh.close()
    value = steps / (ms / 1000.0)
    peak, peak_kind = measured_peaks()
    s_main = 8 if args.precision == "fp64" else 4
    main_iters = steps if args.precision == "fp64" else max(0, steps - 2)
    dom = max(classes, key=lambda kc: classes[kc][1])
    nl, tot = classes[dom]
    achieved = n * (c1 - c0) * s_main * main_iters / (tot / 1000.0) / 1e9 if tot > 0 else None
    if rank == 0:
        print(json.dumps({
            "metric": f"{args.method} iterations/s of one solve split by columns over {world} "
                      f"GPU(s), {args.workload} {n}x{p} rank {r}, {args.precision} form",
            "value": value, "unit": "iters/s", "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None,
            "dtype": {"fp32": "f32", "bf16x3": "bf16x3 (split bf16, f32 accumulation)",
                      "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded generator, each rank its column block)",
            "config": {"workload": args.workload, "n": n, "p": p, "rank": r,
                       "method": args.method, "precision": args.precision, "form": "shard",
                       "parallelism": f"column shards x{world}, NCCL all-reduce of "
                                      f"{8 * (n * r + r * r + r) / 1e6:.1f} MB per iteration",
                       "columns_per_rank": c1 - c0,
                       "l2": "V is larger than L2 (no flush needed)"},
            "gpu_launches": launches, "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "kernel": "rank 0's dominant V pass",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "peak_kind": peak_kind,
                         "traffic": None, "launches": nl,
                         "avg_launch_ms": tot / max(nl, 1)},
            "cpu_baseline": None,
            "e2e": None,
            "note": "e2e and cpu_baseline: see the iterate form, which runs the same passes",
        }), flush=True)


# ---------------------------------------------------------------------------
# Sparse form: V as CSR
# ---------------------------------------------------------------------------

def device_sparse_workload(n, p, k, alpha, rank, density, seed, device):
    """The workload's V with all but about `density` of its entries set to
    zero (a seeded mask), as a device CSR: (indptr int64, indices int32,
    data f64, W0, H0), built 2048 rows at a time."""
    import torch

    V64, ld64, V32, _, W0, H0 = device_workload(n, p, k, alpha, rank, seed, device)
    del V32
    g = torch.Generator(device=device)
    g.manual_seed(seed + 1)
    nz_frac = float((V64[: min(n, 512), :p] > 0).double().mean())
    keep = min(1.0, density / max(nz_frac, 1e-9))
    counts, cols, vals = [], [], []
    for r0 in range(0, n, 2048):
        blk = V64[r0:r0 + 2048, :p]
        blk = torch.where(torch.rand(blk.shape, generator=g, device=device, dtype=torch.float32)
                          < keep, blk, torch.zeros_like(blk))
        csr = blk.to_sparse_csr()
        counts.append(csr.crow_indices().diff())
        cols.append(csr.col_indices().to(torch.int32))
        vals.append(csr.values())
        del blk, csr
    del V64
    torch.cuda.empty_cache()
    indptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    indptr[1:] = torch.cumsum(torch.cat(counts), 0)
    return indptr, torch.cat(cols), torch.cat(vals), W0, H0


def run_sparse(args, world, rank, local):
    """One solve on a sparse V through nmfcu_run_csr_device (value) and
    nmfcu_run_csr with host arrays (e2e).  The roofline counts the CSR bytes
    a pass streams (12 per stored entry: the f64 value and the int32 index)
    against HBM; the factor rows each stored entry gathers come from L2."""
    import ctypes

    import torch

    from nmf_rs import _native

    n, p, k, alpha, r, iters = WORKLOADS[args.workload]
    steps = args.steps or iters
    warm = max(3, args.warmup)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    indptr, indices, data, W0, H0 = device_sparse_workload(n, p, k, alpha, r, args.density,
                                                           1234 + rank, dev)
    nnz = int(data.numel())
    torch.cuda.synchronize()
    ctx = _native.Context(local)
    stream = torch.cuda.current_stream(dev)
    lib = _native.load()

    def opts(iters_):
        o = _native.default_options()
        o.method = _native.parse_method(args.method)
        o.max_iter = iters_
        o.device = local
        return o

    def device_run(iters_, W, H):
        nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)
        _native.check(lib.nmfcu_run_csr_device(
            ctx.handle, ctypes.byref(opts(iters_)), n, p, r, nnz,
            ctypes.c_void_p(indptr.data_ptr()), ctypes.c_void_p(indices.data_ptr()),
            ctypes.c_void_p(data.data_ptr()), ctypes.c_void_p(W.data_ptr()),
            ctypes.c_void_p(H.data_ptr()), None, ctypes.byref(nd), ctypes.byref(ni),
            ctypes.c_void_p(stream.cuda_stream)))

    device_run(warm, W0.clone(), H0.clone())
    W, H = W0.clone(), H0.clone()
    torch.cuda.synchronize()
    ctx.reset_timing()
    ctx.set_timing(True)
    barrier(world)
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        device_run(steps, W, H)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    launches = ctx.launch_count()
    classes = {name: ctx.kernel_time(kc) for name, kc in
               (("hstep", _native.KCLASS_HSTEP), ("wstep", _native.KCLASS_WSTEP),
                ("other", _native.KCLASS_OTHER))}
    ctx.set_timing(False)
    value = world * steps / (ms / 1000.0)
    peak, peak_kind = measured_peaks()
    dom = max(("hstep", "wstep"), key=lambda c: classes[c][1])
    nl, tot = classes[dom]
    avg = tot / max(nl, 1)
    csr_bytes = nnz * 12
    achieved = csr_bytes / (avg / 1000.0) / 1e9
    roof = {"bound": "hbm", "kernel": ("sparse_pass<H> (CSC columns)" if dom == "hstep"
                                        else "sparse_pass<W> (CSR rows)"),
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "launches": nl, "avg_launch_ms": avg, "traffic": None,
            "algorithmic_bytes_per_launch": csr_bytes,
            "gathered_factor_bytes_per_launch": nnz * (r + r % 2) * 8,
            "class_ms": {c: classes[c][1] for c in classes},
            "note": ("algorithmic bytes = the CSR a pass streams (12 B a stored entry); each "
                     "stored entry also gathers an f64 factor row from L2")}
    # End to end: host CSR arrays through nmfcu_run_csr.
    e2e = None
    if not args.no_e2e:
        hp = indptr.cpu().numpy()
        hi = indices.cpu().numpy()
        hd = data.cpu().numpy()
        W0h, H0h = W0.cpu().numpy(), H0.cpu().numpy()
        Wo, Ho = np.empty_like(W0h), np.empty_like(H0h)
        nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)

        def host_run(iters_):
            _native.check(lib.nmfcu_run_csr(
                ctypes.byref(opts(iters_)), n, p, r, nnz, hp.ctypes.data_as(_native._i64p),
                hi.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _native._ptr(hd),
                _native._ptr(W0h), _native._ptr(H0h), _native._ptr(Wo), _native._ptr(Ho), None,
                0, ctypes.byref(nd), ctypes.byref(ni)))

        host_run(1)
        barrier(world)
        t0 = time.perf_counter()
        host_run(steps)
        t_e2e = max_over_ranks(time.perf_counter() - t0, world)
        e2e = {"value": world * steps / t_e2e, "unit": "iters/s",
               "h2d_bytes_per_step": (hp.nbytes + hi.nbytes + hd.nbytes + W0h.nbytes +
                                      H0h.nbytes) / steps,
               "d2h_bytes_per_step": (Wo.nbytes + Ho.nbytes) / steps,
               "note": "one nmfcu_run_csr call per K steps (host CSR validated and uploaded)"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # The reference densifies V (python/nmf_rs/__init__.py:495) and runs
        # the dense loop: the dense CPU restatement on slices of this V.
        hp = indptr.cpu().numpy()
        hi = indices.cpu().numpy()
        hd = data.cpu().numpy()
        import scipy.sparse as sps

        Vs = sps.csr_matrix((hd, hi, hp), shape=(n, p))
        W0h, H0h = W0.cpu().numpy(), H0.cpu().numpy()

        def V_host_fn(p_s):
            v = np.ascontiguousarray(Vs[:, :p_s].toarray())
            return v, W0h, np.ascontiguousarray(H0h[:, :p_s])

        cpu = cpu_baseline(V_host_fn, n, p, r, args.method, args.cpu_seconds)
        cpu["sample"] = "the reference densifies V; " + cpu["sample"]
    if rank == 0:
        print(json.dumps({
            "metric": f"{args.method} iterations/s, sparse {args.workload} {n}x{p} rank {r}, "
                      f"{args.density:.0%} stored",
            "value": value, "unit": "iters/s", "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator on the device, seeded mask to the density)",
            "config": {"workload": args.workload, "n": n, "p": p, "rank": r, "nnz": nnz,
                       "density": nnz / (n * p), "method": args.method, "form": "sparse",
                       "parallelism": f"replicas x{world}",
                       "l2": "the CSR is larger than L2 (no flush needed)"},
            "gpu_launches": launches, "clocks": clk.summary(), "roofline": roof,
            "cpu_baseline": cpu, "e2e": e2e,
        }), flush=True)
    ctx.close()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.form == "shard":
            if args.impl == "reference":
                run_reference(args, world, rank)
            else:
                run_shard_bench(args, world, rank, local)
        elif args.form == "sparse":
            if args.impl == "reference":
                run_reference(args, world, rank)
            else:
                run_sparse(args, world, rank, local)
        elif args.form == "nndsvd":
            if args.impl == "reference":
                run_nndsvd_reference(args, world, rank)
            else:
                run_nndsvd(args, world, rank, local)
        elif args.form == "serve":
            if args.impl == "reference":
                run_serve_reference(args, world, rank)
            else:
                run_serve(args, world, rank, local)
        elif args.form == "consensus":
            if args.impl == "reference":
                run_consensus_reference(args, world, rank)
            else:
                run_consensus(args, world, rank, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
