"""Benchmark of the B200 delayed-pivoting LU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload serve|lu|batched|ir|stream|update|sytrf|front]

Workloads (one JSON line on rank 0 each run):

serve (default; the headline metric: solves/s and p99 latency of the served
    mixed-precision form against plain FP64 at backward error <= 1e-14).  One
    step = one burst of --requests factor+solve requests (n log-uniform in
    [64, 8192] on a 24-size grid, A = U diag(sigma) V^T with kappa
    log-uniform in [1e2, 1e6] for 90 % and 1e10 for 10 %, 1-32 right-hand
    sides, 0-4 follow-up solves each) through dp_server; value = solves per
    second of the mixed-precision server.  Latency comes from an open-loop
    Poisson stream at 70 % of the measured capacity, with host timestamps at
    submission and completion; the plain-FP64 server runs the same bursts
    and the same stream.
lu  one plain-FP64 delayed_getrf of an n x n N(0,1) matrix with 0.1 % tiny
    (x1e-18) and 0.02 % exact-zero columns (n = 16384: 16 + 3), 2/3 n^3 / t in
    GFLOP/s (delayed_lu_cuda/benchmark.cu:67).
batched  one persistent launch (CUDA graph) factoring 8192 matrices, n
    log-uniform in [32, 512], 0-2 exact-zero columns each; matrices/s.
sytrf  one delayed Bunch-Kaufman LDL^T (delayed_sytrf_blocked's semantics) of
    an n x n symmetric N(0,1) matrix, n^3/3 / t in GFLOP/s; the reference arm
    times the reference's delayed_sytrf_blocked on the host cores.
front  one multifrontal hand-off (dp_front_factor) of an n x n front with n/2
    fully-summed rows / columns, partial-LU flops / t in GFLOP/s; the
    reference has no code for it, so its arm reports "unavailable".

Inputs are generated once (seeded), kept resident in HBM and restored by a
device copy before every step, outside the timed region; every step's inputs
are larger than L2, so no flush is needed between steps.  With N > 1
(torchrun) each rank runs its own replica (a single LU does not shard;
batches and request streams are independent per GPU) and `value` is the sum
over ranks divided by the slowest rank's time.
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
sys.path.insert(0, str(ROOT / "delayed-pivoting_b200"))

# ncu on B200: DRAM bytes (read + write) of one dgemm_minus_kernel launch on
# an 8192 x 8192 x 256 update per algorithmic byte (16 M N + 8 K (M + N)).
DMMA_DRAM_PER_ALGORITHMIC_BYTE = 1060.07e6 / 1107.30e6
# ncu on B200: DRAM bytes of one bk_panel_kernel launch (n = 4096, 64 columns
# over 3781 rows: 28.153 GB/s x 419.52 us) per algorithmic byte (32 B per row
# per factored column).
BK_PANEL_DRAM_PER_ALGORITHMIC_BYTE = (28.153166e9 * 419.52e-6) / (32.0 * 64 * 3781)


def lu_metric(n):
    return f"plain FP64 delayed_getrf GFLOP/s (2/3 n^3), n={n}, 0.1% tiny + 0.02% zero columns"
UNIT = "GFLOP/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nb", type=int, default=0,
                    help="LU panel width (0: the autotuned / default width)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="lu: skip dp_getrf_autotune (default widths 64 / 256)")
    ap.add_argument("--nb-outer", type=int, default=0,
                    help="LU outer block width (0: the library's default)")
    ap.add_argument("--lookahead", type=int, default=0, choices=[0, 1, 2],
                    help="LU trailing-update schedule: 0 automatic, 1 two streams, 2 one stream")
    ap.add_argument("--seed", type=int, default=16384)
    ap.add_argument("--cpu-n", type=int, default=8192, help="CPU baseline sample size")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-lu-key", action="store_true",
                    help="serve: skip the n=16384 plain-LU key of the line")
    ap.add_argument("--no-sytrf-key", action="store_true",
                    help="serve: skip the n=16384 LDL^T key of the line")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "mixed3"],
                    help="trailing-update arithmetic of the lu workload: FP64, BF16x6, BF16x3")
    ap.add_argument("--workload", default="serve",
                    choices=["serve", "lu", "batched", "ir", "stream", "update", "sytrf",
                             "front"])
    ap.add_argument("--k", type=int, default=256, help="update: inner dimension (outer block)")
    ap.add_argument("--loads", default="0.5,0.7,0.9",
                    help="stream: offered loads as fractions of the measured mixed capacity")
    ap.add_argument("--requests", type=int, default=1000, help="requests per serve step")
    ap.add_argument("--max-n", type=int, default=8192, help="largest order of the serve stream")
    ap.add_argument("--load", type=float, default=0.7, help="open-loop load / capacity")
    ap.add_argument("--count", type=int, default=8192, help="matrices per batched step")
    return ap.parse_args()


def workload(n):
    return {"n_tiny": n // 1000, "n_zero": n // 5000}


def flops(n):
    return 2.0 / 3.0 * float(n) ** 3


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi's start-up (NVML initialisation) can hold driver
            # locks for ~100 ms: let it reach its first sample before the
            # caller's timed region begins
            deadline = time.time() + 3.0
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


def fp64_peak_tflops(torch, dev):
    """FP64 ceiling measured live: cuBLAS DGEMM 8192^3 (measurement only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n**3 / (best * 1e-3) / 1e12


def cpu_reference_gflops(n, seed, threads, repeats=1):
    """The reference's own delayed_getrf (oracle/_ref, OpenBLAS) on the host cores."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import delayed_pivoting as dp
    import oracle as orc

    if orc.ref_available():
        kind, fn = "reference", orc.ref_getrf
    else:
        kind, fn = "port", orc.oracle_getrf
    w = workload(n)
    a = dp.planted_matrix(n, n, seed, w["n_tiny"], w["n_zero"])
    best = 1e30
    info = None
    for _ in range(repeats):
        f = a.copy(order="F")
        if kind == "reference":
            orc.ref_lib().ref_set_threads(threads)
        t0 = time.perf_counter()
        _, _, info = fn(f)
        best = min(best, time.perf_counter() - t0)
    return flops(n) / best / 1e9, best, kind, info


def cpu_lapack_gflops(n, seed, threads):
    """LAPACK dgetrf (OpenBLAS) through the reference's own wrapper
    (delayed_lu/lapack_dgetrf.cpp) on the same matrix, on the host cores:
    the partial-pivoting factorisation the delayed LU is compared with.
    None when the reference's CPU build is absent."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import delayed_pivoting as dp
    import oracle as orc

    if not orc.ref_available():
        return None
    w = workload(n)
    f = dp.planted_matrix(n, n, seed, w["n_tiny"], w["n_zero"]).copy(order="F")
    t0 = time.perf_counter()
    orc.ref_lapack_getrf(f, threads=threads)
    t = time.perf_counter() - t0
    return flops(n) / t / 1e9, t


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload in ("serve", "stream"):
        return serve_reference_arm(args)
    if args.workload == "batched":
        return batched_reference_arm(args)
    if args.workload == "sytrf":
        return sytrf_reference_arm(args)
    if args.workload == "front":
        return front_reference_arm(args)
    if args.workload == "ir":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no solve or "
                          "refinement path (delayed_getrf factorises only)"}), flush=True)
        return 0
    threads = os.cpu_count() or 1
    n = args.cpu_n
    times = []
    kind = None
    for i in range(args.warmup + args.steps):
        g, t, kind, info = cpu_reference_gflops(n, args.seed, threads)
        if i >= args.warmup:
            times.append(t)
    tot = sum(times)
    value = flops(n) * len(times) / tot / 1e9
    line = {
        "impl": "reference", "metric": lu_metric(args.n), "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / len(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: N(0,1) MT19937-64 seeded, planted tiny and zero columns",
        "config": {"workload": f"delayed_getrf plain FP64 n={args.n}", "sample_n": n,
                   "threads": threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"one delayed_getrf of n={n} per step (bounded sample of the "
                                   f"n={args.n} workload), OpenBLAS {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "ir":
        return run_ir(args)
    if args.workload == "stream":
        return run_stream(args)
    if args.workload == "update":
        return run_update(args)
    if args.workload == "sytrf":
        return run_sytrf(args)
    if args.workload == "front":
        return run_front(args)
    return run_lu(args)


def run_lu(args):
    import torch
    import delayed_pivoting as dp

    world, rank, local, dev, dist = _dist_setup(torch)

    n = args.n
    w = workload(n)
    a = dp.planted_matrix(n, n, args.seed + rank, w["n_tiny"], w["n_zero"])
    orig = torch.from_numpy(a.T.copy()).to(dev)  # column-major n x n
    work = torch.empty_like(orig)
    ipiv = np.zeros(n, dtype=np.int32)
    jpiv = np.zeros(n, dtype=np.int32)
    stream = torch.cuda.current_stream(dev)
    L = dp.lib()
    prec = {"fp64": dp.PRECISION_FP64, "mixed": dp.PRECISION_MIXED_BF16X6,
            "mixed3": dp.PRECISION_MIXED_BF16X3}[args.precision]
    tuned = None
    if not args.no_autotune and args.nb == 0 and args.nb_outer == 0:
        st_t, tnb, tnbo = dp.getrf_autotune(n, stream=stream)
        if st_t != 0:
            raise RuntimeError(f"dp_getrf_autotune: status {st_t}")
        tuned = {"nb": tnb, "nb_outer": tnbo, "candidates": "nb {32,64,128} x nb_outer "
                 "{64,128,256}, best of 2 on a seeded N(0,1) matrix of the same order"}

    def step(timed_events=None):
        work.copy_(orig)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, info = dp.getrf_device_ex(n, n, work, n, ipiv, jpiv, stream=stream, nb=args.nb,
                                      nb_outer=args.nb_outer, precision=prec,
                                      lookahead=args.lookahead)
        e1.record(stream)
        if st != 0:
            raise RuntimeError(dp.delayed_getrf_cuda_status_string(st))
        return e0, e1, info

    L.dp_stats_enable(1)  # warm-up also warms the library's event pool
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    L.dp_stats_enable(0)
    if dist:
        dist.barrier()

    import ctypes

    # Timed steps record device time for the trailing-update GEMM family
    # only (the roofline kernel); every family is timed in one extra step.
    g = 7 if prec != dp.PRECISION_FP64 else 3  # DP_KFAM_GEMM_MIXED / DP_KFAM_GEMM
    L.dp_stats_families.restype = ctypes.c_uint
    L.dp_stats_families.argtypes = [ctypes.c_uint]
    L.dp_stats_reset()
    L.dp_stats_families(1 << g)
    L.dp_stats_enable(1)
    events = []
    l0 = L.dp_kernel_launches()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        for _ in range(args.steps):
            events.append(step())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    launches = L.dp_kernel_launches() - l0
    L.dp_stats_enable(0)
    ms = sum(e0.elapsed_time(e1) for e0, e1, _ in events)
    info = events[-1][2]
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    stats = _stats(L)
    launches_per_step = launches / max(args.steps, 1)
    L.dp_stats_reset()
    L.dp_stats_families(0xFFFFFFFF)
    L.dp_stats_enable(1)
    step()
    torch.cuda.synchronize()
    L.dp_stats_enable(0)
    fam_stats = _stats(L)

    # e2e: host buffers through the host-memory entry point (H2D + LU + D2H).
    e2e = None
    if not args.no_e2e:
        host = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        src = torch.from_numpy(a.T.copy())
        e2e_ms = 0.0
        for i in range(max(1, min(args.steps, 3)) + 1):
            host.copy_(src)
            hnp = host.numpy().T  # Fortran view of the pinned buffer
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, _ = dp.delayed_getrf_cuda_host(n, n, hnp, n, ipiv, jpiv, stream=stream)
            e1.record(stream)
            e1.synchronize()
            if st != 0:
                raise RuntimeError(dp.delayed_getrf_cuda_status_string(st))
            if i > 0:
                e2e_ms += e0.elapsed_time(e1)
        k = max(1, min(args.steps, 3))
        e2e_ms /= k
        if dist:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": world * flops(n) / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * n * 8 + 2 * n * 4,
               "ms_per_step": e2e_ms, "api": "dp_getrf_host (delayed_getrf_cuda_host)"}

    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(torch, dev)
    gemm_ms = stats["ms"][g]
    gemm_tf = stats["flops"][g] / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else 0.0
    if g == 3:
        roofline = {"bound": "tensor", "kernel": "dgemm_minus_kernel (FP64 DMMA m16n8k4)",
                    "achieved": gemm_tf, "peak": fp64, "unit": "TFLOP/s",
                    "frac": gemm_tf / fp64 if fp64 else None,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured live (FP64 is not in "
                                   "MEASURED_PEAKS.json)"}
    else:
        terms = 6 if prec == dp.PRECISION_MIXED_BF16X6 else 3
        bf16 = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
        roofline = {"bound": "tensor", "kernel": f"gemm_bf16x3_kernel (tcgen05, {terms} products)",
                    "achieved": terms * gemm_tf, "peak": bf16, "unit": "TFLOP/s",
                    "frac": terms * gemm_tf / bf16 if bf16 else None,
                    "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (measured)",
                    "algorithmic_fp64_tflops": gemm_tf}
    alg_bytes = stats["bytes"][g] / max(stats["launches"][g], 1)
    traffic = None
    if g == 3:
        # DRAM bytes per launch scaled from one ncu capture of the same kernel
        # (8192 x 8192 x 256 update: 1060.1 MB read + written against 1107.3 MB
        # algorithmic): traffic grows with the algorithmic bytes of a launch
        traffic = alg_bytes * DMMA_DRAM_PER_ALGORITHMIC_BYTE
    roofline.update({"traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                     "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of an "
                                        "8192^2 x 256 update, scaled by algorithmic bytes"
                                        if traffic is not None else None),
                     "per_launch_flops": stats["flops"][g] / max(stats["launches"][g], 1),
                     "avg_launch_ms": gemm_ms / max(stats["launches"][g], 1),
                     "launches_timed": stats["launches"][g]})

    value = world * flops(n) * args.steps / (ms * 1e-3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        g_cpu, t_cpu, kind, cinfo = cpu_reference_gflops(args.cpu_n, args.seed, threads)
        cpu = {"value": g_cpu, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"one delayed_getrf of n={args.cpu_n} (same generator, 0.1%/0.02% "
                         f"planted columns), {t_cpu:.2f} s, OpenBLAS {threads} threads"}
        lap = cpu_lapack_gflops(args.cpu_n, args.seed, threads)
        if lap is not None:
            cpu["lapack_dgetrf"] = {"value": lap[0], "unit": UNIT, "cores": threads,
                                    "sample": f"LAPACK dgetrf (OpenBLAS) of the same n={args.cpu_n} "
                                              f"matrix, {lap[1]:.2f} s"}
        # one host thread, on a sample of half the order (same generator)
        n1 = max(256, args.cpu_n // 2)
        g1, t1, kind1, _ = cpu_reference_gflops(n1, args.seed, 1)
        cpu["one_thread"] = {"value": g1, "unit": UNIT, "cores": 1, "kind": kind1,
                             "sample": f"one delayed_getrf of n={n1}, {t1:.2f} s"}
        lap1 = cpu_lapack_gflops(n1, args.seed, 1)
        if lap1 is not None:
            cpu["one_thread"]["lapack_dgetrf"] = {"value": lap1[0], "unit": UNIT, "cores": 1,
                                                  "sample": f"n={n1}, {lap1[1]:.2f} s"}
    if rank == 0:
        # one extra step with every family timed (events on both streams:
        # with look-ahead the families overlap, so shares add up past 1)
        fam = ["panel", "laswp", "trsm", "gemm", "search", "swap", "other", "gemm_mixed"]
        kern = {}
        fs = fam_stats
        for i, nm in enumerate(fam):
            if fs["launches"][i] == 0:
                continue
            kern[nm] = {"ms_per_step": fs["ms"][i], "launches_per_step": fs["launches"][i],
                        "share": fs["ms"][i] / max(ms / args.steps, 1e-9)}
            if fs["flops"][i]:
                kern[nm]["tflops"] = fs["flops"][i] / (fs["ms"][i] * 1e-3) / 1e12
            if fs["bytes"][i]:
                kern[nm]["gbs"] = fs["bytes"][i] / (fs["ms"][i] * 1e-3) / 1e9
        line = {
            "metric": lu_metric(n), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic: N(0,1) MT19937-64 seeded per rank, {w['n_tiny']} tiny (x1e-18) + "
                    f"{w['n_zero']} zero columns",
            "config": {"workload": f"delayed_getrf {args.precision} n={n} (single matrix)", "n": n,
                       "nb": (tuned or {}).get("nb", args.nb or 64),
                       "nb_outer": (tuned or {}).get("nb_outer", args.nb_outer or 256),
                       "autotuned": tuned,
                       "lookahead": {0: "auto", 1: "on", 2: "off"}[args.lookahead],
                       "parallelism": f"replicas x{world}",
                       "l2": f"input {8 * n * n / 2**30:.2f} GiB " + (
                           "> L2 (no flush needed)" if 8 * n * n > 126e6 else "<= L2"), "info": info},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "gpu_launches_per_step": launches_per_step,
            "step_ms": [round(e0.elapsed_time(e1), 3) for e0, e1, _ in events],
            "clocks": clk.summary(),
            "kernels": kern,
            "reference_gpu": reference_cuda_figures(n) if args.precision == "fp64" else None,
            "fp64_peak_tflops": fp64,
            "frac_of_fp64_peak": value / world / 1e3 / fp64,
            "hbm_peak_gbs": peaks.get("hbm_gbs"),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------- ir ----

IR_KAPPAS = (1e2, 1e4, 1e6)


def run_ir(args):
    """Mixed-precision factorisation + FP64 iterative refinement against the
    plain FP64 factorisation + solve on A = U diag(sigma) V^T (U, V from the QR
    of seeded N(0,1) matrices, sigma geometric from 1 to 1/kappa) for kappa
    1e2, 1e4, 1e6, with b = A x_true at 1 and 64 right-hand sides.  Per kappa
    and precision: time of the resident factorisation and of each refined
    solve (CUDA events), refinement steps, normwise backward error and forward
    error ||x - x_true||_inf / ||x_true||_inf."""
    import torch
    import delayed_pivoting as dp

    world, rank, local, dev, dist = _dist_setup(torch)
    n = args.n
    cur = torch.cuda.current_stream()
    L = dp.lib()
    L.dp_kernel_launches.restype = ctypes_longlong()
    launches = 0  # this library's kernels in the timed repetitions

    def ev():
        return torch.cuda.Event(enable_timing=True)

    rows, mixed_rate = [], []
    clk = ClockSampler(local)
    clk.__enter__()
    for kappa in IR_KAPPAS:
        g = torch.Generator(device=dev).manual_seed(args.seed + rank + int(round(np.log10(kappa))))
        u, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
        v, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
        sigma = torch.logspace(0, -np.log10(kappa), n, dtype=torch.float64, device=dev)
        A = (u * sigma) @ v.T
        del u, v
        dA = A.T.contiguous()  # column-major A
        xs = {k: torch.randn(n, k, dtype=torch.float64, device=dev, generator=g) for k in (1, 64)}
        bs = {k: (A @ x).T.contiguous() for k, x in xs.items()}  # column-major B
        normA = torch.linalg.norm(A, float("inf"))
        for name, prec in (("mixed", dp.PRECISION_MIXED_BF16X6), ("plain", dp.PRECISION_FP64)):
            rec = None
            for it in range(args.warmup + args.steps):
                torch.cuda.synchronize()
                l0 = L.dp_kernel_launches()
                e0, e1 = ev(), ev()
                e0.record(cur)
                f = dp.Factor(n, dA, n, precision=prec)
                e1.record(cur)
                sol = {}
                for k in (1, 64):
                    X = bs[k].clone()
                    s0, s1 = ev(), ev()
                    s0.record(cur)
                    st, res = f.solve(X, n, k)
                    s1.record(cur)
                    assert st == 0, st
                    sol[k] = (X, res, s0, s1)
                torch.cuda.synchronize()
                f.close()
                if it < args.warmup:
                    continue
                launches += L.dp_kernel_launches() - l0
                fms = e0.elapsed_time(e1)
                r = {"factor_ms": fms}
                for k, (X, res, s0, s1) in sol.items():
                    Xr = X.T
                    Bk = bs[k].T
                    berr = (torch.linalg.norm(Bk - A @ Xr, float("inf"), dim=0) /
                            (normA * torch.linalg.norm(Xr, float("inf"), dim=0) +
                             torch.linalg.norm(Bk, float("inf"), dim=0))).max().item()
                    ferr = (torch.linalg.norm(Xr - xs[k], float("inf")) /
                            torch.linalg.norm(xs[k], float("inf"))).item()
                    r[f"rhs{k}"] = {"solve_ms": s0.elapsed_time(s1), "iterations": res.iterations,
                                    "refactored": res.refactored, "backward_error": berr,
                                    "forward_error": ferr}
                if rec is None or r["factor_ms"] + r["rhs64"]["solve_ms"] < \
                        rec["factor_ms"] + rec["rhs64"]["solve_ms"]:
                    rec = r  # the best of the timed repetitions
            rows.append({"kappa": kappa, "precision": name, **rec})
            if name == "mixed":
                mixed_rate.append(flops(n) / ((rec["factor_ms"] + rec["rhs64"]["solve_ms"]) * 1e-3) / 1e9)
        del A, dA, xs, bs
    clk.__exit__(None, None, None)
    value = sum(mixed_rate) / len(mixed_rate)
    if rank == 0:
        line = {
            "metric": f"mixed BF16x6 LU + FP64 refinement, time to a 64-RHS solution as GFLOP/s "
                      f"(2/3 n^3 / (factor + refined solve)), n={n}, mean over kappa 1e2/1e4/1e6",
            "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (update BF16x6, FP32 accumulation)",
            "data": "synthetic: A = U diag(sigma) V^T, U and V from the QR of seeded N(0,1), "
                    "x_true ~ N(0,1), b = A x_true",
            "config": {"workload": f"gesv with refinement n={n}, kappa {list(IR_KAPPAS)}, 1 and 64 RHS",
                       "n": n, "max_iter": 10, "tol": 1e-14, "l2": "inputs > L2 (no flush needed)"},
            "cpu_baseline": None, "e2e": None, "clocks": clk.summary(),
            "gpu_launches": int(launches), "kappas": rows,
        }
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- serve ----

SERVE_METRIC = "solves/s, p99 latency: served mixed-prec vs plain FP64 LU @ bwd err<=1e-14"
SERVE_WORKLOAD = ("served stream: n log-uniform [64, max_n = 8192] (24-order grid), A = U diag(sigma) "
                  "V^T, kappa log-uniform [1e2, 1e6] (90%) / 1e10 (10%), 1-32 RHS, 0-4 follow-up "
                  "solves, HBM budget 160 GB")


def _dist_setup(torch):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    return world, rank, local, dev, dist


def _max_over_ranks(torch, dist, dev, v):
    if not dist:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(torch, dist, dev, v):
    if not dist:
        return v
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if len(xs) else None


def _serve_summary(reqs, results):
    lat = [(r.t_done - r.t_submit) * 1e3 for r in results.values()]
    berr = [r.backward_error for r in results.values()]
    bad = [r.id for r in results.values() if r.status != 0 or not (r.backward_error <= 1e-14)]
    ill = [q for q in reqs if q.kappa >= 1e10]
    ill_fp64 = sum(1 for q in ill if results[q.rid].precision == 0)
    refac_other = sum(1 for q in reqs if q.kappa < 1e10 and results[q.rid].refactored)
    return {"p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "max_ms": max(lat) if lat else None,
            "berr_max": max(berr) if berr else None, "berr_p50": _pct(berr, 50),
            "berr_p99": _pct(berr, 99), "violations": len(bad),
            "kappa_1e10_requests": len(ill), "kappa_1e10_ended_fp64": ill_fp64,
            "refactored_below_1e10": refac_other,
            "factored_mixed": sum(1 for q in reqs if results[q.rid].precision != 0)}


def _cpu_serve_baseline(reqs, seed, orders=None, lapack=True):
    """The reference's CPU delayed_getrf (oracle/_ref, OpenBLAS on every host
    core) on the whole stream: one factorisation of a matrix of every
    distinct order the stream uses, timed, then the stream's CPU time is the
    sum over ALL its requests of the time of their order.  A nonsingular
    matrix without exact-zero columns costs delayed_getrf the same work
    whatever its entries or condition number (the same idamax / dswap /
    dscal / dger / dtrsm / dgemm calls; no fallback search fires), so one
    seeded N(0,1) matrix per order stands for every request of that order;
    info == n is checked.  The reference has no solve (delayed_getrf only
    factors): each request's solves are counted as served by its
    factorisation, which overstates the CPU.  With `lapack`, LAPACK dgetrf
    through the reference's wrapper is timed the same way.  `orders` limits
    the timed orders (warm-up passes); the value then covers only them."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import delayed_pivoting as dp
    import oracle as orc

    kind, fn = ("reference", orc.ref_getrf) if orc.ref_available() else ("port", orc.oracle_getrf)
    threads = os.cpu_count() or 1
    if kind == "reference":
        orc.ref_lib().ref_set_threads(threads)
    todo = sorted({q.n for q in reqs} if orders is None else set(orders))
    t_n, t_lap = {}, {}
    for n in todo:
        a = dp.planted_matrix(n, n, seed + n)
        f = a.copy(order="F")
        t0 = time.perf_counter()
        _, _, info = fn(f)
        t_n[n] = time.perf_counter() - t0
        if info != n:
            raise RuntimeError(f"CPU baseline: info {info} != {n}")
        if lapack and kind == "reference":
            f = a.copy(order="F")
            t0 = time.perf_counter()
            orc.ref_lapack_getrf(f)
            t_lap[n] = time.perf_counter() - t0
    sub = [q for q in reqs if q.n in t_n]
    solves = sum(len(q.solves) for q in sub)
    stream_s = sum(t_n[q.n] for q in sub)
    out = {"value": solves / stream_s, "unit": "solves/s", "cores": threads, "kind": kind,
           "sample": f"delayed_getrf timed once per distinct order ({len(t_n)} orders, "
                     f"{sum(t_n.values()):.1f} s of CPU work, seeded N(0,1) matrices), weighted by "
                     f"the stream's {len(sub)} requests ({solves} solves): {stream_s:.1f} s of CPU "
                     f"time for the stream; solves counted as free",
           "stream_cpu_s": stream_s, "requests": len(sub), "solves": solves,
           "per_order_s": {str(n): round(t, 5) for n, t in t_n.items()}}
    if t_lap:
        lap_s = sum(t_lap[q.n] for q in sub)
        out["lapack_dgetrf"] = {"value": solves / lap_s, "unit": "solves/s", "cores": threads,
                                "stream_cpu_s": lap_s,
                                "sample": "LAPACK dgetrf (OpenBLAS) through the reference's "
                                          "wrapper, timed the same way"}
    return out


FAMILY_KERNELS = {0: "panel_cluster_kernel / panel_single_kernel (panel factorisation)",
                  1: "laswp_kernel (row permutation outside the panel)",
                  2: "trsm_lower_unit_kernel (U12 = L11^-1 A12)",
                  3: "dgemm_minus_kernel (FP64 DMMA m16n8k4)",
                  7: "gemm_bf16x3_kernel<3> (tcgen05 kind::f16, 6 products, incl. operand split)"}


def _family_roofline(stats, i, peaks):
    """Roofline of one kernel family from the library's per-family CUDA events
    (dp_stats_*: events on the launching stream around every launch group):
    achieved = algorithmic bytes (and flops) per launch / average launch
    duration.  In the served burst a launch's event interval includes the
    time it waits for SMs behind other requests' kernels."""
    ms, launches = stats["ms"][i], max(stats["launches"][i], 1)
    if not stats["launches"][i] or ms <= 0:
        return None
    avg_s = ms * 1e-3 / launches
    by = stats["bytes"][i] / launches
    fl = stats["flops"][i] / launches
    hbm = peaks.get("hbm_gbs")
    gbs = by / avg_s / 1e9
    r = {"kernel": FAMILY_KERNELS.get(i, f"family {i}"), "avg_launch_ms": avg_s * 1e3,
         "launches": stats["launches"][i], "algorithmic_bytes_per_launch": by,
         "algorithmic_flops_per_launch": fl, "hbm_gbs": gbs, "hbm_peak_gbs": hbm,
         "hbm_frac": gbs / hbm if hbm else None, "traffic": None,
         "peak_source": "MEASURED_PEAKS.json (measured)" if not peaks.get("fallback")
         else "fallback figures (MEASURED_PEAKS.json absent)"}
    if i == 7:
        bf16 = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
        tf = 6 * fl / avg_s / 1e12
        r.update({"bound": "tensor", "achieved": tf, "peak": bf16, "unit": "TFLOP/s",
                  "frac": tf / bf16 if bf16 else None, "algorithmic_fp64_tflops": fl / avg_s / 1e12,
                  "tensor_frac": tf / bf16 if bf16 else None})
    else:
        r.update({"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                  "frac": gbs / hbm if hbm else None, "tflops": fl / avg_s / 1e12})
    return r


def _serve_e2e(torch, dp, sv, dist, dev, pool, rhs, reqs, warm):
    """solves/s of the mixed server on the full stream `reqs` with every input
    in pinned host memory (see run_serve)."""
    keys = sorted({(q.n, q.kappa) for q in reqs})
    hostA = {k: pool[k].cpu().pin_memory() for k in keys}
    hostB = {s.rid: rhs.src[s.rid].cpu().pin_memory() for q in reqs for s in q.solves}
    hostX = {k: torch.empty_like(v).pin_memory() for k, v in hostB.items()}
    devA = [torch.empty_like(pool[(q.n, q.kappa)]) for q in reqs]
    srv = dp.Server(precision=dp.PRECISION_MIXED_BF16X6)
    rhs.reset(torch)
    sv.replay(srv, pool, rhs, warm)  # the same warm-up as the bursts' server
    rhs.reset(torch)
    cs = torch.cuda.Stream()
    h2d = sum(8 * q.n * q.n for q in reqs) + sum(v.numel() * 8 for v in hostB.values())
    d2h = sum(v.numel() * 8 for v in hostB.values())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(cs)
    results = {}
    for q, dA in zip(reqs, devA):
        with torch.cuda.stream(cs):
            dA.copy_(hostA[(q.n, q.kappa)], non_blocking=True)
            for s_ in q.solves:
                rhs.work[s_.rid].copy_(hostB[s_.rid], non_blocking=True)
        cs.synchronize()
        for s_ in q.solves:
            b = rhs.work[s_.rid]
            if s_.factor_id == 0:
                st = srv.submit(s_.rid, q.n, dA, q.n, b, q.n, s_.nrhs,
                                followups=len(q.solves) - 1)
            else:
                st = srv.submit(s_.rid, q.n, None, q.n, b, q.n, s_.nrhs, factor_id=s_.factor_id)
            assert st == 0
        for r in srv.poll(1024, 0):
            results[r.id] = r
    total = sum(len(q.solves) for q in reqs)
    while len(results) < total:
        for r in srv.poll(1024, 20):
            results[r.id] = r
    with torch.cuda.stream(cs):
        for k_, v in hostX.items():
            v.copy_(rhs.work[k_], non_blocking=True)
    e1.record(cs)
    e1.synchronize()
    srv.close()
    e_ms = _max_over_ranks(torch, dist, dev, e0.elapsed_time(e1))
    bad = sum(1 for r in results.values() if r.status != 0 or not (r.backward_error <= 1e-14))
    del devA, hostA, hostB, hostX
    torch.cuda.empty_cache()
    return {"value": _sum_over_ranks(torch, dist, dev, total) / (e_ms * 1e-3),
            "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": e_ms, "requests": len(reqs), "solves": total,
            "api": "dp_server_submit / dp_server_poll (mixed), inputs from pinned host memory",
            "backward_error_max": max(r.backward_error for r in results.values()),
            "violations": bad}


def reference_cuda_figures(n, repeats=1, timeout=600):
    """The reference's own cuBLAS GPU build timed by its own harness
    (delayed_lu_cuda/benchmark.cu:38-72: best-of-repeats wall time around the
    device call, 2/3 n^3 GFLOP/s, diagonally dominant U(-1,1) + n I input
    from mt19937_64(20260807)), and the same unmodified harness linked against
    this library (oracle/_ref/benchmark_on_b200, the drop-in build).  Each
    line of the harness: "<name> best=<s> s, <GFLOP/s> GFLOP/s"."""
    import re

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    out = {}
    for key, name in (("reference_cublas", "ref_cuda_benchmark"),
                      ("this_library_via_reference_harness", "benchmark_on_b200")):
        p = orc.ref_binary(name)
        if p is None:
            out[key] = {"unavailable": f"oracle/_ref/{name} not built"}
            continue
        try:
            r = subprocess.run([str(p), str(n), str(repeats)], capture_output=True, text=True,
                               timeout=timeout)
        except subprocess.TimeoutExpired:
            out[key] = {"unavailable": f"{name} {n} {repeats} exceeded {timeout} s"}
            continue
        rows = {}
        for ln in r.stdout.splitlines():
            m = re.match(r"(\S+)\s+best=\s*([0-9.eE+-]+) s,\s*([0-9.eE+-]+) GFLOP/s", ln.strip())
            if m:
                rows[m.group(1)] = {"seconds": float(m.group(2)), "gflops": float(m.group(3))}
        out[key] = {"rc": r.returncode, "n": n, "repeats": repeats, "paths": rows,
                    "harness": "delayed_lu_cuda/benchmark.cu (unmodified)"}
    return out


def lu_key(torch, dp, dev, L, n=16384, warmup=2, steps=3):
    """Config-2 check carried by the default line: plain FP64 delayed_getrf of
    the n = 16384 planted matrix (seed 16384, 16 tiny + 3 zero columns), time
    per factorisation (CUDA events), GFLOP/s against the FP64 peaks measured
    live (cuBLAS DGEMM), the kernel families, and whether the records equal
    the reference's (tests/golden/config2_n16384.npz, written by the
    reference's own delayed_getrf)."""
    gold = ROOT / "tests" / "golden" / f"config2_n{n}.npz"
    w = workload(n)
    a = dp.planted_matrix(n, n, n, w["n_tiny"], w["n_zero"])
    orig = torch.from_numpy(a.T.copy()).to(dev)
    del a
    work = torch.empty_like(orig)
    ipiv = np.zeros(n, dtype=np.int32)
    jpiv = np.zeros(n, dtype=np.int32)
    stream = torch.cuda.current_stream(dev)
    st_t, tnb, tnbo = dp.getrf_autotune(n, stream=stream)
    if st_t != 0:
        raise RuntimeError(f"dp_getrf_autotune: status {st_t}")
    ms, info = [], None
    for i in range(warmup + steps + 1):
        work.copy_(orig)
        last = i == warmup + steps
        if last:
            L.dp_stats_reset()
            L.dp_stats_enable(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, info = dp.delayed_getrf_cuda_device(n, n, work, n, ipiv, jpiv, stream=stream)
        e1.record(stream)
        e1.synchronize()
        if st != 0:
            raise RuntimeError(dp.delayed_getrf_cuda_status_string(st))
        if i == warmup + steps - 1:
            report = dp.getrf_last_report()
        if last:
            L.dp_stats_enable(0)
        elif i >= warmup:
            ms.append(e0.elapsed_time(e1))
    stats = _stats(L)
    L.dp_stats_reset()
    del orig, work
    torch.cuda.empty_cache()
    fp64 = fp64_peak_tflops(torch, dev)
    gf = flops(n) / (statistics.mean(ms) * 1e-3) / 1e9
    fam = ["panel", "laswp", "trsm", "gemm", "search", "swap", "other", "gemm_mixed"]
    kern = {nm: {"ms": round(stats["ms"][i], 3), "launches": stats["launches"][i]}
            for i, nm in enumerate(fam) if stats["launches"][i]}
    out = {"n": n, "gflops": gf, "ms_per_factorisation": statistics.mean(ms),
           "step_ms": [round(x, 3) for x in ms], "info": info,
           "autotuned_widths": {"nb": tnb, "nb_outer": tnbo}, "near_tie_report": report,
           "fp64_peak_tflops_cublas_dgemm": fp64, "frac_of_fp64_peak": gf / 1e3 / fp64,
           "target_frac": 0.70, "kernels_one_step": kern,
           "reference_gpu": reference_cuda_figures(n),
           "panel_roofline": _family_roofline(stats, 0, measured_peaks())}
    if gold.exists():
        with np.load(gold) as z:
            out["records_match_reference"] = bool(
                np.array_equal(z["ipiv"], ipiv) and np.array_equal(z["jpiv"], jpiv)
                and int(z["info"]) == info)
    return out


def run_serve(args):
    import torch
    import delayed_pivoting as dp
    from delayed_pivoting import serving as sv

    world, rank, local, dev, dist = _dist_setup(torch)
    L = dp.lib()
    L.dp_kernel_launches.restype = ctypes_longlong()
    seed = args.seed + rank
    R = args.requests
    reqs = sv.make_stream(R, seed, hi=args.max_n)
    warm = reqs[:max(10, R // 10)]
    pool = sv.MatrixPool(torch, [(q.n, q.kappa) for q in reqs], seed=seed)
    rhs = sv.RhsSet(torch, pool, reqs, seed=seed + 1)
    solves_per_step = sum(len(q.solves) for q in reqs)

    def bursts(server, k, stream):
        ms = []
        res = None
        for _ in range(k):
            rhs.reset(torch)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res, _, _ = sv.replay(server, pool, rhs, stream)
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms, res

    out = {}
    modes = (("mixed", dp.PRECISION_MIXED_BF16X6), ("plain", dp.PRECISION_FP64))
    servers = {mode: dp.Server(precision=prec) for mode, prec in modes}
    # W untimed full bursts of the same stream per server: the first full
    # bursts pay one-time costs (device memory pools, resident structures)
    for mode, _ in modes:
        bursts(servers[mode], max(1, args.warmup), reqs)
    if dist:
        dist.barrier()
    # the two servers' timed bursts interleaved (mixed, plain, mixed, ...), so
    # drift over the run affects both alike
    ks = {"mixed": args.steps, "plain": max(1, min(args.steps, 2))}
    acc = {mode: {"ms": [], "res": None, "launches": 0} for mode, _ in modes}
    with ClockSampler(local) as clk:
        for i in range(max(ks.values())):
            for mode, _ in modes:
                if i >= ks[mode]:
                    continue
                l0 = L.dp_kernel_launches()
                ms1, res1 = bursts(servers[mode], 1, reqs)
                acc[mode]["launches"] += L.dp_kernel_launches() - l0
                acc[mode]["ms"] += ms1
                acc[mode]["res"] = res1
    for mode, _ in modes:
        ms = acc[mode]["ms"]
        ms_tot = _max_over_ranks(torch, dist, dev, sum(ms))
        capacity = _sum_over_ranks(torch, dist, dev, solves_per_step * ks[mode]) / (ms_tot * 1e-3)
        out[mode] = {"ms": ms, "ms_tot": ms_tot, "capacity": capacity,
                     "burst": _serve_summary(reqs, acc[mode]["res"]), "clocks": clk.summary(),
                     "launches": acc[mode]["launches"], "server": servers[mode]}
    # open-loop latency at the same offered load for both servers
    rate = args.load * (R / (out["mixed"]["ms_tot"] / args.steps * 1e-3))
    for mode in ("mixed", "plain"):
        srv = out[mode]["server"]
        rhs.reset(torch)
        res, first, last = sv.replay(srv, pool, rhs, reqs, rate=rate, seed=seed + 2)
        out[mode]["open"] = _serve_summary(reqs, res)
        out[mode]["open"]["span_s"] = last - first
    # kernel families of the mixed server (one extra burst with device timing on)
    srv = out["mixed"]["server"]
    L.dp_stats_reset()
    L.dp_stats_enable(1)
    bursts(srv, 1, reqs)
    L.dp_stats_enable(0)
    stats = _stats(L)
    for mode in ("mixed", "plain"):
        out[mode]["server"].close()
        out[mode]["server"] = None

    # e2e: the same requests as `value`, but every matrix and right-hand side
    # starts in pinned host memory: per request the H2D copies of its matrix
    # (its own device buffer) and right-hand sides, then its submission; the
    # D2H of every solution after the last result.  All inside the timed
    # region, on a server warmed like the bursts' one.
    e2e = None
    if not args.no_e2e:
        e2e = _serve_e2e(torch, dp, sv, dist, dev, pool, rhs, reqs, warm)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = _cpu_serve_baseline(reqs, seed)

    pool_gb = pool.bytes / 1e9
    lu = None
    if not args.no_lu_key:
        del pool, rhs
        torch.cuda.empty_cache()
        lu = lu_key(torch, dp, dev, L)
    sy = None
    if not args.no_sytrf_key:
        sy = sytrf_key(torch, dp, dev, cpu=rank == 0 and not args.no_cpu_baseline)

    peaks = measured_peaks()
    fam = ["panel", "laswp", "trsm", "gemm", "search", "swap", "other", "gemm_mixed"]
    kern = {nm: {"ms": stats["ms"][i], "launches": stats["launches"][i],
                 "avg_launch_us": 1e3 * stats["ms"][i] / stats["launches"][i],
                 "tflops": (stats["flops"][i] / (stats["ms"][i] * 1e-3) / 1e12
                            if stats["flops"][i] and stats["ms"][i] else None),
                 "gbs": (stats["bytes"][i] / (stats["ms"][i] * 1e-3) / 1e9
                         if stats["bytes"][i] and stats["ms"][i] else None)}
            for i, nm in enumerate(fam) if stats["launches"][i]}
    # the dominant kernel family of the burst (largest event time)
    top = max(kern, key=lambda k: kern[k]["ms"])
    roofline = _family_roofline(stats, fam.index(top), peaks)
    roofline_gemm = _family_roofline(stats, 7, peaks)
    if rank == 0:
        m, pl = out["mixed"], out["plain"]
        line = {
            "metric": SERVE_METRIC, "value": m["capacity"], "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_tot"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded QR-conditioned matrices, seeded Poisson stream",
            "config": {"workload": SERVE_WORKLOAD, "requests_per_step": R, "max_n": args.max_n,
                       "solves_per_step": solves_per_step,
                       "precision": ("mixed BF16x6 (six-product BF16 split, FP32 accumulation) + "
                                     "FP64 IR for blocked orders >= dp_server_options.mixed_min_n "
                                     f"({dp.server_options().mixed_min_n}, the measured crossover "
                                     "against FP64); FP64 factors below it and for orders <= 512"),
                       "mixed_min_n": dp.server_options().mixed_min_n,
                       "pool_gb": pool_gb, "parallelism": f"replicas x{world}",
                       "l2": "inputs per step >> L2 (no flush needed)"},
            "p99_ms": m["open"]["p99_ms"], "p50_ms": m["open"]["p50_ms"],
            "open_loop": {"rate_rps": rate, "load": args.load, "mixed": m["open"],
                          "plain": pl["open"]},
            "burst": {"mixed": m["burst"], "plain": pl["burst"]},
            "step_ms": [round(x, 1) for x in m["ms"]],
            "plain_fp64": {"solves_per_s": pl["capacity"], "ms_per_step": pl["ms_tot"] / len(pl["ms"]),
                           "step_ms": [round(x, 1) for x in pl["ms"]],
                           "p50_ms": pl["open"]["p50_ms"], "p99_ms": pl["open"]["p99_ms"],
                           "mixed_over_plain": m["capacity"] / pl["capacity"]},
            "roofline": roofline,
            "roofline_gemm_mixed": roofline_gemm,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(m["launches"]),
            "clocks": m["clocks"],
            "kernels_mixed_burst": kern,
            "lu_n16384": lu,
            "sytrf_n16384": sy,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_update(args):
    """The trailing update alone, C (n x n) -= A (n x k) B (k x n), as the LU
    runs it: on the tensor cores (BF16x6 split, dp_schur_update_mixed_device:
    the two split kernels and the persistent tcgen05 kernel) and in FP64 on
    DMMA (dp_schur_update_device).  Per call: CUDA events on the stream
    around the call; the mixed entry point synchronises itself, so its time
    includes one host round trip.  Rooflines: algorithmic bytes 16 n^2 +
    8 k (2 n) (C read and written once, A and B read once) against the
    measured HBM copy bandwidth, and 6 x 2 n^2 k BF16 flops against the
    measured BF16 peak; the FP64 kernel against the live cuBLAS DGEMM."""
    import torch
    import delayed_pivoting as dp

    world, rank, local, dev, dist = _dist_setup(torch)
    n, k = args.n, args.k
    A = torch.randn(k, n, dtype=torch.float64, device=dev)  # column-major n x k
    B = torch.randn(n, k, dtype=torch.float64, device=dev)  # column-major k x n
    C = torch.randn(n, n, dtype=torch.float64, device=dev)
    peaks = measured_peaks()
    out = {}
    for name, fn in (("mixed_bf16x6", lambda: dp.schur_update_mixed_device(n, n, k, A, n, B, k, C, n)),
                     ("fp64_dmma", lambda: dp.schur_update_device(n, n, k, A, n, B, k, C, n))):
        for _ in range(args.warmup):
            assert fn() == 0
        torch.cuda.synchronize()
        ms = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                assert fn() == 0
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        t = statistics.median(ms) * 1e-3
        fl, by = 2.0 * n * n * k, 16.0 * n * n + 16.0 * k * n
        out[name] = {"ms_median": t * 1e3, "fp64_equiv_tflops": fl / t / 1e12,
                     "alg_gbs": by / t / 1e9, "hbm_frac": by / t / 1e9 / peaks["hbm_gbs"],
                     "clocks": clk.summary()}
        if name.startswith("mixed"):
            bf16 = peaks.get("bf16_tflops") or 1590.0
            out[name]["bf16_tflops"] = 6 * fl / t / 1e12
            out[name]["tensor_frac"] = 6 * fl / t / 1e12 / bf16
    fp64 = fp64_peak_tflops(torch, dev)
    out["fp64_dmma"]["frac_of_cublas_dgemm"] = out["fp64_dmma"]["fp64_equiv_tflops"] / fp64
    m = out["mixed_bf16x6"]
    if rank == 0:
        print(json.dumps({
            "metric": f"trailing update C -= A B, n={n}, k={k}: mixed BF16x6 tensor-core kernel",
            "value": m["fp64_equiv_tflops"], "unit": "TFLOP/s (FP64-equivalent 2 n^2 k)",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["ms_median"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (operands split to BF16, FP32 accumulation)",
            "data": "synthetic N(0,1)",
            "config": {"workload": f"Schur update n={n} k={k}", "n": n, "k": k,
                       "l2": f"C {8 * n * n / 2**30:.2f} GiB"},
            "roofline": {"bound": "hbm", "achieved": m["alg_gbs"], "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": m["hbm_frac"], "traffic": None,
                         "tensor_frac": m["tensor_frac"]},
            "kernels": out, "fp64_peak_tflops_cublas_dgemm": fp64}), flush=True)
    return 0


def run_stream(args):
    """Config 5 as a swept open-loop stream: --requests requests (default
    20,000 when the flag is left at its serve default) drawn like the served
    bursts, Poisson arrivals at each offered load of --loads (fractions of the
    mixed server's capacity, measured first on one 1000-request burst), run
    through the mixed and the plain-FP64 server in turn.  Per rate and server:
    solves/s over the stream's span (first submission to last completion),
    p50 / p99 latency from the server's own timestamps, the backward-error
    distribution, and how the kappa = 1e10 requests ended."""
    import torch
    import delayed_pivoting as dp
    from delayed_pivoting import serving as sv

    world, rank, local, dev, dist = _dist_setup(torch)
    R = 20000 if args.requests == 1000 else args.requests
    seed = args.seed + rank
    reqs = sv.make_stream(R, seed, hi=args.max_n)
    probe = reqs[:1000]
    pool = sv.MatrixPool(torch, [(q.n, q.kappa) for q in reqs], seed=seed)
    rhs = sv.RhsSet(torch, pool, reqs, seed=seed + 1)
    solves = sum(len(q.solves) for q in reqs)
    out = {}
    servers = {m: dp.Server(precision=p) for m, p in
               (("mixed", dp.PRECISION_MIXED_BF16X6), ("plain", dp.PRECISION_FP64))}
    cap = {}
    for mode, srv in servers.items():
        rhs.reset(torch)
        sv.replay(srv, pool, rhs, reqs[:100])  # warm-up
        rhs.reset(torch)
        t0 = time.perf_counter()
        sv.replay(srv, pool, rhs, probe)
        torch.cuda.synchronize()
        cap[mode] = len(probe) / (time.perf_counter() - t0)
    rates = []
    for load in [float(x) for x in args.loads.split(",")]:
        rate = load * cap["mixed"]
        row = {"load": load, "rate_rps": rate}
        for mode, srv in servers.items():
            rhs.reset(torch)
            with ClockSampler(local) as clk:
                res, first, last = sv.replay(srv, pool, rhs, reqs, rate=rate, seed=seed + 2,
                                             timeout=3600.0)
            summ = _serve_summary(reqs, res)
            berr = np.array([r.backward_error for r in res.values()])
            summ.update({"solves_per_s": solves / (last - first), "span_s": last - first,
                         "berr_hist": {f"<=1e-{e}": int((berr <= 10.0 ** -e).sum())
                                       for e in (14, 15, 16)},
                         "clocks": clk.summary()})
            row[mode] = summ
        rates.append(row)
    for srv in servers.values():
        srv.close()
    if rank == 0:
        print(json.dumps({
            "metric": SERVE_METRIC + " (open-loop stream, swept rate)",
            "value": max(r["mixed"]["solves_per_s"] for r in rates), "unit": "solves/s",
            "n_gpus": world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic: seeded QR-conditioned matrices, seeded Poisson stream",
            "config": {"workload": SERVE_WORKLOAD, "requests": R, "solves": solves,
                       "max_n": args.max_n, "capacity_rps_1000_burst": cap,
                       "pool_gb": pool.bytes / 1e9},
            "rates": rates}), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def serve_reference_arm(args):
    """The reference's CPU delayed_getrf on the same stream as the GPU arm's
    `value` (the same seed, all --requests requests): every step times one
    factorisation per distinct order and weights it by the stream's counts
    (_cpu_serve_baseline); the step's solves/s are the stream's solves over
    the stream's CPU time.  Warm-up steps time the orders up to 1024 only
    (they warm OpenBLAS's thread pool and the caches)."""
    from delayed_pivoting import serving as sv

    reqs = sv.make_stream(args.requests, args.seed, hi=args.max_n)
    small = [n for n in sorted({q.n for q in reqs}) if n <= 1024]
    stream_s, solves, cpu, t_all = 0.0, 0, None, 0.0
    for i in range(args.warmup + args.steps):
        if i < args.warmup:
            _cpu_serve_baseline(reqs, args.seed, orders=small, lapack=False)
            continue
        t0 = time.perf_counter()
        cpu = _cpu_serve_baseline(reqs, args.seed, lapack=(i == args.warmup + args.steps - 1))
        t_all += time.perf_counter() - t0
        stream_s += cpu["stream_cpu_s"]
        solves += cpu["solves"]
    value = solves / stream_s
    line = {"impl": "reference", "metric": SERVE_METRIC, "value": value, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_all / max(args.steps, 1) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the GPU arm's seeded stream; seeded N(0,1) matrices per order",
            "step": "one timing pass: delayed_getrf once per distinct order of the stream "
                    "(ms_per_step is its wall time); value = the stream's solves over the "
                    "stream's CPU time (the per-order times weighted by the stream's counts)",
            "stream_cpu_s_per_step": stream_s / max(args.steps, 1),
            "config": {"workload": SERVE_WORKLOAD, "requests_per_step": args.requests,
                       "max_n": args.max_n, "solves_per_step": cpu["solves"]},
            "cpu_baseline": dict(cpu, value=value),
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# -------------------------------------------------------------- batched ----

def batch_metric(count):
    return f"batched delayed_getrf matrices/s ({count} matrices, n log-uniform [32, 512])"


def run_batched(args):
    import torch
    import delayed_pivoting as dp

    world, rank, local, dev, dist = _dist_setup(torch)
    L = dp.lib()
    L.dp_kernel_launches.restype = ctypes_longlong()
    count, seed = args.count, 8192 + rank
    ns, nz = dp.batch_orders(count, seed)
    st, tuned = dp.batch_autotune(samples=16)
    b = dp.Batch(ns, options=tuned)
    host = np.zeros(b.total_elements, dtype=np.float64)
    dp.fill_batch(host, b.offsets, ns, nz, seed)
    src = torch.from_numpy(host).to(dev)
    work = torch.empty_like(src)
    ip = torch.empty(b.total_records, dtype=torch.int32, device=dev)
    jp = torch.empty_like(ip)
    info = torch.empty(count, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        work.copy_(src)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        assert b.getrf_graph(work, ip, jp, info, stream=stream) == 0
        e1.record(stream)
        return e0, e1

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    l0 = L.dp_kernel_launches()
    with ClockSampler(local) as clk:
        ev = [step() for _ in range(args.steps)]
        torch.cuda.synchronize()
    launches = L.dp_kernel_launches() - l0
    ms = _max_over_ranks(torch, dist, dev, sum(a.elapsed_time(c) for a, c in ev))
    value = _sum_over_ranks(torch, dist, dev, count * args.steps) / (ms * 1e-3)
    fl = float((2.0 / 3.0 * ns.astype(np.float64) ** 3).sum())
    fp64 = fp64_peak_tflops(torch, dev)
    tf = fl * args.steps / (ms * 1e-3) / 1e12
    bytes_alg = float((16.0 * ns.astype(np.float64) ** 2).sum())

    # e2e: matrices from pinned host memory through the plan (H2D, launch, D2H
    # of factors and records), timed on the stream
    e2e = None
    if not args.no_e2e:
        hsrc = torch.from_numpy(host).pin_memory()
        hout = torch.empty_like(hsrc).pin_memory()
        hip = torch.empty(b.total_records, dtype=torch.int32).pin_memory()
        hjp = torch.empty_like(hip).pin_memory()
        hinfo = torch.empty(count, dtype=torch.int32).pin_memory()
        e_ms = 0.0
        k = max(1, min(args.steps, 3))
        for i in range(k + 1):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            work.copy_(hsrc, non_blocking=True)
            assert b.getrf_graph(work, ip, jp, info, stream=stream) == 0
            hout.copy_(work, non_blocking=True)
            hip.copy_(ip, non_blocking=True)
            hjp.copy_(jp, non_blocking=True)
            hinfo.copy_(info, non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            if i:
                e_ms += e0.elapsed_time(e1)
        e_ms = _max_over_ranks(torch, dist, dev, e_ms / k)
        e2e = {"value": _sum_over_ranks(torch, dist, dev, count) / (e_ms * 1e-3),
               "unit": "matrices/s", "h2d_bytes_per_step": host.nbytes,
               "d2h_bytes_per_step": host.nbytes + 8 * b.total_records + 4 * count,
               "ms_per_step": e_ms, "api": "Batch.getrf_graph (dp_batch_getrf_graph)"}

    # the mixed form (BF16x6 split trailing updates) of the same launch
    mixed = None
    opt_m = dp.batch_options(nb_bucket=list(tuned.nb_bucket), precision=dp.PRECISION_MIXED_BF16X6)
    if b.set_options(opt_m) == 0:
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ev = [step() for _ in range(args.steps)]
        torch.cuda.synchronize()
        ms_m = _max_over_ranks(torch, dist, dev, sum(a.elapsed_time(c) for a, c in ev))
        fac = work.cpu().numpy()
        ipm, jpm, infm = ip.cpu().numpy(), jp.cpu().numpy(), info.cpu().numpy()
        worst = 0.0
        for i in range(0, count, max(1, count // 24)):  # a sample of the batch
            n = int(ns[i])
            o, r0 = int(b.offsets[i]), int(b.record_offsets[i])
            a = host[o:o + n * n].reshape(n, n, order="F")
            f = fac[o:o + n * n].reshape(n, n, order="F")
            worst = max(worst, _lu_rel_residual(a, f, ipm[r0:r0 + n], jpm[r0:r0 + n], int(infm[i])))
        mixed = {"value": _sum_over_ranks(torch, dist, dev, count * args.steps) / (ms_m * 1e-3),
                 "unit": "matrices/s", "ms_per_step": ms_m / args.steps,
                 "precision": "BF16x6 trailing updates (FP32 accumulation), FP64 panels",
                 "max_rel_residual_sampled": worst,
                 "sample": "every (count / 24)-th matrix: ||PAQ - LU||_F / ||A||_F"}
        b.set_options(tuned)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = _cpu_batched_baseline(ns, nz, seed)
    if rank == 0:
        line = {"metric": batch_metric(count), "value": value, "unit": "matrices/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: N(0,1) MT19937-64 per matrix, 0-2 zero columns (p = 0.3)",
                "config": {"workload": f"batched delayed_getrf, {count} matrices, n log-uniform "
                                       f"[32, 512], one CUDA-graph launch per step",
                           "nb_bucket": list(tuned.nb_bucket), "gflop_per_step": fl / 1e9,
                           "parallelism": f"replicas x{world}",
                           "l2": f"{host.nbytes / 1e9:.2f} GB per step > L2 (no flush needed)"},
                "roofline": {"bound": "tensor", "kernel": "batched_getrf_kernel (whole launch)",
                             "achieved": tf, "peak": fp64, "unit": "TFLOP/s", "frac": tf / fp64,
                             "peak_source": "cuBLAS DGEMM 8192^3 measured live",
                             "hbm_gbs": bytes_alg * args.steps / (ms * 1e-3) / 1e9,
                             "hbm_peak_gbs": measured_peaks().get("hbm_gbs"), "traffic": None},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary(), "mixed_form": mixed}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _lu_rel_residual(a, f, ipiv, jpiv, info):
    """||P A Q - L U||_F / ||A||_F of a delayed LU (records applied in step
    order; L unit lower, U upper of the first `info` steps, the rest of f the
    untouched active block)."""
    n = a.shape[0]
    pa = np.array(a, dtype=np.float64, copy=True)
    for k in range(n):
        if ipiv[k] != k:
            pa[[k, ipiv[k]], :] = pa[[ipiv[k], k], :]
        if jpiv[k] != k:
            pa[:, [k, jpiv[k]]] = pa[:, [jpiv[k], k]]
    k = max(0, min(info, n))
    L = np.tril(f, -1)[:, :k] + np.eye(n)[:, :k]
    U = np.triu(f)[:k, :]
    lu = L @ U
    lu[k:, k:] += f[k:, k:]
    an = np.linalg.norm(a)
    return float(np.linalg.norm(pa - lu) / an) if an > 0 else 0.0


def _cpu_batched_baseline(ns, nz, seed, budget_s=15.0):
    """The reference's delayed_getrf on the host cores, matrix after matrix
    (OpenBLAS threads inside each), over the first matrices of the batch."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import delayed_pivoting as dp
    import oracle as orc

    kind, fn = ("reference", orc.ref_getrf) if orc.ref_available() else ("port", orc.oracle_getrf)
    threads = os.cpu_count() or 1
    if kind == "reference":
        orc.ref_lib().ref_set_threads(threads)
    t, k = 0.0, 0
    while k < len(ns) and t < budget_s:
        a = dp.batch_matrix(ns, nz, seed, k)
        t0 = time.perf_counter()
        fn(a)
        t += time.perf_counter() - t0
        k += 1
    return {"value": k / t, "unit": "matrices/s", "cores": threads, "kind": kind,
            "sample": f"first {k} matrices of the batch, one delayed_getrf each, {t:.1f} s"}


def batched_reference_arm(args):
    import delayed_pivoting as dp

    ns, nz = dp.batch_orders(args.count, 8192)
    vals, cpu, t_all = [], None, 0.0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cpu = _cpu_batched_baseline(ns, nz, 8192, budget_s=10.0)
        if i >= args.warmup:
            vals.append(cpu["value"])
            t_all += time.perf_counter() - t0
    value = float(np.mean(vals))
    print(json.dumps({"impl": "reference", "metric": batch_metric(args.count), "value": value,
                      "unit": "matrices/s", "n_gpus": args.gpus, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": t_all / max(args.steps, 1) * 1e3,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64", "data": "synthetic",
                      "config": {"workload": f"batched delayed_getrf, {args.count} matrices"},
                      "cpu_baseline": dict(cpu, value=value),
                      "e2e": {"value": value, "unit": "matrices/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)
    return 0


def ctypes_longlong():
    import ctypes

    return ctypes.c_longlong


def _stats(L):
    import ctypes

    class S(ctypes.Structure):
        _fields_ = [("ms", ctypes.c_double * 8), ("flops", ctypes.c_double * 8),
                    ("bytes", ctypes.c_double * 8), ("launches", ctypes.c_longlong * 8),
                    ("calls", ctypes.c_longlong)]

    s = S()
    L.dp_stats_get.argtypes = [ctypes.POINTER(S)]
    L.dp_stats_get(ctypes.byref(s))
    return {"ms": list(s.ms), "flops": list(s.flops), "bytes": list(s.bytes),
            "launches": list(s.launches), "calls": s.calls}




# ---------------------------------------------------------------- sytrf ----

def sytrf_metric(n):
    return (f"delayed Bunch-Kaufman LDL^T (delayed_sytrf_blocked) GFLOP/s (n^3/3), n={n}, "
            f"N(0,1) symmetric indefinite")


def sytrf_flops(n):
    return float(n) ** 3 / 3.0


def cpu_sytrf_gflops(n, seed, threads, variant="blocked"):
    """The reference's delayed_sytrf_blocked (delayed-bunch-kaufman/, compiled
    into oracle/_ref/; `variant` "lapack": its LAPACK dsytrf wrapper) on the
    host cores; the C restatement ('port') when the reference was not built.
    Returns (GFLOP/s, seconds, kind, info)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    import delayed_pivoting as dp

    a = dp.symmetric_matrix(n, seed)
    t0 = time.perf_counter()
    if orc.ref_bk_available():
        _, _, info = orc.ref_sytrf(a, variant, threads=threads)
        kind = "reference"
    else:
        _, _, info = orc.oracle_sytrf(a)
        kind = "port"
    t = time.perf_counter() - t0
    return sytrf_flops(n) / t / 1e9, t, kind, info


def sytrf_records_check(dp, n=4096):
    """Records of the GPU path on the seeded n = 4096 case against the
    reference's (tests/golden/sytrf/sym_4096.npz, written by the reference's
    own delayed_sytrf_blocked), with the near-tie report."""
    import torch

    gold = ROOT / "tests" / "golden" / "sytrf" / f"sym_{n}.npz"
    a = dp.symmetric_matrix(n, n)
    d = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    st, perm, piv, info = dp.sytrf_device(n, d, n)
    rep = dp.sytrf_last_report()
    out = {"n": n, "status": st, "info": info, "near_tie_report": rep}
    if gold.exists():
        with np.load(gold) as z:
            out["records_match_reference"] = bool(
                np.array_equal(z["perm"], perm) and np.array_equal(z["piv_size"], piv)
                and int(z["info"]) == info)
    del d
    return out


def sytrf_key(torch, dp, dev, n=16384, steps=2, cpu=True):
    """f4 check carried by the default line: delayed Bunch-Kaufman LDL^T of a
    seeded n = 16384 symmetric matrix (CUDA events), the records check at
    n = 4096, and the reference's CPU code on the same n = 4096 case."""
    stream = torch.cuda.current_stream(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(n)
    orig = torch.randn(n, n, dtype=torch.float64, device=dev, generator=g)
    work = torch.empty_like(orig)
    ms = []
    for i in range(steps + 1):
        work.copy_(orig)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, _, _, info = dp.sytrf_device(n, work, n, stream=stream)
        e1.record(stream)
        e1.synchronize()
        if st != 0:
            raise RuntimeError(f"dp_sytrf_device: status {st}")
        if i:
            ms.append(e0.elapsed_time(e1))
    del orig, work
    torch.cuda.empty_cache()
    t = statistics.mean(ms)
    out = {"n": n, "ms_per_factorisation": t, "gflops": sytrf_flops(n) / (t * 1e-3) / 1e9,
           "step_ms": [round(x, 3) for x in ms], "info": info,
           "records_check": sytrf_records_check(dp)}
    if cpu:
        threads = os.cpu_count() or 1
        gc, tc, kind, _ = cpu_sytrf_gflops(4096, 4096, threads)
        out["cpu_reference_n4096"] = {"gflops": gc, "seconds": tc, "kind": kind,
                                      "cores": threads}
    return out


def run_sytrf(args):
    import ctypes

    import torch
    import delayed_pivoting as dp

    world, rank, local, dev, dist = _dist_setup(torch)

    n = args.n
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + rank)
    # column-major storage; only the lower triangle is read
    orig = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
    work = torch.empty_like(orig)
    stream = torch.cuda.current_stream(dev)
    L = dp.lib()
    L.dp_stats_families.restype = ctypes.c_uint
    L.dp_stats_families.argtypes = [ctypes.c_uint]

    def step():
        work.copy_(orig)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, _, piv, info = dp.sytrf_device(n, work, n, nb=args.nb, stream=stream)
        e1.record(stream)
        if st != 0:
            raise RuntimeError(f"dp_sytrf_device: status {st}")
        return e0, e1, info, piv

    L.dp_stats_enable(1)  # warm-up also warms the library's event pool
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    L.dp_stats_enable(0)
    if dist:
        dist.barrier()
    # timed steps record the panel family only (the roofline kernel)
    L.dp_stats_reset()
    L.dp_stats_families(1 << 0)
    L.dp_stats_enable(1)
    events = []
    l0 = L.dp_kernel_launches()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        for _ in range(args.steps):
            events.append(step())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    launches = L.dp_kernel_launches() - l0
    L.dp_stats_enable(0)
    ms = sum(e0.elapsed_time(e1) for e0, e1, _, _ in events)
    info, piv = events[-1][2], events[-1][3]
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    stats = _stats(L)
    L.dp_stats_reset()
    L.dp_stats_families(0xFFFFFFFF)
    L.dp_stats_enable(1)
    step()
    torch.cuda.synchronize()
    L.dp_stats_enable(0)
    fam_stats = _stats(L)
    L.dp_stats_reset()

    e2e = None
    if not args.no_e2e:
        host = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        src = orig.cpu()
        k = max(1, min(args.steps, 3))
        e2e_s = 0.0
        for i in range(k + 1):
            host.copy_(src)
            hnp = host.numpy().T  # Fortran view of the pinned buffer
            t0 = time.perf_counter()
            st, _, _, _ = dp.sytrf_host(hnp)  # H2D, factorisation, D2H; synchronous
            if st != 0:
                raise RuntimeError(f"dp_sytrf_host: status {st}")
            if i:
                e2e_s += time.perf_counter() - t0
        e2e_ms = e2e_s / k * 1e3
        if dist:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": world * sytrf_flops(n) / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * n * 8 + 2 * n * 4,
               "ms_per_step": e2e_ms, "api": "dp_sytrf_host (delayed_sytrf_blocked drop-in)"}

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    pl = max(stats["launches"][0], 1)
    panel_avg_ms = stats["ms"][0] / pl
    panel_bytes = stats["bytes"][0] / pl
    achieved = panel_bytes / (panel_avg_ms * 1e-3) / 1e9 if panel_avg_ms > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": "bk_panel_kernel (cooperative, grid barrier per phase)",
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks.get("hbm_gbs")
                else "fallback 6650 GB/s (MEASURED_PEAKS.json absent)",
                "traffic": panel_bytes * BK_PANEL_DRAM_PER_ALGORITHMIC_BYTE,
                "traffic_source": "ncu dram__bytes of one n = 4096 panel launch "
                                  "(profiles/bk_panel_kernel_sytrf_n4096.md), scaled by the "
                                  "launch's algorithmic bytes",
                "algorithmic_bytes_per_launch": panel_bytes,
                "avg_launch_ms": panel_avg_ms, "launches_timed": stats["launches"][0],
                "note": "latency-bound: every pivot step is 2-3 grid barriers with a decision "
                        "between them; bytes are 32 per row per factored column"}
    fp64 = fp64_peak_tflops(torch, dev)
    value = world * sytrf_flops(n) * args.steps / (ms * 1e-3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        gc, tc, kind, _ = cpu_sytrf_gflops(args.cpu_n, args.seed, threads)
        cpu = {"value": gc, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"one delayed_sytrf_blocked of n={args.cpu_n} (seeded N(0,1) symmetric),"
                         f" {tc:.2f} s, OpenBLAS {threads} threads"}
        if kind == "reference":
            gl, tl, _, _ = cpu_sytrf_gflops(args.cpu_n, args.seed, threads, "lapack")
            cpu["lapack_dsytrf"] = {"value": gl, "unit": UNIT, "cores": threads,
                                    "sample": f"LAPACK dsytrf('L') + dsyconv through the "
                                              f"reference's lapack_sytrf, same n={args.cpu_n} "
                                              f"matrix, {tl:.2f} s"}
        n1 = max(256, args.cpu_n // 2)
        g1, t1, kind1, _ = cpu_sytrf_gflops(n1, args.seed, 1)
        cpu["one_thread"] = {"value": g1, "unit": UNIT, "cores": 1, "kind": kind1,
                             "sample": f"one delayed_sytrf_blocked of n={n1}, {t1:.2f} s"}
    if rank == 0:
        fam = ["panel", "laswp", "trsm", "gemm", "search", "swap", "other", "gemm_mixed"]
        kern = {}
        fs = fam_stats
        for i, nm in enumerate(fam):
            if fs["launches"][i] == 0:
                continue
            kern[nm] = {"ms_per_step": fs["ms"][i], "launches_per_step": fs["launches"][i],
                        "share": fs["ms"][i] / max(ms / args.steps, 1e-9)}
            if fs["flops"][i]:
                kern[nm]["tflops"] = fs["flops"][i] / (fs["ms"][i] * 1e-3) / 1e12
            if fs["bytes"][i]:
                kern[nm]["gbs"] = fs["bytes"][i] / (fs["ms"][i] * 1e-3) / 1e9
        upd = kern.get("gemm", {})
        line = {
            "metric": sytrf_metric(n), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: N(0,1) (torch Philox, seeded per rank), lower triangle read",
            "config": {"workload": f"delayed_sytrf_blocked n={n} (single matrix)", "n": n,
                       "nb": args.nb or 64, "parallelism": f"replicas x{world}", "info": info,
                       "pivots_2x2": int((piv == 2).sum()),
                       "l2": f"input {8 * n * n / 2**30:.2f} GiB " + (
                           "> L2 (no flush needed)" if 8 * n * n > 126e6 else "<= L2")},
            "roofline": roofline,
            "update_roofline": {"bound": "tensor", "kernel": "dgemm_minus_kernel lower (DMMA)",
                                "achieved": upd.get("tflops"), "peak": fp64, "unit": "TFLOP/s",
                                "frac": (upd.get("tflops") or 0.0) / fp64 if fp64 else None,
                                "peak_source": "cuBLAS DGEMM 8192^3 measured live"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "gpu_launches_per_step": launches / max(args.steps, 1),
            "step_ms": [round(e0.elapsed_time(e1), 3) for e0, e1, _, _ in events],
            "clocks": clk.summary(),
            "kernels": kern,
            "records_check": sytrf_records_check(dp),
            "fp64_peak_tflops": fp64,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def sytrf_reference_arm(args):
    """The reference's own delayed_sytrf_blocked on the host cores, each step a
    bounded sample (n = --cpu-n) of the n = --n workload, in GFLOP/s (n^3/3)."""
    threads = os.cpu_count() or 1
    n = args.cpu_n
    times, kind = [], None
    for i in range(args.warmup + args.steps):
        _, t, kind, _ = cpu_sytrf_gflops(n, args.seed, threads)
        if i >= args.warmup:
            times.append(t)
    tot = sum(times)
    value = sytrf_flops(n) * len(times) / tot / 1e9
    lapack = None
    if kind == "reference":
        gl, tl, _, _ = cpu_sytrf_gflops(n, args.seed, threads, "lapack")
        lapack = {"value": gl, "unit": UNIT, "cores": threads, "seconds": tl,
                  "sample": f"LAPACK dsytrf('L') + dsyconv through the reference's lapack_sytrf, "
                            f"n={n}"}
    line = {
        "impl": "reference", "metric": sytrf_metric(args.n), "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot / len(times) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: N(0,1) PCG64 seeded symmetric",
        "config": {"workload": f"delayed_sytrf_blocked n={args.n}", "sample_n": n,
                   "threads": threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"one delayed_sytrf_blocked of n={n} per step (bounded sample "
                                   f"of the n={args.n} workload), OpenBLAS {threads} threads",
                         "lapack_dsytrf": lapack},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- front ----

def front_metric(n, p):
    return (f"multifrontal front: partial delayed LU of an {n} x {n} front over its {p} "
            f"fully-summed rows / columns, GFLOP/s (partial-LU flops)")


def front_flops(m, n, k):
    """Multiply-adds x 2 of eliminating k pivots of an m x n front:
    sum_{j<k} 2 (m - j - 1)(n - j - 1), to leading order."""
    k = float(k)
    return 2.0 * (m * n * k - (m + n) * k * k / 2.0 + k ** 3 / 3.0)


def cpu_front_gflops(m, p, seed):
    """The C restatement of the path (oracle_front: the reference's
    delayed_getrf rules on the fully-summed block, NumPy for the rest; the
    reference itself has no code for the hand-off) on the host cores."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    rng = np.random.default_rng(seed)
    f = np.asfortranarray(rng.standard_normal((m, m)))
    t0 = time.perf_counter()
    k, _, _, _ = orc.oracle_front(f, p)
    t = time.perf_counter() - t0
    return front_flops(m, m, k) / t / 1e9, t


def run_front(args):
    """One multifrontal hand-off per step: dp_front_factor on an n x n front
    (N(0,1), torch Philox, seeded per rank) whose leading n / 2 rows and
    columns are fully summed; the contribution block is F(k:n, k:n)."""
    import torch
    import delayed_pivoting as dp

    world, rank, local, dev, dist = _dist_setup(torch)
    n = args.n
    p = n // 2
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + rank)
    orig = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)  # column-major front
    work = torch.empty_like(orig)
    stream = torch.cuda.current_stream(dev)
    L = dp.lib()

    def step():
        work.copy_(orig)
        rows = np.arange(n, dtype=np.int32)
        cols = np.arange(n, dtype=np.int32)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, k, _, _ = dp.front_factor(n, n, p, work, n, rows, cols, stream=stream)
        e1.record(stream)
        if st != 0:
            raise RuntimeError(f"dp_front_factor: status {st}")
        return e0, e1, k

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    events = []
    l0 = L.dp_kernel_launches()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        for _ in range(args.steps):
            events.append(step())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    launches = L.dp_kernel_launches() - l0
    ms = sum(e0.elapsed_time(e1) for e0, e1, _ in events)
    k = events[-1][2]
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    flops = front_flops(n, n, k)
    value = world * flops * args.steps / (ms * 1e-3) / 1e9

    e2e = None
    if not args.no_e2e:
        host = orig.cpu().pin_memory()
        back = torch.empty_like(host).pin_memory()
        kk = max(1, min(args.steps, 3))
        e2e_ms = 0.0
        for i in range(kk + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            work.copy_(host, non_blocking=True)
            st, _, _, _ = dp.front_factor(n, n, p, work, n, np.arange(n, dtype=np.int32),
                                          np.arange(n, dtype=np.int32), stream=stream)
            back.copy_(work, non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            if st != 0:
                raise RuntimeError(f"dp_front_factor: status {st}")
            if i:
                e2e_ms += e0.elapsed_time(e1)
        e2e_ms /= kk
        if dist:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": world * flops / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * n * 8,
               "ms_per_step": e2e_ms,
               "api": "dp_front_factor, the front copied from and back to pinned host memory"}
    fp64 = fp64_peak_tflops(torch, dev)
    achieved = value / world / 1e3
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        m1 = max(256, min(args.cpu_n, 4096) // 2)
        gc, tc = cpu_front_gflops(m1, m1 // 2, args.seed)
        cpu = {"value": gc, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"oracle_front (the C restatement of delayed_getrf on the fully-summed "
                         f"block, NumPy / OpenBLAS for the rest) on a {m1} x {m1} front with "
                         f"{m1 // 2} fully-summed rows, {tc:.2f} s"}
    if rank == 0:
        line = {
            "metric": front_metric(n, p), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: N(0,1) front (torch Philox, seeded per rank)",
            "config": {"workload": f"dp_front_factor n={n} p={p} (single front)", "n": n, "p": p,
                       "npiv": k, "parallelism": f"replicas x{world}",
                       "l2": f"front {8 * n * n / 2**30:.2f} GiB > L2 (no flush needed)"},
            "roofline": {"bound": "tensor", "kernel": "whole call (the DMMA Schur update "
                         "dominates: partial-LU flops over the call's time)",
                         "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                         "frac": achieved / fp64 if fp64 else None, "traffic": None,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured live"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "step_ms": [round(e0.elapsed_time(e1), 3) for e0, e1, _ in events],
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def front_reference_arm(args):
    print(json.dumps({"impl": "reference", "unavailable": "the reference has no code for the "
                      "multifrontal hand-off (its design document describes it, "
                      "doc/...LU方法.md:228-457)"}, ensure_ascii=False), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
