"""Benchmark of the B200 delayed-pivoting LU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--n 16384]

One step = one plain-FP64 delayed_getrf of an n x n N(0,1) matrix with
0.1 % tiny (x1e-18) and 0.02 % exact-zero columns (n = 16384: 16 + 3), the
single-GPU configuration of the reference's plain path.  Inputs are
generated once (seeded MT19937-64), kept resident in HBM, and restored by a
device copy before every step, outside the timed region; the 2 GiB matrix is
larger than L2, so no flush is needed between steps.  Throughput is
2/3 n^3 / t in GFLOP/s (delayed_lu_cuda/benchmark.cu:67).

Rank 0 prints one JSON line.  With N > 1 (torchrun) each rank factors its own
matrix (replicas: a single LU does not shard) and `value` is the sum over
ranks divided by the slowest rank's time.
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

METRIC = "plain FP64 delayed_getrf GFLOP/s (2/3 n^3), n=16384, 0.1% tiny + 0.02% zero columns"
UNIT = "GFLOP/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--nb", type=int, default=64)
    ap.add_argument("--seed", type=int, default=16384)
    ap.add_argument("--cpu-n", type=int, default=8192, help="CPU baseline sample size")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="trailing-update arithmetic of the factorisation")
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


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
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
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
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

    import torch
    import delayed_pivoting as dp

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
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)

    n = args.n
    w = workload(n)
    a = dp.planted_matrix(n, n, args.seed + rank, w["n_tiny"], w["n_zero"])
    orig = torch.from_numpy(a.T.copy()).to(dev)  # column-major n x n
    work = torch.empty_like(orig)
    ipiv = np.zeros(n, dtype=np.int32)
    jpiv = np.zeros(n, dtype=np.int32)
    stream = torch.cuda.current_stream(dev)
    L = dp.lib()
    prec = dp.PRECISION_MIXED_BF16X3 if args.precision == "mixed" else dp.PRECISION_FP64

    def step(timed_events=None):
        work.copy_(orig)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, info = dp.getrf_device_ex(n, n, work, n, ipiv, jpiv, stream=stream, nb=args.nb,
                                      precision=prec)
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

    L.dp_stats_reset()
    L.dp_stats_enable(1)
    events = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        for _ in range(args.steps):
            events.append(step())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    L.dp_stats_enable(0)
    ms = sum(e0.elapsed_time(e1) for e0, e1, _ in events)
    info = events[-1][2]
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    stats = _stats(L)
    launches_per_step = sum(stats["launches"]) / max(args.steps, 1)

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
    g = 3  # DP_KFAM_GEMM
    gemm_ms = stats["ms"][g]
    gemm_tf = stats["flops"][g] / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else 0.0
    roofline = {"bound": "tensor", "kernel": "dgemm_minus_kernel (FP64 DMMA m16n8k4)",
                "achieved": gemm_tf, "peak": fp64, "unit": "TFLOP/s",
                "frac": gemm_tf / fp64 if fp64 else None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured live (FP64 is not in MEASURED_PEAKS.json)",
                "traffic": None,
                "per_launch_flops": stats["flops"][g] / max(stats["launches"][g], 1),
                "avg_launch_ms": gemm_ms / max(stats["launches"][g], 1)}

    value = world * flops(n) * args.steps / (ms * 1e-3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        g_cpu, t_cpu, kind, cinfo = cpu_reference_gflops(args.cpu_n, args.seed, threads)
        cpu = {"value": g_cpu, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"one delayed_getrf of n={args.cpu_n} (same generator, 0.1%/0.02% "
                         f"planted columns), {t_cpu:.2f} s, OpenBLAS {threads} threads"}
    if rank == 0:
        fam = ["panel", "laswp", "trsm", "gemm", "search", "swap", "other", "gemm_mixed"]
        kern = {}
        for i, nm in enumerate(fam):
            if stats["launches"][i] == 0:
                continue
            t = stats["ms"][i] / args.steps
            kern[nm] = {"ms_per_step": t, "launches_per_step": stats["launches"][i] / args.steps,
                        "share": stats["ms"][i] / max(ms / world, 1e-9)}
            if stats["flops"][i]:
                kern[nm]["tflops"] = stats["flops"][i] / (stats["ms"][i] * 1e-3) / 1e12
            if stats["bytes"][i]:
                kern[nm]["gbs"] = stats["bytes"][i] / (stats["ms"][i] * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: N(0,1) MT19937-64 seeded per rank, 16 tiny (x1e-18) + 3 zero columns",
            "config": {"workload": f"delayed_getrf plain FP64 n={n} (single matrix)", "n": n,
                       "nb": args.nb, "parallelism": f"replicas x{world}",
                       "l2": "input 2 GiB > L2 (no flush needed)", "info": info},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "gpu_launches_per_step": launches_per_step,
            "clocks": clk.summary(),
            "kernels": kern,
            "fp64_peak_tflops": fp64,
            "frac_of_fp64_peak": value / world / 1e3 / fp64,
            "hbm_peak_gbs": peaks.get("hbm_gbs"),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


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


if __name__ == "__main__":
    sys.exit(main())
