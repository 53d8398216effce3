#!/usr/bin/env python
"""Benchmark: GP fit + predict-with-uncertainty on one B200 per rank.

Workload (default "c2"): n_train=32768, n_test=8192, n_regressors=64,
lengthscale=4.0, vertical_lengthscale=1.0, noise_variance=0.01, seeded
synthetic series (x ~ N(0,1), y_i = sum_j sin(X_ij)/8 + N(0, 0.01^2)).
One step = SE assembly of K + Cholesky + alpha solves + predictive mean
(cross covariance . alpha) + per-point variance (K* L^-T row sums), all in
FP64 unless --precision selects a mixed mode.  K alone is 8.6 GB (> L2), so
no L2 flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints ONE JSON line (rank 0).  Multi-GPU runs (torchrun) are replicas: each
rank fits and predicts its own copy (the factorisation does not shard), the
step time is the max over ranks, and `value` is that time / N (aggregate
seconds per fit+predict job).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fit+predict s @n=32768, mixed vs FP64 GPU at <=1e-8 rel err; serve p50/p99 ms"

WORKLOADS = {
    # name: n_train, n_test, n_regressors, tile, hyper
    "c2": dict(n=32768, m=8192, d=64, T=1024, hyper=(4.0, 1.0, 0.01)),
    "c1": dict(n=16384, m=4096, d=8, T=512, hyper=(1.0, 1.0, 0.1)),
}

# Bounded CPU sample of the same workload: same d, hyper-parameters and
# n_test/n_train ratio; time scales with n^3 (n^3/3 Cholesky + n^2 m solve).
CPU_SAMPLE_N = 8192


def algorithmic_flops(n: int, m: int) -> float:
    """fit+predict_var (excluding assembly): n^3/3 + 2n^2 + n^2 m + 2nm."""
    return n ** 3 / 3 + 2 * n ** 2 + n ** 2 * m + 2 * n * m


def synthetic(n, m, d):
    from oracle import gprat_oracle as O  # input generator only (seeded numpy)

    return O.synthetic(n, m, d)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if getattr(self, "out", None):
            self.out.close()

    def summary(self):
        if self.proc is None or self.path is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def measure_fp64_gemm_peak(torch, device) -> float:
    """cuBLAS DGEMM throughput (torch.matmul fp64 8192^3, best of 5), TF/s:
    the FP64 counterpart of the driver's bf16 GEMM peak."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) / 1e3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def cpu_reference_sample(wl, reps: int):
    """The reference's own CPU path (compiled from source, oracle/_ref) on a
    bounded sample: n=8192 with the workload's d, hyper-parameters and
    n_test/n_train ratio.  Returns (seconds per rep, scale factor to the
    full workload, description, threads)."""
    from oracle import ref

    n, d = CPU_SAMPLE_N, wl["d"]
    m = wl["m"] * n // wl["n"]
    T = 512
    threads = os.cpu_count() or 1
    ref.start(threads)
    x, y, xt = synthetic(n, m, d)
    gp = ref.RefGP(x, y, n // T, T, d, wl["hyper"])
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        gp.predict_with_uncertainty(xt, m // T, T)
        times.append(time.perf_counter() - t0)
    scale = algorithmic_flops(wl["n"], wl["m"]) / algorithmic_flops(n, m)
    desc = (f"reference CPU predict_with_uncertainty (assembly+Cholesky+solves+mean+var), n_train={n}, "
            f"n_test={m}, d={d}, {n // T}x{n // T} tiles of {T}; median of {reps}; scaled x{scale:.0f} by "
            f"algorithmic flops to n_train={wl['n']}, n_test={wl['m']}; HPX replaced by std::thread shim, "
            f"OpenBLAS 0.3.30 single-threaded per task")
    return statistics.median(times), scale, desc, threads


def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    for _ in range(args.warmup):
        pass  # warm-up happens inside cpu_reference_sample's first rep
    sample_s, scale, desc, threads = cpu_reference_sample(wl, max(args.steps, 1))
    value = sample_s * scale
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(wl, "fp64"),
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_of(wl, precision):
    return {"workload": f"GP fit+predict_with_uncertainty n_train={wl['n']} n_test={wl['m']} "
                        f"n_regressors={wl['d']}", "n_train": wl["n"], "n_test": wl["m"], "n_regressors": wl["d"],
            "tile": wl["T"], "hyper": list(wl["hyper"]), "precision": precision,
            "l2": "inputs larger than L2 (K alone is %.1f GB)" % (wl["n"] ** 2 * 8 / 1e9),
            "parallelism": "replicas"}


def run_ours(args, wl):
    import torch
    import torch.distributed as dist

    from gprat_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    n, m, d, T, hyper = wl["n"], wl["m"], wl["d"], wl["T"], wl["hyper"]
    x, y, xt = synthetic(n, m, d)
    gp = capi.CudaGP(x, y, n // T, T, d, device=local)
    precision = {"fp64": capi.PREC_FP64, "mixed-tf32": capi.PREC_MIXED_TF32,
                 "mixed-bf16": capi.PREC_MIXED_BF16}[args.precision]
    gp.set_precision(precision)

    dxt = torch.tensor(xt, device=device)
    dmean = torch.empty(m, dtype=torch.float64, device=device)
    dvar = torch.empty(m, dtype=torch.float64, device=device)
    stream = torch.cuda.current_stream(device)

    def step():
        gp.fit_predict_device(hyper, dxt.data_ptr(), dxt.numel(), m, dmean.data_ptr(), dvar.data_ptr(),
                              stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    gp.check_status()

    def barrier():
        if world > 1:
            dist.barrier()

    capi.stats_reset()
    capi.stats_enable_timing(True)
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
        barrier()
    capi.stats_enable_timing(False)
    stats = capi.stats_read()
    gp.check_status()
    elapsed_ms = start.elapsed_time(end)
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps

    mean_h, var_h = dmean.cpu().numpy(), dvar.cpu().numpy()
    sane = bool(np.all(np.isfinite(mean_h)) and np.all(var_h > 0) and np.all(var_h <= hyper[1] + 1e-12))
    if args.profile:
        print(json.dumps({"profile_run": True, "ms_per_step": ms_per_step, "gpu_launches": int(stats["launches"]),
                          "sanity": sane}), flush=True)
        return

    # end-to-end through the C ABI with host buffers (H2D of the test series,
    # D2H of mean and variance inside every call)
    xt_pinned = torch.tensor(xt, dtype=torch.float64).pin_memory().numpy()
    gp.predict_with_uncertainty(hyper, xt_pinned, 1, m)
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        gp.predict_with_uncertainty(hyper, xt_pinned, 1, m)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_times))

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    peaks = measured_peaks()
    fp64_peak = measure_fp64_gemm_peak(torch, device)
    gemm_tflops = stats["gemm_flops"] / (stats["gemm_ms"] / 1e3) / 1e12 if stats["gemm_ms"] > 0 else None
    step_flops = algorithmic_flops(n, m)
    if world == 1 and not args.skip_cpu_baseline:
        sample_s, scale, desc, threads = cpu_reference_sample(wl, 3)
        cpu = {"value": sample_s * scale, "unit": "s", "cores": threads, "kind": "reference", "sample": desc}
    else:
        cpu = None
    clk = clocks.summary()
    line = {
        "metric": METRIC,
        "value": ms_per_step / 1e3 / world,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else args.precision,
        "data": "synthetic",
        "config": config_of(wl, args.precision),
        "pipeline_tflops": step_flops / (ms_per_step / 1e3) / 1e12,
        "roofline": {
            "kernel": "dgemm_kernel (FP64 DMMA m16n8k8: Cholesky panel/trailing updates + variance solve)",
            "bound": "tensor",
            "achieved": gemm_tflops,
            "peak": fp64_peak,
            "peak_source": "cuBLAS DGEMM (torch.matmul fp64 8192^3, best of 5) measured in this run; "
                           "MEASURED_PEAKS.json holds no FP64 figure",
            "unit": "TFLOP/s",
            "frac": (gemm_tflops / fp64_peak) if gemm_tflops else None,
            "traffic": None,
            "gemm_share_of_step": (stats["gemm_ms"] / args.steps) / ms_per_step,
            "gemm_launches_per_step": stats["gemm_launches"] / args.steps,
        },
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int((m + d - 1) * 8),
                "d2h_bytes_per_step": int(2 * m * 8)},
        "gpu_launches": int(stats["launches"]),
        "clocks": clk,
        "hbm_peak_gbs": peaks.get("hbm_gbs"),
        "pcg_iterations": gp.pcg_iterations(),
        "sanity": sane,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--precision", choices=["fp64", "mixed-tf32", "mixed-bf16"], default="fp64")
    ap.add_argument("--skip-cpu-baseline", action="store_true",
                    help="omit the CPU reference sample (cpu_baseline becomes null)")
    ap.add_argument("--profile", action="store_true",
                    help="device steps only (no CPU sample, e2e loop or peak measurement): for ncu captures")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl)
    else:
        run_ours(args, wl)


if __name__ == "__main__":
    main()
