#!/usr/bin/env python
"""Benchmark: GP fit + predict-with-uncertainty on one B200 per rank.

Workload (default "c2"): n_train=32768, n_test=8192, n_regressors=64,
lengthscale=4.0, vertical_lengthscale=1.0, noise_variance=0.01, seeded
synthetic series (x ~ N(0,1), y_i = sum_j sin(X_ij)/8 + N(0, 0.01^2)).
One step = SE assembly of K + Cholesky + alpha solves + predictive mean
(cross covariance . alpha) + per-point variance (K* L^-T row sums).  The
default precision is fp64-int8: every product of the factorisation and of
the variance solve emulated in FP64 on the int8 tensor cores (5 digit
planes), FP64 diagonal blocks and triangular solves.  The same run times the
plain FP64 path on the same inputs ("fp64") and reports the headline mode's
error against it, times the other modes ("arms": 5 planes with 4 digit
groups in every product, 4 and 7 planes, TF32, BF16) with their errors, and runs the serving stream ("serving": four
resident models, Poisson requests, p50/p99 latency).  K alone is 8.6 GB
(> L2), so no L2 flush is needed between steps.

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

# Per-call CPU and GPU timings of the API calls (cholesky, predict,
# calculate_loss, optimize_step) are taken at this smaller training size.
CPU_SAMPLE_N = 8192


def algorithmic_flops(n: int, m: int) -> float:
    """fit+predict_var (excluding assembly): n^3/3 + 2n^2 + n^2 m + 2nm."""
    return n ** 3 / 3 + 2 * n ** 2 + n ** 2 * m + 2 * n * m


def synthetic(n, m, d):
    from oracle import gprat_oracle as O  # input generator only (seeded numpy)

    return O.synthetic(n, m, d)


class ClockSampler:
    """SM clocks and clock-event reasons of the bench's GPU, sampled DURING the
    timed region. NVML is read from a thread every 10 ms (read-only queries; the
    device is found by its UUID, so CUDA_VISIBLE_DEVICES remapping cannot point
    the sampler at another GPU). Without NVML the fallback is `nvidia-smi -lms 200`,
    started early enough that its first sample exists before timing begins."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.device)
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))
        except Exception:
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _poll(self, nv, h):
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), [self.NAMES[i] for i, b in enumerate(bits) if r & b]))
            except Exception:
                pass
            self.stop.wait(0.01)

    def __enter__(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            self.source = "nvml 10 ms"
            return self
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi 200 ms"
            t0 = time.time()
            while time.time() - t0 < 10 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if getattr(self, "out", None):
            self.out.close()

    def summary(self):
        if self.thread is None:
            if self.proc is None or self.path is None:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
            with open(self.path) as f:
                for line in f:
                    p = [x.strip() for x in line.split(",")]
                    if len(p) >= 9 and p[1].replace(".", "").isdigit():
                        mx = float(p[2]) if p[2].replace(".", "").isdigit() else None
                        self.rows.append((float(p[1]), mx,
                                          [self.NAMES[i] for i in range(4) if p[5 + i].lower() == "active"]))
            os.unlink(self.path)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0,
                    "source": self.source}
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows if r[1] is not None]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted({n for r in self.rows for n in r[2]}), "samples": len(self.rows),
                "source": self.source}


def max_over_ranks(value: float, dist, device) -> float:
    """The step time of a multi-GPU run: the maximum over all ranks (every rank
    calls this, in the same order, like every collective)."""
    import torch

    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_seconds(ms_per_step: float, world: int) -> float:
    """Whole-job seconds per fit+predict job: N replicas finish N jobs per step."""
    return ms_per_step / 1e3 / world


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def measure_gemm_peak(torch, device, dtype) -> float:
    """cuBLAS GEMM throughput (torch.matmul 8192^3, best of 5), TF/s; fp32
    inputs run as TF32 (allow_tf32)."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(8192, 8192, dtype=dtype, device=device)
    b = torch.randn(8192, 8192, dtype=dtype, device=device)
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
    torch.backends.cuda.matmul.allow_tf32 = old
    return best


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


def measure_int8_peak(torch, device) -> float:
    """cuBLASLt int8 GEMM throughput (torch._int_mm, int8 x int8 -> int32,
    8192^3, best of 5), tera-ops/s."""
    a = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device=device)
    b = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device=device)
    torch._int_mm(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) / 1e3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def cpu_reference_full(wl, reps: int):
    """The reference's own CPU path (compiled from source, oracle/_ref) at the
    FULL workload on all host cores: `reps` timed predict_with_uncertainty
    calls (assembly + Cholesky + alpha solves + mean + variance), after one
    small untimed call that starts the task pool and pages the libraries in.
    Returns (seconds of each rep, description, threads)."""
    from oracle import ref

    n, m, d, T = wl["n"], wl["m"], wl["d"], wl["T"]
    threads = os.cpu_count() or 1
    ref.start(threads)
    xw, yw, xtw = synthetic(1024, 256, d)
    ref.RefGP(xw, yw, 8, 128, d, wl["hyper"]).predict_with_uncertainty(xtw, 2, 128)
    x, y, xt = synthetic(n, m, d)
    nt = n // T
    mt, mts = ref.compute_test_tiles(m, nt, T)
    gp = ref.RefGP(x, y, nt, T, d, wl["hyper"])
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        gp.predict_with_uncertainty(xt, mt, mts)
        times.append(time.perf_counter() - t0)
    desc = (f"reference CPU predict_with_uncertainty (assembly+Cholesky+solves+mean+var) at the full workload "
            f"n_train={n}, n_test={m}, d={d}, {nt}x{nt} tiles of {T}; {reps} timed call(s) after one small "
            f"untimed warm-up call (n_train=1024); HPX replaced by a std::thread shim, OpenBLAS 0.3.30 "
            f"single-threaded per task, {threads} threads")
    return times, desc, threads


def cpu_reference_calls(wl, reps: int = 3):
    """Wall time of the reference's CPU API calls (compiled from source,
    oracle/_ref, all host cores) at the bounded sample size n_train=8192 with
    the workload's d and hyper-parameters: cholesky, predict_with_uncertainty,
    calculate_loss (median of reps) and one optimize_step."""
    from oracle import ref

    n, d, T = CPU_SAMPLE_N, wl["d"], 512
    m = wl["m"] * n // wl["n"]
    ref.start(os.cpu_count() or 1)
    x, y, xt = synthetic(n, m, d)
    gp = ref.RefGP(x, y, n // T, T, d, wl["hyper"])

    def med(f, r):
        ts = []
        for _ in range(r):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts)

    return {
        "n_train": n, "n_test": m, "n_regressors": d, "tile": T,
        "cholesky_s": med(gp.cholesky, reps),
        "predict_with_uncertainty_s": med(lambda: gp.predict_with_uncertainty(xt, m // T, T), reps),
        "calculate_loss_s": med(gp.calculate_loss, reps),
        "optimize_step_s": med(lambda: gp.optimize_step(0, 0.1, 0.9, 0.999, 1e-8), 1),
    }


# Hyper-parameter optimisation at its own configuration (the adjoint path):
# n_train=8192, d=8, initial (lengthscale, vertical lengthscale, noise) =
# (0.5, 2.0, 0.5), 50 Adam steps at lr=0.1, beta1=0.9, beta2=0.999, FP64.
C3 = dict(n=8192, d=8, T=512, theta0=(0.5, 2.0, 0.5), steps=50, adam=(0.1, 0.9, 0.999, 1e-8))


def c3_optimize(reference: bool):
    """The 50 Adam steps timed whole: this library's gprat_cu_optimize (one
    call, every step on the GPU) and, if `reference`, the reference's own
    CPU optimize (compiled from source, oracle/_ref) on all host cores."""
    from gprat_b200 import capi

    c = C3
    x, y, _ = synthetic(c["n"], 16, c["d"])
    gp = capi.CudaGP(x, y, c["n"] // c["T"], c["T"], c["d"])
    params = np.array(list(c["theta0"]) + [0.0] * 6)
    gp.optimize(params.copy(), list(c["adam"]), [1, 1, 1], 1)  # untimed: pages the kernels in
    t0 = time.perf_counter()
    losses, final = gp.optimize(params.copy(), list(c["adam"]), [1, 1, 1], c["steps"])
    ours = time.perf_counter() - t0
    gp.close()
    out = {"config": "n_train=8192 n_regressors=8 theta0=(0.5, 2.0, 0.5), 50 Adam steps lr=0.1 b1=0.9 b2=0.999",
           "ours_s": ours, "ours_final_loss": float(losses[-1]), "ours_final_theta": [float(v) for v in final[:3]]}
    if reference:
        from oracle import ref

        threads = os.cpu_count() or 1
        ref.start(threads)
        g = ref.RefGP(x, y, c["n"] // c["T"], c["T"], c["d"], c["theta0"])
        lr, b1, b2, eps = c["adam"]
        t0 = time.perf_counter()
        rl = g.optimize(lr, b1, b2, eps, c["steps"])
        out.update({"reference_s": time.perf_counter() - t0, "reference_cores": threads,
                    "reference_final_loss": float(rl[-1]),
                    "final_loss_rel_diff": abs(float(losses[-1]) - float(rl[-1])) / abs(float(rl[-1]))})
    return out


def gpu_calls(wl, mode, reps: int = 3):
    """The same calls through this library's C ABI (host buffers, synchronous),
    at the same sample size as cpu_reference_calls."""
    from gprat_b200 import capi

    n, d, T = CPU_SAMPLE_N, wl["d"], 512
    m = wl["m"] * n // wl["n"]
    x, y, xt = synthetic(n, m, d)
    gp = capi.CudaGP(x, y, n // T, T, d)
    if isinstance(mode, str):
        set_mode(gp, mode)
        precision = PRECISIONS[mode][0]
    else:
        precision = mode
        gp.set_precision(precision)
    h = wl["hyper"]
    params = np.array(list(h) + [0.0] * 6)

    def med(f, r):
        f()
        ts = []
        for _ in range(r):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts)

    out = {
        "predict_with_uncertainty_s": med(lambda: gp.predict_with_uncertainty(h, xt, m // T, T), reps),
        "calculate_loss_s": med(lambda: gp.compute_loss(h), reps),
    }
    if precision == capi.PREC_FP64:
        out["cholesky_s"] = med(lambda: gp.cholesky(h), reps)
        out["optimize_step_s"] = med(lambda: gp.optimize_step(params.copy(), [0.1, 0.9, 0.999, 1e-8], [1, 1, 1], 0),
                                     reps)
    gp.close()
    return out


def cusolver_fp64_comparator(torch, device, wl):
    """FP64 library comparator: the same fit+predict_with_uncertainty written
    with torch's FP64 linear algebra on the GPU (cdist, cuSOLVER Cholesky,
    triangular solves), device-timed with CUDA events (best of 2)."""
    n, m, d, hyper = wl["n"], wl["m"], wl["d"], wl["hyper"]
    x, y, xt = synthetic(n, m, d)
    X = torch.tensor(x, dtype=torch.float64, device=device).unfold(0, d, 1)[:n]
    Xt = torch.tensor(xt, dtype=torch.float64, device=device).unfold(0, d, 1)[:m]
    yy = torch.tensor(y[:n], dtype=torch.float64, device=device)
    l, v, noise = hyper

    def step():
        K = v * torch.exp(-0.5 / l ** 2 * torch.cdist(X, X).square_())
        K.diagonal().add_(noise)
        L = torch.linalg.cholesky(K)
        del K
        alpha = torch.cholesky_solve(yy.unsqueeze(1), L)
        Ks = v * torch.exp(-0.5 / l ** 2 * torch.cdist(Xt, X).square_())
        mean = Ks @ alpha
        V = torch.linalg.solve_triangular(L, Ks.T, upper=False)
        var = v - V.square().sum(0)
        return mean, var

    best = float("inf")
    for _ in range(2):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        step()
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    torch.cuda.empty_cache()
    return {"value": best / 1e3, "unit": "s",
            "what": "torch FP64 on the GPU: cdist + exp assembly, torch.linalg.cholesky (cuSOLVER), cholesky_solve, "
                    "solve_triangular for the variance; same inputs; best of 2"}


# Full-size calls the reference arm times (one C2 call is about 30 s on 16
# host cores, so the requested --steps are not all run at full size).
REF_FULL_REPS = 2


def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    reps = min(max(args.steps, 1), REF_FULL_REPS)
    times, desc, threads = cpu_reference_full(wl, reps)
    value = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": reps, "warmup": 1, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(wl),
        "seconds_per_call": times,
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_of(wl):
    return {"workload": f"GP fit+predict_with_uncertainty n_train={wl['n']} n_test={wl['m']} "
                        f"n_regressors={wl['d']}", "n_train": wl["n"], "n_test": wl["m"], "n_regressors": wl["d"],
            "tile": wl["T"], "hyper": list(wl["hyper"]),
            "l2": "inputs larger than L2 (K alone is %.1f GB)" % (wl["n"] ** 2 * 8 / 1e9),
            "parallelism": "replicas"}


# name: (GPRAT_CU_PREC_*, int8 digit planes or 0 for the library default,
#        int8 digit groups kept in every product or 0 for all)
PRECISIONS = {"fp64": (0, 0, 0), "mixed-tf32": (1, 0, 0), "mixed-bf16": (2, 0, 0), "fp64-int8": (3, 0, 0),
              "fp64-int8-4": (3, 4, 0), "fp64-int8-6": (3, 6, 0), "fp64-int8-7": (3, 7, 0),
              "fp64-int8-5g4": (3, 5, 4)}
# modes timed beside the headline one (besides FP64, which every run times)
ARM_ORDER = ("fp64-int8", "fp64-int8-5g4", "fp64-int8-4", "fp64-int8-7", "mixed-tf32", "mixed-bf16")


DEFAULT_SLICES = 5  # the library's default digit-plane count


def set_mode(gp, name, slices_override=0):
    prec, slices, groups = PRECISIONS[name]
    gp.set_precision(prec)
    if prec == 3:
        gp.set_int8_slices(slices_override or slices or DEFAULT_SLICES)
        gp.set_int8_groups(groups, groups)

# DRAM traffic of one representative launch of the dominant kernel, from an
# ncu capture (dram__bytes_read.sum + dram__bytes_write.sum); the live
# roofline above aggregates every GEMM launch of the step, so the per-launch
# traffic is quoted from the capture instead of being measured in this run.
TRAFFIC_SAMPLE = {
    "fp64-int8": {
        "launch": "oz_gemm_kernel, every launch of one fit+predict step at n_train=32768, 5 digit planes "
                  "(1035 launches, 1-pass ncu launch list); per-launch mean below; largest launch (variance top "
                  "update 8192 x 16384 x 16384): 35.86 GB DRAM against 4.1 GB algorithmic",
        "dram_bytes": 208.86e9 / 1035,
        "dram_bytes_step": 208.86e9,
        "workload": "c2",
        "source": "profiles/launch_list_fit_predict_c2_fp64_int8.md",
    },
    "mixed-tf32": {
        "launch": "tc_gemm_pair_kernel<TF32>, trailing update after panel 0 at n_train=16384: "
                  "lower 14336 x 14336, K=1024, 51 CTA pairs",
        "dram_bytes": 587.0e6 + 378.9e6,
        "algorithmic_bytes": 2 * 14336 * 14337 / 2 * 4 + 14336 * 1024 * 4,
        "source": "profiles/tc_gemm_trailing_update_c1.md",
    },
    "fp64": {
        "launch": "dgemm_kernel<2,0,1>, trailing update after the first outer panel at n_train=16384: "
                  "lower 15872 x 15872, K=512",
        "dram_bytes": 2.524e9 + 0.986e9,
        "algorithmic_bytes": 2 * 15872 * 15873 / 2 * 8 + 15872 * 512 * 8,
        "source": "profiles/dgemm_trailing_update_c1.md",
    },
}

# Serving stream (resident models n in SERVE_MODELS, d=8, Poisson arrivals):
# 90 % predict_with_uncertainty with m log-uniform in [1, 8192] on a uniformly
# chosen model, 10 % fits with n log-uniform in [1024, 16384] (rounded to 128).
SERVE_MODELS = (2048, 8192, 16384, 32768)
SERVE_REQUESTS = 200
SERVE_RATE = 40.0  # requests per second


def time_device_steps(torch, gp, hyper, dxt, m, dmean, dvar, stream, steps, warmup, barrier, local,
                      instrumented=True):
    """Device-timed fit+predict steps (CUDA events on the launching stream).

    Two timed regions of `steps` steps each: the first one plain (its time is
    the step time reported), the second one with the library's per-GEMM CUDA
    events on (their durations and flops give the tensor-core GEMM's achieved
    rate; recording an event around every GEMM also separates launches that
    would otherwise overlap, so that region's wall time is not reported)."""
    from gprat_b200 import capi

    def step():
        gp.fit_predict_device(hyper, dxt.data_ptr(), dxt.numel(), m, dmean.data_ptr(), dvar.data_ptr(),
                              stream.cuda_stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    gp.check_status()
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
        barrier()
    gp.check_status()
    elapsed = start.elapsed_time(end)
    if not instrumented:
        return elapsed, {"launches": 0, "gemm_launches": 0, "gemm_ms": 0.0, "gemm_flops": 0.0}, clocks.summary()
    # instrumented region: one step first fills the library's event pool
    capi.stats_enable_timing(True)
    step()
    torch.cuda.synchronize()
    capi.stats_read()
    capi.stats_reset()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    capi.stats_enable_timing(False)
    stats = capi.stats_read()
    gp.check_status()
    return elapsed, stats, clocks.summary()


def serving_bench(precision: int, seed: int = 7):
    """Runs the serving stream against a fresh server; returns latency and
    throughput figures (device 0 / the current device)."""
    from gprat_b200 import serving
    from oracle import gprat_oracle as O  # input generator only (seeded numpy)

    d, hyper, T = 8, (1.0, 1.0, 0.1), 512
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(SERVE_REQUESTS):
        if rng.random() < 0.1:
            nf = max(1024, int(np.exp(rng.uniform(np.log(1024), np.log(16384)))) // 128 * 128)
            xf, yf, _ = O.synthetic(nf, 16, d, seeds=(1000 + i, 2000 + i, 3000 + i))
            reqs.append(("fit", xf, yf, nf))
        else:
            m = int(np.exp(rng.uniform(0.0, np.log(8192))))
            reqs.append(("predict", int(rng.integers(0, len(SERVE_MODELS))), rng.standard_normal(m + d - 1), m))
    gaps = rng.exponential(1.0 / SERVE_RATE, SERVE_REQUESTS)
    with serving.Server(precision=precision) as sv:
        t0 = time.perf_counter()
        mids = []
        for n in SERVE_MODELS:
            x, y, _ = O.synthetic(n, 16, d, seeds=(n, n + 1, n + 2))
            mids.append(sv.add_model(x, y, n // T, T, d, hyper))
        setup_s = time.perf_counter() - t0
        for mid in mids:  # warm-up: size the batch buffers of every model
            sv.wait(sv.submit_predict(mid, rng.standard_normal(8192 + d - 1), 8192))
        ids, kinds, sizes, t_sub = [], [], [], []
        t_start = time.perf_counter()
        t_next = t_start
        for (kind, *rest), gap in zip(reqs, gaps):
            t_next += gap
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            t_sub.append(time.perf_counter())
            if kind == "fit":
                xf, yf, nf = rest
                ids.append(sv.submit_fit(xf, yf, nf // 128, 128, d, hyper))
                sizes.append(nf)
            else:
                mi, series, m = rest
                ids.append(sv.submit_predict(mids[mi], series, m))
                sizes.append(m)
            kinds.append(kind)
        lat_p, lat_f, t_done = [], [], []
        for rid, kind, ts in zip(ids, kinds, t_sub):
            _, _, _, lat = sv.wait(rid)
            (lat_f if kind == "fit" else lat_p).append(lat)
            t_done.append(ts + lat / 1e3)
        wall = max(t_done) - t_start
        st = sv.stats()
        # capacity: the same kind of stream submitted all at once
        burst = []
        for _ in range(SERVE_REQUESTS):
            m = int(np.exp(rng.uniform(0.0, np.log(8192))))
            burst.append((mids[int(rng.integers(0, len(SERVE_MODELS)))], rng.standard_normal(m + d - 1), m))
        t0 = time.perf_counter()
        bids = [sv.submit_predict(mid, series, m) for mid, series, m in burst]
        for rid in bids:
            sv.wait(rid)
        burst_wall = time.perf_counter() - t0
    points = sum(sz for sz, k in zip(sizes, kinds) if k == "predict")
    return {
        "requests": SERVE_REQUESTS, "rate_per_s": SERVE_RATE,
        "predict_p50_ms": float(np.percentile(lat_p, 50)), "predict_p99_ms": float(np.percentile(lat_p, 99)),
        "fit_p50_ms": float(np.percentile(lat_f, 50)) if lat_f else None,
        "fit_p99_ms": float(np.percentile(lat_f, 99)) if lat_f else None,
        "predictions_per_s": points / wall, "predict_requests": len(lat_p), "fit_requests": len(lat_f),
        "batches": st.batches, "model_setup_s": setup_s,
        "saturated_predictions_per_s": sum(b[2] for b in burst) / burst_wall,
        "saturated_requests": len(burst),
    }


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

    def barrier():
        if world > 1:
            dist.barrier()

    n, m, d, T, hyper = wl["n"], wl["m"], wl["d"], wl["T"], wl["hyper"]
    x, y, xt = synthetic(n, m, d)
    gp = capi.CudaGP(x, y, n // T, T, d, device=local)
    set_mode(gp, args.precision, args.slices)

    dxt = torch.tensor(xt, device=device)
    dmean = torch.empty(m, dtype=torch.float64, device=device)
    dvar = torch.empty(m, dtype=torch.float64, device=device)
    stream = torch.cuda.current_stream(device)

    elapsed_ms, stats, clk = time_device_steps(torch, gp, hyper, dxt, m, dmean, dvar, stream, args.steps,
                                               args.warmup, barrier, local)
    ms_per_step = max_over_ranks(elapsed_ms, dist if world > 1 else None, device) / args.steps

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
    # per-phase device time of one more call (step timers; not part of the timed region)
    capi.steps_reset()
    capi.steps_enable(True)
    gp.predict_with_uncertainty(hyper, xt_pinned, 1, m)
    phases = {k: round(v[1], 3) for k, v in capi.steps().items()}
    capi.steps_enable(False)
    capi.steps_reset()
    loss = gp.compute_loss(hyper)
    pcg_iters = gp.pcg_iterations()

    # the other precision modes on the same inputs, timed the same way, and
    # every mode's error against the plain FP64 path
    fp64 = None
    arms = {}
    if not args.skip_fp64:
        results = {}
        others = ["fp64"] + ([a for a in ARM_ORDER if a != args.precision] if not args.skip_arms else [])
        for prec in others:
            if prec == args.precision:
                continue
            set_mode(gp, prec)
            ma, va = torch.empty_like(dmean), torch.empty_like(dvar)
            el, st, ck = time_device_steps(torch, gp, hyper, dxt, m, ma, va, stream, args.steps, args.warmup,
                                           barrier, local, instrumented=(prec == "fp64"))
            msa = max_over_ranks(el, dist if world > 1 else None, device) / args.steps
            results[prec] = dict(mean=ma.cpu().numpy(), var=va.cpu().numpy(), loss=gp.compute_loss(hyper), ms=msa,
                                 clocks=ck, stats=st)
        set_mode(gp, args.precision, args.slices)
        ref64 = results["fp64"]

        def error_vs_fp64(mean_a, var_a, loss_a):
            return {
                "mean_max_rel": float(np.max(np.abs(mean_a - ref64["mean"])) / np.max(np.abs(ref64["mean"]))),
                "var_max_rel": float(np.max(np.abs(var_a - ref64["var"]) / ref64["var"])),
                "loss_rel": float(abs(loss_a - ref64["loss"]) / abs(ref64["loss"])),
            }

        st64 = ref64["stats"]
        fp64 = {
            "value": aggregate_seconds(ref64["ms"], world), "ms_per_step": ref64["ms"],
            "gemm_tflops": st64["gemm_flops"] / (st64["gemm_ms"] / 1e3) / 1e12 if st64["gemm_ms"] > 0 else None,
            "clocks": ref64["clocks"],
            "speedup_of_mixed": ref64["ms"] / ms_per_step,
            "mixed_error_vs_fp64": error_vs_fp64(mean_h, var_h, loss),
        }
        for prec, r in results.items():
            if prec != "fp64":
                arms[prec] = {"ms_per_step": r["ms"], "speedup_over_fp64": ref64["ms"] / r["ms"],
                              "error_vs_fp64": error_vs_fp64(r["mean"], r["var"], r["loss"]), "clocks": r["clocks"]}

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    peaks = measured_peaks()
    sustained = peaks.get("bf16_tflops_sustained")
    extra_peaks = {}
    if args.precision == "fp64":
        peak = measure_fp64_gemm_peak(torch, device)
        kernel = "dgemm_kernel (FP64 DMMA m16n8k8: Cholesky panel/trailing updates + variance solve)"
        peak_source = ("cuBLAS DGEMM (torch.matmul fp64 8192^3, best of 5) measured in this run; "
                       "MEASURED_PEAKS.json holds no FP64 figure")
    elif args.precision.startswith("fp64-int8"):
        # int8 tensor-core operations run at twice the bf16 rate on B200, so the
        # measured dense bf16 figure (sustained: the GEMMs run inside a
        # half-second step) doubled is this kernel's denominator
        in_run = measure_int8_peak(torch, device)
        peak = 2.0 * sustained if sustained else in_run
        kernel = ("oz_gemm_kernel (tcgen05.mma.cta_group::2 kind::i8, int32 groups in TMEM, FP64 accumulation in the "
                  "epilogue: every product of the factorisation and of the variance solve)")
        peak_source = ("2 x MEASURED_PEAKS.json bf16_tflops_sustained (of measured; int8 runs at twice the bf16 "
                       "rate)" if sustained else "cuBLASLt int8 GEMM measured in this run (MEASURED_PEAKS.json absent)")
        extra_peaks = {"cublaslt_int8_in_run": in_run,
                       "frac_of_cublaslt_int8_in_run": None}
    elif args.precision == "mixed-tf32":
        peak = sustained or measure_gemm_peak(torch, device, torch.bfloat16)
        kernel = ("tc_gemm_kernel<TF32> (tcgen05.mma kind::tf32, TMA-staged, TMEM accumulators: panel solves, "
                  "trailing updates, variance solve)")
        peak_source = ("MEASURED_PEAKS.json bf16_tflops_sustained (of measured); TF32 runs at half that rate"
                       if sustained else "cuBLAS bf16 measured in this run (MEASURED_PEAKS.json absent)")
        extra_peaks = {"tf32_half_rate": peak / 2.0, "frac_of_tf32_half_rate": None}
    else:
        peak = sustained or measure_gemm_peak(torch, device, torch.bfloat16)
        kernel = "tc_gemm_kernel<BF16> (tcgen05.mma kind::f16 with bf16 operands)"
        peak_source = ("MEASURED_PEAKS.json bf16_tflops_sustained (of measured)" if sustained
                       else "cuBLAS bf16 measured in this run (MEASURED_PEAKS.json absent)")
    gemm_tflops = stats["gemm_flops"] / (stats["gemm_ms"] / 1e3) / 1e12 if stats["gemm_ms"] > 0 else None
    if gemm_tflops and "cublaslt_int8_in_run" in extra_peaks:
        extra_peaks["frac_of_cublaslt_int8_in_run"] = gemm_tflops / extra_peaks["cublaslt_int8_in_run"]
    if gemm_tflops and "tf32_half_rate" in extra_peaks:
        extra_peaks["frac_of_tf32_half_rate"] = gemm_tflops / extra_peaks["tf32_half_rate"]
    step_flops = algorithmic_flops(n, m)
    if world == 1 and not args.skip_cpu_baseline:
        times, desc, threads = cpu_reference_full(wl, 1)
        cpu = {"value": times[0], "unit": "s", "cores": threads, "kind": "reference", "sample": desc,
               "calls_at_sample": cpu_reference_calls(wl),
               "gpu_calls_at_sample": {"fp64": gpu_calls(wl, capi.PREC_FP64),
                                       args.precision: gpu_calls(wl, args.precision)}}
        if not args.skip_c3:
            cpu["c3_optimize"] = c3_optimize(reference=True)
    else:
        cpu = None
    comparator = None
    if world == 1 and not args.skip_fp64:
        comparator = cusolver_fp64_comparator(torch, device, wl)
    serve = None
    if world == 1 and not args.skip_serving:
        serve = {args.precision: serving_bench(PRECISIONS[args.precision][0])}
        if args.precision != "fp64" and not args.skip_fp64:
            serve["fp64"] = serving_bench(capi.PREC_FP64)
    line = {
        "metric": METRIC,
        "value": aggregate_seconds(ms_per_step, world),
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
        "config": config_of(wl),
        "pipeline_tflops": step_flops / (ms_per_step / 1e3) / 1e12,
        "roofline": {
            "kernel": kernel,
            "bound": "tensor",
            "achieved": gemm_tflops,
            "peak": peak,
            "peak_source": peak_source,
            "unit": "TOP/s (int8)" if args.precision.startswith("fp64-int8") else "TFLOP/s",
            "frac": (gemm_tflops / peak) if gemm_tflops else None,
            **extra_peaks,
            # per-launch DRAM bytes of the dominant kernel where a capture of this workload exists
            "traffic": ((TRAFFIC_SAMPLE.get(args.precision) or {}).get("dram_bytes")
                        if (TRAFFIC_SAMPLE.get(args.precision) or {}).get("workload") == args.workload else None),
            "traffic_sample": TRAFFIC_SAMPLE.get(args.precision),
            "gemm_share_of_step": (stats["gemm_ms"] / args.steps) / ms_per_step,
            "gemm_launches_per_step": stats["gemm_launches"] / args.steps,
        },
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int((m + d - 1) * 8),
                "d2h_bytes_per_step": int(2 * m * 8)},
        "gpu_launches": int(stats["launches"]),
        "phases_ms": phases,
        "clocks": clk,
        "fp64": fp64,
        "arms": arms,
        "fp64_library_comparator": comparator,
        "serving": serve,
        "hbm_peak_gbs": peaks.get("hbm_gbs"),
        "pcg_iterations": pcg_iters,
        "sanity": sane,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--precision", choices=sorted(PRECISIONS), default="fp64-int8")
    ap.add_argument("--slices", type=int, default=0, help="int8 digit planes of the fp64-int8 mode (0 = default)")
    ap.add_argument("--skip-cpu-baseline", action="store_true",
                    help="omit the CPU reference sample (cpu_baseline becomes null)")
    ap.add_argument("--skip-fp64", action="store_true", help="omit the FP64 comparison arm")
    ap.add_argument("--skip-serving", action="store_true", help="omit the serving stream")
    ap.add_argument("--skip-c3", action="store_true", help="omit the 50-step optimisation timing (ours and reference)")
    ap.add_argument("--skip-arms", action="store_true", help="omit the other precision modes (FP64 still runs)")
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
