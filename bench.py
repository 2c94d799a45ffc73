#!/usr/bin/env python
"""Headline benchmark: pair-evaluations per second of the Hawkes log-likelihood
plus gradient at N = 100,000 events, FP32-compensated, with the plain FP64
CUDA path measured in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: N = 100,000 events, D = 2, locations U[0,20)^2 km, times U[0,8760) h
sorted, numpy default_rng(5), parameters (sigma=1, tauX=1/1.6, tauT=1/336,
omega=1, theta=1, mu0=1).  One step = one log-likelihood + gradient
evaluation = N^2 pair-evaluations (every ordered pair for one parameter
vector).

--impl ours (default): one process per GPU (torchrun for N > 1); every rank
evaluates the full workload on its own GPU (replicas, weak scaling).  Inputs
are resident in HBM when the timed region starts; L2 is flushed (a 256 MiB
write) before every timed step and the flush is outside the step's CUDA-event
pair.  "e2e" repeats the measurement through the public API with host buffers
(setTimesData / updateLocations / setParameters / getLogLikelihoodAndGradient,
host->device copies and the result read-back inside the timed region).

--impl reference: the reference's own CPU engine (hpHawkes NewHawkes, double,
"TBB" path over all host cores, compiled from its sources into oracle/_ref) on
a bounded sample of the same workload; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "pair-evals/s loglik+grad, N=100k: FP32-comp vs FP64 plain @ rel err<=1e-8"
UNIT = "pair-evals/s"
N_EVENTS = 100000
SEED = 5
L2_FLUSH_BYTES = 256 << 20

# Algorithmic FP32 work per evaluated pair term (counted once per
# instruction, FMA = 1): background term 11 (dx, dy, dt; d^2; exponent;
# three weighted sums) + 1 ex2; self-excitation term 5 (exponent; three
# weighted sums) + 1 ex2.
FP32_PER_B, FP32_PER_S = 11.0, 5.0
FP32_LANES_PER_SM = 128


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"sm_max_mhz": 1965.0}, "fallback"


# ----------------------------------------------------------- clock sampling --

class ClockSampler:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, gpu_indices):
        self.tmp.flush()
        self.tmp.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.tmp.read())) if len(r) >= 10]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                idx, clk, cmax, util = int(r[0]), float(r[1]), float(r[2]), float(r[4])
            except ValueError:
                continue
            if gpu_indices is not None and idx not in gpu_indices:
                continue
            if util < 50:
                continue
            sm.append(clk)
            smax.append(cmax)
            for name, v in zip(names, r[6:10]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ reference arm --

def reference_arm(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    import oracle
    from hawkes_b200 import workloads

    cores = os.cpu_count() or 1
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU engine (oracle/_ref) not built"}))
        return 0
    # Calibrate the sample size so the whole run (warm-up + steps) takes about
    # two minutes on this host, and no step more than ~6 s.
    step_s = min(6.0, 120.0 / max(1, args.steps + args.warmup))
    loc, t = workloads.uniform(4000, seed=SEED)
    eng = oracle.RefEngine(2, 4000, threads=cores)
    eng.set_data(loc, t)
    eng.set_parameters(workloads.BASE_PARAMS)
    t0 = time.perf_counter()
    eng.loglik()
    rate = 4000.0 ** 2 / (time.perf_counter() - t0)
    eng.close()
    n = int(min(N_EVENTS, max(2000, math.sqrt(step_s * rate)) // 1000 * 1000))
    loc, t = workloads.uniform(n, seed=SEED)
    eng = oracle.RefEngine(2, n, threads=cores)
    variant = eng.variant.splitlines()[0]
    eng.set_data(loc, t)
    eng.set_parameters(workloads.BASE_PARAMS)
    for _ in range(args.warmup):
        eng.loglik()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        eng.loglik()
        times.append(time.perf_counter() - t0)
    eng.close()
    ms = 1e3 * statistics.mean(times)
    value = n * n / (ms / 1e3)
    sample = (f"N={n} events of the same generator (uniform 20x20 km, [0,8760) h, seed {SEED}); "
              f"log-likelihood only (the reference has no gradient); {variant}, {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"uniform N={n} D=2 (bounded sample of N={N_EVENTS}), base params,"
                               " loglik", "N": n, "D": 2},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def cpu_baseline(budget_s=15.0):
    """The reference CPU engine (or the oracle port when it is not built) on
    a bounded sample, all host cores."""
    import oracle
    from hawkes_b200 import workloads

    cores = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    loc, t = workloads.uniform(4000, seed=SEED)
    if kind == "reference":
        def evaluate(loc, t):
            e = oracle.RefEngine(2, len(t), threads=cores)
            e.set_data(loc, t)
            e.set_parameters(workloads.BASE_PARAMS)
            t0 = time.perf_counter()
            e.loglik()
            dt = time.perf_counter() - t0
            v = e.variant.splitlines()[0]
            e.close()
            return dt, v
    else:
        def evaluate(loc, t):
            t0 = time.perf_counter()
            oracle.oracle_eval(loc, t, workloads.BASE_PARAMS, threads=cores)
            return time.perf_counter() - t0, "oracle port (C, FP64, long double sums)"
    dt, _ = evaluate(loc, t)
    rate = 4000.0 ** 2 / dt
    n = int(min(N_EVENTS, max(4000, math.sqrt(budget_s * rate)) // 1000 * 1000))
    loc, t = workloads.uniform(n, seed=SEED)
    dt, variant = evaluate(loc, t)
    what = "log-likelihood only (the reference has no gradient)" if kind == "reference" else \
        "log-likelihood + gradient"
    return {"value": n * n / dt, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"one evaluation at N={n} (same generator, seed {SEED}), {what}; {variant}"}


# ------------------------------------------------------------------ our arm --

def time_device(eng, steps, warmup, torch, stream, flush):
    """Per-step device time (CUDA events on the engine's stream), L2 flushed
    before each step outside the event pair; also the sweep-kernel time."""
    eng.setKernelTiming(True)
    for _ in range(warmup):
        eng.enqueueLogLikelihoodAndGradient()
        eng.readResults()
    step_ms, sweep_ms = [], []
    res = None
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.enqueueLogLikelihoodAndGradient()
        e1.record(stream)
        res = eng.readResults()
        step_ms.append(e0.elapsed_time(e1))
        sweep_ms.append(eng.kernelTimes()[0])
    eng.setKernelTiming(False)
    return step_ms, sweep_ms, res


def time_e2e(hb, flags, loc, t, p, steps, warmup, device):
    eng = hb.CudaHawkes(2, len(t), flags, device)
    loc_flat = np.ascontiguousarray(loc).reshape(-1)

    def step():
        eng.setTimesData(t)
        eng.updateLocations(-1, loc_flat)
        eng.setParameters(p)
        return eng.getLogLikelihoodAndGradient()

    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = (time.perf_counter() - t0) / steps
    eng.close()
    return dt


def ours_arm(args):
    import torch

    import hawkes_b200 as hb
    from hawkes_b200 import workloads

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    N = args.n
    loc, t = workloads.uniform(N, seed=SEED)
    p = workloads.BASE_PARAMS.copy()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    def make(flags):
        e = hb.CudaHawkes(2, N, flags, local)
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(p)
        return e

    fp32 = make(hb.CUDA | hb.COMPENSATED)
    fp64 = make(hb.CUDA)
    s32 = torch.cuda.ExternalStream(fp32.stream, device=f"cuda:{local}")
    s64 = torch.cuda.ExternalStream(fp64.stream, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # FP64 plain path (the comparison in the metric)
    barrier()
    ms64, sweep64, res64 = time_device(fp64, args.steps, args.warmup, torch, s64, flush)
    barrier()
    # FP32-compensated path (the headline), clocks sampled while it runs
    with ClockSampler() as clocks:
        barrier()
        ms32, sweep32, res32 = time_device(fp32, args.steps, args.warmup, torch, s32, flush)
        barrier()
    launches, nb, ns = fp32.lastLaunchStats()
    shape32 = fp32.sweepShape()
    _, nb64, ns64 = fp64.lastLaunchStats()

    tot32 = torch.tensor([sum(ms32), sum(ms64)], dtype=torch.float64, device=f"cuda:{local}")
    if dist:
        dist.all_reduce(tot32, op=dist.ReduceOp.MAX)
    ms_step32 = float(tot32[0]) / args.steps
    ms_step64 = float(tot32[1]) / args.steps

    # End to end through the public API with host buffers.
    barrier()
    e2e_s = time_e2e(hb, hb.CUDA | hb.COMPENSATED, loc, t, p, args.steps, args.warmup, local)
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_t[0])

    clock_summary = clocks.summary(None)
    fp32.close()
    fp64.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    pairs = float(N) * N
    value = world * pairs / (ms_step32 / 1e3)
    value64 = world * pairs / (ms_step64 / 1e3)
    peaks, peak_src = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    max_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    peak_inst = sm_count * FP32_LANES_PER_SM * max_mhz * 1e6 / 1e12
    sweep_mean = statistics.mean(sweep32)
    achieved = (FP32_PER_B * nb + FP32_PER_S * ns) / (sweep_mean / 1e3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get("fp32c_N100000_bytes_per_launch")

    ll32, g32 = res32
    ll64, g64 = res64
    acc = {"loglik_rel_vs_fp64": abs(ll32 - ll64) / abs(ll64),
           "grad_rel_vs_fp64": [abs(a - b) / abs(b) if b else None for a, b in zip(g32, g64)]}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step32, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair terms (compensated), f64 reductions", "data": "synthetic",
        "config": {"workload": f"uniform N={N} D=2, 20x20 km, [0,8760) h sorted, seed {SEED}, "
                               "base params; log-likelihood + 6-parameter gradient",
                   "N": N, "D": 2, "precision": "fp32-compensated",
                   "l2": "flushed before every timed step (256 MiB write, outside the timing)",
                   "parallelism": f"replicas x{world}"},
        "fp64_plain": {"value": value64, "ms_per_step": ms_step64,
                       "sweep_ms": statistics.mean(sweep64),
                       "terms": {"background": nb64, "self_excitation": ns64}},
        "speedup_fp32c_vs_fp64": value / value64,
        "accuracy": acc,
        "terms": {"background": nb, "self_excitation": ns, "possible": 2 * pairs,
                  "note": "pair terms the sweep evaluated; the rest are the non-causal half of "
                          "the self-excitation sum and tile pairs whose terms are all exactly "
                          "zero in FP32"},
        "roofline": {"bound": "fp32",
                     "kernel": f"sweep_f32c_kernel<D=2, R={shape32[0]}>, {shape32[1]} items/SM",
                     "achieved": achieved, "peak": peak_inst, "unit": "Tinst/s",
                     "frac": achieved / peak_inst, "traffic": traffic,
                     "count": "FP32-pipe instructions, FMA = 1: 11 per background term + 5 per "
                              "self-excitation term evaluated, per sweep launch, over the mean "
                              "CUDA-event duration of the sweep kernel",
                     "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {max_mhz:.0f} MHz "
                                    f"(sm_max_mhz, {peak_src})",
                     "sweep_ms": sweep_mean},
        "e2e": {"value": world * pairs / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": N * 2 * 8 + N * 8 + N * 4, "d2h_bytes_per_step": 64},
        "gpu_launches": launches * args.steps,
        "clocks": clock_summary,
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=N_EVENTS, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
