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

--shard: the same N = 100,000 evaluation split across the ranks (strong
scaling): each rank sweeps its share of the target strips, the shares of the
per-event unit sums (6 N doubles per rank) are all-gathered over NCCL and
every rank runs the O(N) finish (hawkes_b200.shard).  The step is timed with
CUDA events on the engine's stream around sweep, gather and finish.

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

# Algorithmic work (FMA = 1 instruction).  The roofline counts the terms a
# sweep launch evaluated: a background exponential costs 11 FP32 instructions
# (dx, dy, dt; d^2; exponent; three weighted sums) + 1 ex2, and 3 more (the
# other event's three weighted sums) when one evaluation serves both events
# of a pair; a self-excitation term costs 5 (exponent; three weighted sums) +
# 1 ex2.  The brute-force sum over every ordered pair would cost 11 + 5/2 =
# 13.5 FP32 instructions and 1.5 ex2 per pair-eval; the sweep skips the
# non-causal half, exact underflows, the truncated background tail and one
# order of each background pair, so that count ("effective") is a rate
# equivalent and can exceed the pipe's peak.
FP32_PER_PAIR_EVAL, EX2_PER_PAIR_EVAL = 13.5, 1.5
FP32_PER_B, FP32_PER_COL, FP32_PER_S = 11.0, 3.0, 5.0
# The roofline counts the algorithm, not its compensation.  As a second
# figure, the FP32-compensated implementation adds the work its precision
# pattern requires: every near background term (a tile pair not in the far
# tail) and every self-excitation term takes its time difference from hi and
# lo parts (+2) and enters its three sums by Fast2Sum (+3 each, +9); far-tail
# background terms (each at most 2^-10 of the event's own term) and the
# symmetric column adds keep the plain count.
FP32C_PER_NEAR_B, FP32C_PER_S = FP32_PER_B + 11.0, FP32_PER_S + 11.0
FP32_LANES_PER_SM = 128
MUFU_LANES_PER_SM = 16


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

def load_workloads():
    """hawkes_b200/workloads.py loaded by path, without importing the
    hawkes_b200 package (whose __init__ loads the CUDA library): the CPU arms
    map only the reference engine."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_hawkes_workloads", os.path.join(ROOT, "hawkes_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def headline_config(world, n=N_EVENTS):
    """The config object both arms print: the same events, sizes and
    parameters."""
    return {"workload": f"uniform N={n} D=2, 20x20 km, [0,8760) h sorted, seed {SEED}, "
                        "base params (sigma=1, tauX=1/1.6, tauT=1/336, omega=1, theta=1, mu0=1)",
            "N": n, "D": 2,
            "l2": "GPU arm: flushed before every timed step (256 MiB device write, outside the "
                  "timing); CPU arm: host memory",
            "parallelism": f"replicas x{world}"}


# The reference arm times whole evaluations of the headline events while
# --steps K of them fit about REF_BUDGET_S seconds (one N = 100,000
# evaluation takes ~17 s on 16 host threads, so K <= 20 stays at the
# headline size); a larger K times evaluations of the first N sqrt(K0 / K)
# events instead, K0 = the K that fits, so the run still ends in minutes.
REF_BUDGET_S = 360.0
REF_STEP_S_100K = 17.0


def reference_arm(args):
    """The reference's own CPU engine (NewHawkes, double, its TBB path over
    all host cores; src/NewHawkes.hpp:812-848) on the headline events: every
    timed step is one full evaluation (N = 100,000 for up to 20 steps, see
    REF_BUDGET_S).  Warm-up steps evaluate the first 20,000 events (they only
    warm the thread pool and caches)."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    import oracle

    wl = load_workloads()
    cores = os.cpu_count() or 1
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU engine (oracle/_ref) not built"}))
        return 0
    n = args.n
    fit = REF_BUDGET_S / (REF_STEP_S_100K * (n / 1e5) ** 2)  # full steps that fit the budget
    if args.steps > fit:
        n = max(2000, int(n * math.sqrt(fit / args.steps)) // 1000 * 1000)
    loc, t = wl.uniform(args.n, seed=SEED)
    loc, t = loc[:n], t[:n]
    nw = min(n, 20000)
    warm = oracle.RefEngine(2, nw, threads=cores)
    warm.set_data(loc[:nw], t[:nw])
    warm.set_parameters(wl.BASE_PARAMS)
    for _ in range(args.warmup):
        warm.loglik()
    warm.close()
    eng = oracle.RefEngine(2, n, threads=cores)
    variant = eng.variant.splitlines()[0]
    eng.set_data(loc, t)
    eng.set_parameters(wl.BASE_PARAMS)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        eng.loglik()
        times.append(time.perf_counter() - t0)
    eng.close()
    ms = 1e3 * statistics.mean(times)
    value = float(n) * n / (ms / 1e3)
    which = (f"the headline events, seed {SEED}" if n == args.n else
             f"the first {n} of the N={args.n} headline events, seed {SEED}, so that "
             f"{args.steps} steps fit about {REF_BUDGET_S:.0f} s")
    sample = (f"{args.steps} full evaluations at N={n} ({which}); "
              f"log-likelihood only (the reference has no gradient); {variant}, {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "computes": "log-likelihood (the reference has no gradient)",
        "config": headline_config(args.gpus, n),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def cpu_baseline(n=N_EVENTS):
    """The reference CPU engine (or the oracle port when it is not built):
    one full evaluation of the headline events on all host cores."""
    import oracle

    wl = load_workloads()
    cores = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    loc, t = wl.uniform(n, seed=SEED)
    if kind == "reference":
        e = oracle.RefEngine(2, n, threads=cores)
        e.set_data(loc, t)
        e.set_parameters(wl.BASE_PARAMS)
        t0 = time.perf_counter()
        e.loglik()
        dt = time.perf_counter() - t0
        variant = e.variant.splitlines()[0]
        e.close()
        what = "log-likelihood only (the reference has no gradient)"
    else:
        t0 = time.perf_counter()
        oracle.oracle_eval(loc, t, wl.BASE_PARAMS, threads=cores)
        dt = time.perf_counter() - t0
        variant = "oracle port (C, FP64, long double sums)"
        what = "log-likelihood + gradient"
    return {"value": float(n) * n / dt, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"one full evaluation at N={n} (the headline events, seed {SEED}), {what}; "
                      f"{variant}; {dt:.1f} s"}


# ------------------------------------------------------------------ our arm --

class Ranks:
    """One process per GPU: the process group, barriers and the max-over-ranks
    reduction of device times.  backend "nccl" on GPUs (the bench), "gloo" on
    CPU (the multi-process tests); world 1 needs no process group."""

    def __init__(self, world: int, backend: str = "nccl", device=None, timeout_s: int = 120):
        import torch
        self.world = world
        self.device = device
        self.dist = None
        if world > 1:
            import datetime

            import torch.distributed as dist
            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist
        self._torch = torch

    def barrier(self):
        cuda = self.device is not None and self.device.type == "cuda"
        if cuda:
            self._torch.cuda.synchronize()
        if self.dist:
            self.dist.barrier()
        if cuda:
            self._torch.cuda.synchronize()

    def max(self, values):
        """Elementwise maximum over ranks of a list of floats (every rank calls it)."""
        t = self._torch.tensor([float(v) for v in values], dtype=self._torch.float64,
                               device=self.device)
        if self.dist:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return [float(v) for v in t.cpu()]

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(world: int, units_per_rank: float, ms_max: float) -> float:
    """Units all ranks processed per second, over the slowest rank's time."""
    return world * units_per_rank / (ms_max / 1e3)


class Runner:
    """One workload on one GPU: the timed step through the engine (data on the
    device, CUDA-event step time recorded by the engine on its stream) and the
    end-to-end step through the public API with host buffers."""

    def __init__(self, hb, workload, flags, device):
        self.hb, self.w, self.flags, self.device = hb, workload, flags, device
        kind = workload["kind"]
        if kind == "single":
            loc, t, p = workload["loc"], workload["t"], workload["params"]
            self.eng = hb.CudaHawkes(loc.shape[1], len(t), flags, device)
            self.eng.setTimesData(t)
            self.eng.updateLocations(-1, loc)
            self.eng.setParameters(p)
        elif kind == "batch":
            loc, t = workload["loc"], workload["t"]
            self.eng = hb.CudaHawkes(loc.shape[1], len(t), flags, device)
            self.eng.setTimesData(t)
            self.eng.updateLocations(-1, loc)
        else:
            sets = workload["sets"]
            self.eng = hb.Multiset(2, [len(t) for _, t, _ in sets], flags, device)
            for k, (loc, t, _) in enumerate(sets):
                self.eng.setData(k, loc, t)
        self.stream = (self.eng.stream if kind != "sets" else None)

    def evaluate(self):
        kind = self.w["kind"]
        if kind == "single":
            self.eng.enqueueLogLikelihoodAndGradient()
            return self.eng.readResults()
        if kind == "batch":
            return self.eng.batchLogLikelihoodAndGradient(self.w["params"])
        return self.eng.logLikelihoodAndGradient(self.w["params"])

    def e2e_step(self):
        kind, w = self.w["kind"], self.w
        if kind == "single":
            self.eng.setTimesData(w["t"])
            self.eng.updateLocations(-1, w["loc"])
            self.eng.setParameters(w["params"])
            return self.eng.getLogLikelihoodAndGradient()
        if kind == "batch":
            self.eng.setTimesData(w["t"])
            self.eng.updateLocations(-1, w["loc"])
            return self.eng.batchLogLikelihoodAndGradient(w["params"])
        for k, (loc, t, _) in enumerate(w["sets"]):
            self.eng.setData(k, loc, t)
        return self.eng.logLikelihoodAndGradient(w["params"])

    def close(self):
        self.eng.close()


def time_device(run, steps, warmup, flush_fn):
    """Per-step device time from the CUDA events the engine records on its own
    stream around the step (table upload, record build, sweep, finish, result
    copy); L2 is flushed before each step, outside those events.  Also the
    sweep kernel's own event time."""
    run.eng.setKernelTiming(True)
    for _ in range(warmup):
        run.evaluate()
    step_ms, sweep_ms, res = [], [], None
    for _ in range(steps):
        flush_fn()
        res = run.evaluate()
        sweep, _, step = run.eng.kernelTimes()
        step_ms.append(step)
        sweep_ms.append(sweep)
    run.eng.setKernelTiming(False)
    return step_ms, sweep_ms, res


def time_e2e(run, steps, warmup):
    for _ in range(warmup):
        run.e2e_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        run.e2e_step()
    return (time.perf_counter() - t0) / steps


def make_workload(name, n):
    """The timed workloads; every other configuration is a parity-test case."""
    from hawkes_b200 import workloads
    base = workloads.BASE_PARAMS.copy()
    if name == "headline":
        loc, t = workloads.uniform(n, seed=SEED)
        return {"kind": "single", "loc": loc, "t": t, "params": base, "pairs": float(n) * n,
                "h2d": n * 2 * 8 + n * 8, "d2h": 64,
                "desc": f"uniform N={n} D=2, 20x20 km, [0,8760) h sorted, seed {SEED}, base "
                        "params; log-likelihood + 6-parameter gradient",
                "config": {"N": n, "D": 2}}
    if name == "batched":
        loc, t = workloads.uniform(20000, seed=2)
        P = workloads.proposals(256, seed=2)
        return {"kind": "batch", "loc": loc, "t": t, "params": P, "pairs": 256 * 20000.0 ** 2,
                "h2d": 20000 * 24 + P.size * 8, "d2h": 256 * 7 * 8,
                "desc": "uniform N=20000 D=2 (seed 2), 256 proposals base*exp(0.3 z) (seed 2), "
                        "one run; log-likelihood + gradient each",
                "config": {"N": 20000, "K": 256, "D": 2}}
    if name == "uneven":
        sets = workloads.uneven(64, seed=3)
        params = np.stack([p for _, _, p in sets])
        sizes = [len(t) for _, t, _ in sets]
        return {"kind": "sets", "sets": sets, "params": params,
                "pairs": float(sum(float(m) * m for m in sizes)),
                "h2d": sum(m * 24 for m in sizes) + params.size * 8, "d2h": 64 * 7 * 8,
                "desc": "64 uniform sets, sizes log-uniform in [1e3, 1e5] (seed 3), own "
                        "log-normal params each, one run; log-likelihood + gradient each",
                "config": {"sets": 64, "N_total": int(sum(sizes)), "N_max": int(max(sizes)),
                           "D": 2}}
    if name == "clustered":
        loc, t = workloads.clustered()
        m = len(t)
        return {"kind": "single", "loc": loc, "t": t, "params": base, "pairs": float(m) * m,
                "h2d": m * 24, "d2h": 64,
                "desc": "Hawkes branching process N=500000 (50x50 km, [0,8760) h, Poisson(0.5) "
                        "offspring, seed 4), base params; log-likelihood + gradient",
                "config": {"N": m, "D": 2}}
    raise ValueError(name)


def far_tail_share(t, tau_t, R, tile=128):
    """Share of the symmetric FP32 sweep's background exponentials that fall
    in far-tail tile pairs, from the tile-pair decisions on sorted times:
    a strip of R tiles meets every tile up to its own last one; a pair is
    skipped when every background term is below 2^-60 (tail truncation), far
    when below 2^-10 (log2 exponent -(b dt)^2 log2(e) / 2 over min |dt|)."""
    t = np.asarray(t, dtype=np.float64)
    n = len(t)
    nt = (n + tile - 1) // tile
    pad = nt * tile - n
    tp = np.concatenate([t, np.full(pad, np.nan)]).reshape(nt, tile)
    lo, hi = np.nanmin(tp, 1), np.nanmax(tp, 1)
    cnt = np.minimum(tile, n - np.arange(nt) * tile).astype(np.float64)
    k = 0.5 * tau_t * tau_t * math.log2(math.e)  # log2 exponent per squared hour
    near = far = 0.0
    for s0 in range(0, nt, R):
        s1 = min(s0 + R, nt)
        slo, shi = lo[s0:s1].min(), hi[s0:s1].max()
        rows = cnt[s0:s1].sum()
        j = np.arange(s1)
        gap = np.maximum(0.0, np.maximum(slo - hi[j], lo[j] - shi))
        e2 = k * gap * gap
        w = rows * cnt[j]
        keep = e2 < 60.0
        far += float(np.sum(w[keep & (e2 >= 10.0)]))
        near += float(np.sum(w[keep & (e2 < 10.0)]))
    return far / max(near + far, 1.0)


def oracle_accuracy(res32, res64, n):
    """Errors of both arms against the committed oracle fixture of the
    headline events (tests/golden/headline_n100k.npz): log-likelihood
    relative, gradient componentwise |dg_k| / |g_k| and on the per-event
    scale sum_i |per-event contribution|."""
    path = os.path.join(ROOT, "tests", "golden", "headline_n100k.npz")
    if n != N_EVENTS or not os.path.exists(path):
        return None
    z = np.load(path)
    ll_o, g_o, scale = float(z["oracle_loglik"]), z["oracle_grad"], z["grad_scale"]
    out = {"reference": "oracle (C restatement, long-double sums) at N=100000; its "
                        "log-likelihood agrees with the reference engine's to "
                        f"{abs(ll_o - float(z['ref_loglik'])) / abs(ll_o):.1e}"
                        if "ref_loglik" in z else "oracle (C restatement) at N=100000"}
    for name, (ll, g) in (("fp32c", res32), ("fp64", res64)):
        g = np.asarray(g, dtype=np.float64).reshape(-1)
        comp = np.abs(g - g_o) / np.abs(g_o)
        out[name] = {"loglik_rel": abs(float(ll) - ll_o) / abs(ll_o),
                     "grad_rel_componentwise": [float(v) for v in comp],
                     "grad_rel_per_event_scale": [float(v) for v in np.abs(g - g_o) / scale]}
    f = out["fp32c"]
    out["bound_1e-8_met"] = bool(f["loglik_rel"] <= 1e-8 and
                                 max(f["grad_rel_componentwise"]) <= 1e-8)
    return out


def ours_arm(args):
    import torch

    import hawkes_b200 as hb

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    ranks = Ranks(world, "nccl", torch.device("cuda", local))
    barrier = ranks.barrier

    w = make_workload(args.workload, args.n)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    def flusher(run):
        if run.stream:
            ext = torch.cuda.ExternalStream(run.stream, device=f"cuda:{local}")
            def f():
                with torch.cuda.stream(ext):
                    flush.zero_()
        else:
            def f():
                flush.zero_()
                torch.cuda.synchronize()
        return f

    fp32 = Runner(hb, w, hb.CUDA | hb.COMPENSATED, local)
    fp64 = Runner(hb, w, hb.CUDA, local)
    if args.shape and w["kind"] != "sets":
        r_, i_ = (int(v) for v in args.shape.split(":"))
        fp32.eng.setSweepShape(r_, i_)

    # FP64 plain path (the comparison in the metric)
    barrier()
    ms64, sweep64, res64 = time_device(fp64, args.steps64 or args.steps, args.warmup,
                                       flusher(fp64))
    barrier()
    # FP32-compensated path (the headline), clocks sampled while it runs
    with ClockSampler() as clocks:
        barrier()
        ms32, sweep32, res32 = time_device(fp32, args.steps, args.warmup, flusher(fp32))
        barrier()
    launches, nb, ns = fp32.eng.lastLaunchStats()
    nev = fp32.eng.lastLaunchEvals()
    shape32 = fp32.eng.sweepShape() if w["kind"] != "sets" else None
    _, nb64, ns64 = fp64.eng.lastLaunchStats()
    steps64 = args.steps64 or args.steps

    ms_step32, ms_step64 = ranks.max([sum(ms32) / args.steps, sum(ms64) / steps64])

    # End to end through the public API with host buffers.
    fp64.close()
    barrier()
    e2e_s = time_e2e(fp32, max(1, min(args.steps, 50)), args.warmup)
    e2e_s = ranks.max([e2e_s])[0]

    clock_summary = clocks.summary(None)
    fp32.close()
    ranks.close()
    if rank != 0:
        return 0

    pairs = w["pairs"]
    value = whole_job_rate(world, pairs, ms_step32)
    value64 = whole_job_rate(world, pairs, ms_step64)
    peaks, peak_src = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    max_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    peak_inst = sm_count * FP32_LANES_PER_SM * max_mhz * 1e6 / 1e12
    peak_ex2 = sm_count * MUFU_LANES_PER_SM * max_mhz * 1e6 / 1e12
    sweep_mean = statistics.mean(sweep32)
    # the roofline counts the terms the launch evaluated; "effective" counts
    # the brute-force work (every ordered pair) the launch stands for
    # algorithmic count of the evaluated terms (compensation not counted)
    inst = FP32_PER_B * nev + FP32_PER_COL * (nb - nev) + FP32_PER_S * ns
    achieved = inst / (sweep_mean / 1e3) / 1e12
    far = (far_tail_share(w["t"], w["params"][2], shape32[0])
           if w["kind"] == "single" and shape32 else 1.0)
    inst_comp = (FP32C_PER_NEAR_B * (1.0 - far) * nev + FP32_PER_B * far * nev +
                 FP32_PER_COL * (nb - nev) + FP32C_PER_S * ns)
    ncu = None
    npath = os.path.join(ROOT, "profiles", "sweep_pipes.json")
    if os.path.exists(npath):
        with open(npath) as f:
            ncu = json.load(f).get(f"fp32c_{args.workload}")
    achieved_ex2 = (nev + ns) / (sweep_mean / 1e3) / 1e12
    effective = FP32_PER_PAIR_EVAL * pairs / (sweep_mean / 1e3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(f"fp32c_{args.workload}_bytes_per_launch")

    ll32 = np.atleast_1d(np.asarray(res32[0], dtype=np.float64))
    ll64 = np.atleast_1d(np.asarray(res64[0], dtype=np.float64))
    g32 = np.atleast_2d(np.asarray(res32[1], dtype=np.float64))
    g64 = np.atleast_2d(np.asarray(res64[1], dtype=np.float64))
    acc = {"loglik_rel_vs_fp64_max": float(np.max(np.abs(ll32 - ll64) / np.abs(ll64))),
           "grad_rel_vs_fp64_max": [float(v) for v in
                                    np.max(np.abs(g32 - g64) / np.maximum(np.abs(g64), 1e-300),
                                           axis=0)]}
    kernel = ("sweep_f32c_list_kernel" +
              (f"<D=2, R={shape32[0]}>, {shape32[1]} items/SM" if shape32 else ""))
    metric = METRIC if args.workload == "headline" else \
        f"pair-evals/s loglik+grad, {args.workload}: FP32-comp vs FP64 plain"
    config = headline_config(world, args.n) if args.workload == "headline" \
        else dict({"workload": w["desc"],
                   "l2": "flushed before every timed step (256 MiB write, outside the timing)",
                   "parallelism": f"replicas x{world}"}, **w["config"])
    out = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step32, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair terms (compensated), f64 reductions", "data": "synthetic",
        "computes": "log-likelihood + 6-parameter gradient",
        "config": config,
        "fp64_plain": {"value": value64, "ms_per_step": ms_step64,
                       "sweep_ms": statistics.mean(sweep64), "steps": steps64,
                       "terms": {"background": nb64, "self_excitation": ns64}},
        "speedup_fp32c_vs_fp64": value / value64,
        "accuracy": acc,
        "accuracy_vs_oracle": (oracle_accuracy((res32[0], res32[1]), (res64[0], res64[1]), args.n)
                               if w["kind"] == "single" and args.workload == "headline" else None),
        "terms": {"background": nb, "self_excitation": ns, "possible": 2 * pairs,
                  "background_exponentials": nev,
                  "note": "pair terms the sweep accounted for; the rest are the non-causal half "
                          "of the self-excitation sum, self-excitation tile pairs whose terms "
                          "are all exactly zero in FP32, and background tile pairs whose terms "
                          "are all below 2^-60 of an event's own term (tail truncation of the "
                          "FP32 modes: under 2^-33 of any event's sums).  A background pair with the other event "
                          "in an earlier tile is evaluated once (one exponential) for both "
                          "events"},
        "roofline": {"bound": "fp32", "kernel": kernel,
                     "achieved": achieved, "peak": peak_inst, "unit": "Tinst/s",
                     "frac": achieved / peak_inst, "traffic": traffic,
                     "count": "FP32 instructions (FMA = 1) of the terms this launch evaluated, "
                              "compensation not counted: "
                              f"{FP32_PER_B:g} per background exponential, {FP32_PER_COL:g} per "
                              "background pair also added to the earlier event's sums, "
                              f"{FP32_PER_S:g} per self-excitation term; over the mean "
                              "CUDA-event duration of the sweep kernel",
                     "instructions_per_launch": inst,
                     "compensated_count": {
                         "instructions_per_launch": inst_comp,
                         "frac": inst_comp / (sweep_mean / 1e3) / 1e12 / peak_inst,
                         "far_tail_share": far,
                         "count": "the same terms with the work the precision pattern adds: "
                                  f"{FP32C_PER_NEAR_B:g} per near background exponential (hi/lo "
                                  "time difference, three Fast2Sum additions), "
                                  f"{FP32_PER_B:g} per far-tail one, {FP32C_PER_S:g} per "
                                  "self-excitation term"},
                     "ncu": ncu,
                     "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {max_mhz:.0f} MHz "
                                    f"(sm_max_mhz, {peak_src})",
                     "ex2": {"achieved": achieved_ex2, "peak": peak_ex2, "unit": "Tex2/s",
                             "frac": achieved_ex2 / peak_ex2,
                             "count": "one MUFU ex2 per evaluated exponential; peak "
                                      f"{sm_count} SMs x 16 MUFU lanes x {max_mhz:.0f} MHz"},
                     "effective": {"achieved": effective, "frac_equivalent": effective / peak_inst,
                                   "count": f"{FP32_PER_PAIR_EVAL} FP32 instructions per "
                                            f"pair-eval x {pairs:.4g} pair-evals: the brute-force "
                                            "work the launch stands for (it skips the non-causal "
                                            "half, exact underflows, the truncated tail and one "
                                            "order of each background pair), so this is a rate "
                                            "equivalent, not pipe utilisation"},
                     "sweep_ms": sweep_mean},
        "e2e": {"value": whole_job_rate(world, pairs, 1e3 * e2e_s), "unit": UNIT,
                "h2d_bytes_per_step": w["h2d"], "d2h_bytes_per_step": w["d2h"]},
        "gpu_launches": launches * args.steps,
        "clocks": clock_summary,
    }
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    print(json.dumps(out))
    return 0


def shard_arm(args):
    """One likelihood per step, split across the ranks (strong scaling)."""
    import torch

    import hawkes_b200 as hb
    from hawkes_b200.shard import ShardedHawkes

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Ranks(world, "nccl", dev)
    barrier = ranks.barrier
    w = make_workload("headline", args.n)
    loc, t, p = w["loc"], w["t"], w["params"]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def make(flags):
        e = hb.CudaHawkes(2, len(t), flags, local)
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(p)
        return e, ShardedHawkes(e)

    eng64, sh64 = make(hb.CUDA)
    res64 = sh64.getLogLikelihoodAndGradient()
    eng64.close()
    eng, sh = make(hb.CUDA | hb.COMPENSATED)
    ext = torch.cuda.ExternalStream(eng.stream, device=dev)
    eng.setKernelTiming(True)
    for _ in range(args.warmup):
        sh.getLogLikelihoodAndGradient()
    # launches of one step: the share's sweep, the rank-ordered sum, the finish
    sh.sweep()
    n_sweep, nb_share, ns_share = eng.lastLaunchStats()
    nev_share = eng.lastLaunchEvals()
    res = eng.getLogLikelihoodAndGradient()
    launches = n_sweep + 1 + eng.lastLaunchStats()[0]
    step_ms, sweep_ms = [], []
    with ClockSampler() as clocks:
        barrier()
        for _ in range(args.steps):
            with torch.cuda.stream(ext):
                flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(ext)
            sh.sweep()
            sweep_ms.append(eng.kernelTimes()[0])
            res = eng.getLogLikelihoodAndGradient()
            b.record(ext)
            b.synchronize()
            step_ms.append(a.elapsed_time(b))
        barrier()
    ms, sweep_max = ranks.max([statistics.mean(step_ms), statistics.mean(sweep_ms)])

    def e2e_step():
        eng.setTimesData(t)
        eng.updateLocations(-1, loc)
        eng.setParameters(p)
        return sh.getLogLikelihoodAndGradient()

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    n_e2e = max(1, min(args.steps, 50))
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        e2e_step()
    e2e_s = ranks.max([(time.perf_counter() - t0) / n_e2e])[0]
    clock_summary = clocks.summary(None)
    eng.close()
    ranks.close()
    if rank != 0:
        return 0
    pairs = w["pairs"]
    peaks, peak_src = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    max_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    peak_inst = sm_count * FP32_LANES_PER_SM * max_mhz * 1e6 / 1e12
    inst = FP32_PER_B * nev_share + FP32_PER_COL * (nb_share - nev_share) + FP32_PER_S * ns_share
    achieved = inst / (sweep_max / 1e3) / 1e12
    out = {
        "metric": METRIC, "value": pairs / (ms / 1e3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 pair terms (compensated), f64 reductions", "data": "synthetic",
        "config": dict({"workload": w["desc"], "precision": "fp32-compensated",
                        "l2": "flushed before every timed step (256 MiB write, outside the "
                              "timing)",
                        "parallelism": f"target strips sharded x{world}, unit sums "
                                       "all-gathered (NCCL), finish on every rank"},
                       **w["config"]),
        "accuracy": {"loglik_rel_vs_fp64": abs(res[0] - res64[0]) / abs(res64[0]),
                     "grad_rel_vs_fp64": [float(abs(x - y) / abs(y))
                                          for x, y in zip(res[1], res64[1])]},
        "roofline": {"bound": "fp32", "kernel": "sweep_f32c_list_kernel (one rank's share)",
                     "achieved": achieved, "peak": peak_inst, "unit": "Tinst/s",
                     "frac": achieved / peak_inst, "traffic": None,
                     "count": "FP32 instructions of the terms rank 0's share evaluated "
                              f"({FP32_PER_B:g} per background exponential, {FP32_PER_COL:g} per "
                              f"pair also added to the earlier event, {FP32_PER_S:g} per "
                              "self-excitation term), over the slowest rank's mean sweep "
                              "duration",
                     "peak_source": f"{sm_count} SMs x 128 FP32 lanes x {max_mhz:.0f} MHz "
                                    f"(sm_max_mhz, {peak_src})",
                     "sweep_ms": sweep_max},
        "e2e": {"value": pairs / e2e_s, "unit": UNIT, "h2d_bytes_per_step": w["h2d"],
                "d2h_bytes_per_step": w["d2h"]},
        "gpu_launches": launches * args.steps,
        "clocks": clock_summary,
    }
    print(json.dumps(out))
    return 0


def sampler_arm(args):
    """--workload sampler: iterations per second of the reference's MCMC
    sampler (R/Untitled.R:254-422) over 16 chains on the headline events
    (N = 100,000), chains at the base parameters with tauX and tauT fixed as
    the reference keeps them: the host driver, the graph-replayed device
    driver, and the host driver on an engine that keeps no sums (every
    iteration a full sweep of every chain).  One process, one GPU."""
    import torch

    import hawkes_b200 as hb

    w = make_workload("headline", args.n)
    loc, t, base = w["loc"], w["t"], w["params"]
    K = 16
    its = max(3, args.steps // 10)
    init = np.tile(base, (K, 1))
    arms = {}
    with ClockSampler() as clocks:
        for name, flags, device in (("host", hb.CUDA | hb.COMPENSATED, False),
                                    ("device", hb.CUDA | hb.COMPENSATED, True),
                                    ("host_no_reuse",
                                     hb.CUDA | hb.COMPENSATED | hb.NO_INCREMENTAL, False)):
            with hb.CudaHawkes(2, len(t), flags, 0) as e:
                e.setTimesData(t)
                e.updateLocations(-1, loc)
                e.setParameters(base)
                with hb.Sampler(init, radius=0.3, seed=SEED) as s:
                    s.run(e, args.warmup, device=device)
                    n = its if name != "host_no_reuse" else max(3, its // 10)
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    s.run(e, n, device=device)
                    torch.cuda.synchronize()
                    arms[name] = (time.perf_counter() - t0) / n
    out = {
        "metric": f"sampler iterations/s, {K} chains, N={args.n} (FP32-compensated)",
        "value": 1.0 / arms["device"], "unit": "iterations/s", "n_gpus": 1, "steps": its,
        "warmup": args.warmup, "ms_per_step": 1e3 * arms["device"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "data": "synthetic",
        "dtype": "f32 pair terms (compensated), f64 reductions",
        "config": {"workload": w["desc"] + f"; {K} chains at the base parameters, random-scan "
                   "proposals of sigma, omega, theta, mu0 (radius 0.3)", "chains": K},
        "ms_per_iteration": {k: 1e3 * v for k, v in arms.items()},
        "clocks": clocks.summary(None),
    }
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=N_EVENTS, help=argparse.SUPPRESS)
    ap.add_argument("--workload", default="headline",
                    choices=("headline", "batched", "uneven", "clustered", "sampler"),
                    help="headline (default): the metric's N=100k workload; the others are "
                         "the batched-proposal, uneven-set and clustered configurations")
    ap.add_argument("--steps64", type=int, default=0,
                    help="timed steps of the FP64 comparison (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="",
                    help="fix the sweep shape as R:ITEMS_PER_SM instead of autotuning it "
                         "(e.g. to profile one shape)")
    ap.add_argument("--shard", action="store_true",
                    help="split the one N=100k evaluation across the ranks (strong scaling) "
                         "instead of one replica per rank")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.shard:
        return shard_arm(args)
    if args.workload == "sampler":
        return sampler_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
