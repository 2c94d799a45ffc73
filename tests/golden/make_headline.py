"""Generate tests/golden/headline_n100k.npz: the expected results of the
headline workload (N = 100,000 events, D = 2, 20x20 km box, times U[0,8760) h
sorted, numpy default_rng(5), base parameters).

    python tests/golden/make_headline.py [--threads 8]

The events are regenerated from the seed by ``workloads.uniform`` (checksums
of the inputs are stored to detect a generator that drifted), so the fixture
holds only outputs:

* ``oracle_*`` -- the C restatement (oracle/hawkes_oracle.c, long-double
  sums): log-likelihood, analytic gradient, its per-event and term-level
  scales, and the probabilities P_i of every 50th event;
* ``ref_*`` -- the reference hpHawkes CPU engine compiled from its own sources
  (src/NewHawkes.hpp, DOUBLE, threaded through the std::thread stub) when
  oracle/_ref is built: its log-likelihood (src/NewHawkes.hpp:636-660) and
  the same P_i subset (src/NewHawkes.hpp:662-719), which pin the oracle at
  this size.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

N, SEED, STRIDE = 100000, 5, 50


def load_workloads():
    spec = importlib.util.spec_from_file_location(
        "_hawkes_workloads", os.path.join(ROOT, "hawkes_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def input_checksums(loc, t):
    return np.array([t.sum(), t[0], t[-1], loc[:, 0].sum(), loc[:, 1].sum()])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    wl = load_workloads()
    loc, t = wl.uniform(N, seed=SEED)
    p = wl.BASE_PARAMS.copy()
    out = {"N": np.int64(N), "seed": np.int64(SEED), "params": p,
           "input_checksums": input_checksums(loc, t),
           "probs_index": np.arange(0, N, STRIDE)}
    t0 = time.time()
    o = oracle.oracle_eval(loc, t, p, threads=args.threads)
    print(f"oracle: {time.time() - t0:.1f} s, loglik {o['loglik']!r}")
    out.update({"oracle_loglik": np.float64(o["loglik"]), "oracle_grad": o["grad"],
                "grad_scale": o["grad_scale"], "grad_term_scale": o["grad_term_scale"],
                "oracle_probs": o["probs"][::STRIDE], "oracle_probs_sum": np.float64(
                    o["probs"].sum())})
    if oracle.ref_available():
        eng = oracle.RefEngine(2, N, threads=args.threads)
        eng.set_data(loc, t)
        eng.set_parameters(p)
        t0 = time.time()
        ll = eng.loglik()
        print(f"reference: {time.time() - t0:.1f} s, loglik {ll!r} "
              f"(oracle rel {abs(ll - o['loglik']) / abs(ll):.2e}) [{eng.variant.splitlines()[0]}]")
        pr = eng.probs()
        eng.close()
        out.update({"ref_loglik": np.float64(ll), "ref_probs": pr[::STRIDE],
                    "ref_probs_sum": np.float64(pr.sum())})
        print(f"probs: max |ref - oracle| {np.max(np.abs(pr - o['probs'])):.2e}")
    np.savez_compressed(os.path.join(HERE, "headline_n100k.npz"), **out)


if __name__ == "__main__":
    main()
