"""GPU tests on clustered data: N = 500,000 events from a Hawkes branching
process (background Poisson in a 50 x 50 km box over [0, 8760) h, Poisson(0.5)
offspring with N(0, 0.25 km^2) spatial and Exp(1 / h) temporal offsets).

The FP64 oracle runs on the first 50,000 events by time (that subset's T is
its own last time); the full 500,000 are checked FP32-compensated against the
FP64 engine.
"""
import os

import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import workloads

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


@pytest.fixture(scope="module")
def clustered():
    return workloads.clustered()


def evaluate(loc, t, p, flags):
    with hb.CudaHawkes(2, len(t), flags, 0) as e:
        e.setSweepShape(2 if flags == hb.CUDA else 4, 32)
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(p)
        return e.getLogLikelihoodAndGradient()


def test_clustered_subset_vs_oracle(clustered):
    loc, t = clustered
    loc, t = loc[:50000], t[:50000]
    p = workloads.BASE_PARAMS
    o = oracle.oracle_eval(loc, t, p, threads=max(1, os.cpu_count() or 1))
    ll64, g64 = evaluate(loc, t, p, hb.CUDA)
    ll32, g32 = evaluate(loc, t, p, hb.CUDA | hb.COMPENSATED)
    assert abs(ll64 - o["loglik"]) <= 1e-10 * abs(o["loglik"])
    assert np.all(np.abs(g64 - o["grad"]) <= 1e-10 * o["grad_scale"])
    assert abs(ll32 - o["loglik"]) <= 1e-8 * abs(o["loglik"])
    assert np.all(np.abs(g32 - o["grad"]) <= 1e-8 * o["grad_scale"])


def test_clustered_full_fp32_vs_fp64(clustered):
    loc, t = clustered
    assert len(t) == 500000
    p = workloads.BASE_PARAMS
    ll64, g64 = evaluate(loc, t, p, hb.CUDA)
    ll32, g32 = evaluate(loc, t, p, hb.CUDA | hb.COMPENSATED)
    assert np.isfinite(ll64) and abs(ll32 - ll64) <= 1e-8 * abs(ll64)
    assert np.all(np.abs(g32 - g64) <= 1e-6 * (np.abs(g64) + 1e-3 * np.max(np.abs(g64))))
