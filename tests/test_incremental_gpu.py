"""Incremental evaluation: after an evaluation the engine keeps every event's
six unit pair sums; moving a few events (updateLocations with an index, the
reference CLI's per-row updates and BEAST's location proposals) at unchanged
parameters updates them in O(N) per moved event instead of re-running the
O(N^2) sweep.  Each result is checked against the oracle on the moved data
and against a sweep-only engine (HPHC_FLAG_NO_INCREMENTAL); the path each
evaluation took is read back through the C ABI.

Tolerances: FP64 as the parity tests (1e-10 vs the oracle) and 1e-12 relative
vs the sweep-only FP64 engine (the updates add FP64 rounding only); FP32
compensated as its small-size parity bars (loglik 1e-7, gradient 5e-6 of the
term-level scale, probabilities 2e-5).
"""
import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

FP64 = hb.CUDA
FP32C = hb.CUDA | hb.COMPENSATED


def make(loc, t, p, flags):
    e = hb.CudaHawkes(loc.shape[1], len(t), flags, 0)
    e.setTimesData(t)
    e.updateLocations(-1, loc)
    e.setParameters(p)
    return e


def check(e, loc, t, p, flags):
    ll, g = e.getLogLikelihoodAndGradient()
    o = oracle.oracle_eval(loc, t, p, threads=4)
    if flags == FP64:
        assert abs(ll - o["loglik"]) <= 1e-10 * abs(o["loglik"])
        assert np.all(np.abs(g - o["grad"]) <= 1e-10 * o["grad_scale"])
    else:
        assert abs(ll - o["loglik"]) <= 1e-7 * abs(o["loglik"])
        assert np.all(np.abs(g - o["grad"]) <= 5e-6 * o["grad_term_scale"])
    return ll, g


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_moves_update_in_place(flags):
    rng = np.random.default_rng(8)
    loc, t = workloads.uniform(3000, seed=51)
    p = np.asarray(workloads.BASE_PARAMS)
    with make(loc, t, p, flags) as e, make(loc, t, p, flags | hb.NO_INCREMENTAL) as ref:
        ll0, g0 = check(e, loc, t, p, flags)
        assert e.lastEvaluationPath == hb.PATH_SWEEP
        # nothing changed: the finish runs on the kept sums, bit for bit the same
        ll1, g1 = e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS
        assert ll1 == ll0 and np.array_equal(g1, g0)
        # move three events (one of them twice)
        for k in (5, 1700, 2999, 5):
            loc[k] = rng.uniform(0, 20, size=2)
            e.updateLocations(k, loc[k])
            ref.updateLocations(k, loc[k])
        ll2, g2 = check(e, loc, t, p, flags)
        assert e.lastEvaluationPath == hb.PATH_INCREMENTAL
        ll3, g3 = ref.getLogLikelihoodAndGradient()
        assert ref.lastEvaluationPath == hb.PATH_SWEEP
        if flags == FP64:
            assert abs(ll2 - ll3) <= 1e-12 * abs(ll3)
            assert np.all(np.abs(g2 - g3) <= 1e-12 * np.abs(g3) + 1e-9)
        probs = e.getProbsSelfExcite()
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS
        tol = 1e-10 if flags == FP64 else 2e-5
        np.testing.assert_allclose(probs, oracle.oracle_eval(loc, t, p)["probs"], rtol=0,
                                   atol=tol)


def test_many_moves_keep_fp64_accuracy():
    rng = np.random.default_rng(9)
    loc, t = workloads.uniform(2000, seed=52)
    p = np.asarray(workloads.BASE_PARAMS)
    with make(loc, t, p, FP64) as e:
        e.getSumOfLikContribs()
        for step in range(150):
            k = int(rng.integers(0, len(t)))
            loc[k] = loc[k] + rng.normal(0, 0.5, size=2)
            e.updateLocations(k, loc[k])
            e.getSumOfLikContribs()
            assert e.lastEvaluationPath == hb.PATH_INCREMENTAL
        check(e, loc, t, p, FP64)


def test_fallbacks_to_the_sweep():
    loc, t = workloads.uniform(2048, seed=53)
    p = np.asarray(workloads.BASE_PARAMS)
    with make(loc, t, p, FP64) as e:
        e.getSumOfLikContribs()
        # new parameters
        q = p * 1.1
        e.setParameters(q)
        check(e, loc, t, q, FP64)
        assert e.lastEvaluationPath == hb.PATH_SWEEP
        # more moved events than the incremental path takes (N / 512 = 4 here)
        for k in range(6):
            loc[k] += 0.3
            e.updateLocations(k, loc[k])
        check(e, loc, t, q, FP64)
        assert e.lastEvaluationPath == hb.PATH_SWEEP
        # a new time set
        t2 = np.sort(t + 0.25)
        e.setTimesData(t2)
        check(e, loc, t2, q, FP64)
        assert e.lastEvaluationPath == hb.PATH_SWEEP
        # a batch keeps its first parameter vector's sums (here the engine's own)
        e.batchLogLikelihoodAndGradient(np.stack([q, p]))
        e.getSumOfLikContribs()
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_store_restore_brings_back_the_sums(flags):
    loc, t = workloads.uniform(2500, seed=54)
    p = np.asarray(workloads.BASE_PARAMS)
    with make(loc, t, p, flags) as e:
        ll0, g0 = e.getLogLikelihoodAndGradient()
        e.storeState()
        moved = loc.copy()
        moved[100] += [1.0, -2.0]
        e.updateLocations(100, moved[100])
        check(e, moved, t, p, flags)
        assert e.lastEvaluationPath == hb.PATH_INCREMENTAL
        e.restoreState()   # proposal rejected
        ll1, g1 = e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS
        assert ll1 == ll0 and np.array_equal(g1, g0)
        check(e, loc, t, p, flags)
        # and the next proposal moves from the restored locations
        moved2 = loc.copy()
        moved2[7] += [0.5, 0.5]
        e.updateLocations(7, moved2[7])
        check(e, moved2, t, p, flags)
        assert e.lastEvaluationPath == hb.PATH_INCREMENTAL
