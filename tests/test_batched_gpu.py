"""GPU tests of the batched paths: K parameter vectors on one event set (MCMC
proposals) and many event sets of uneven size, each evaluated in one run.

Bars as in test_parity_gpu.py: FP64 plain 1e-10 relative on the
log-likelihood and 1e-10 of the gradient's per-event scale; FP32-compensated
1e-7 / 5e-6 of the term-level scale at small sizes.  A batched result and the
same problem evaluated alone are split into different j-chunks, and the
autotuner may give them different strip heights.  In FP64 that changes only
the order the chunk sums are added (1e-12 relative).  In the
FP32-compensated mode each chunk's compensated FP32 sums start again, with
exact errors, so the chunk bounds move the sums by the rounding of their
error parts alone, and another strip height moves which pairs go to the
FP32 column sums: measured under 1e-15 relative on the log-likelihood and
under 1e-12 of the gradient's per-event scale (2e-10 of |g| on the d/d tauT
component, which cancels ~300-fold); bars 1e-13 and 1e-11 of the per-event
scale.
"""
import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

FP64 = hb.CUDA
FP32C = hb.CUDA | hb.COMPENSATED


def engine(loc, t, flags):
    e = hb.CudaHawkes(loc.shape[1], loc.shape[0], flags, 0)
    e.setTimesData(t)
    e.updateLocations(-1, loc)
    return e


def check_vs_oracle(ll, g, o, flags, tag):
    if flags == FP64:
        assert abs(ll - o["loglik"]) <= 1e-10 * abs(o["loglik"]), tag
        assert np.all(np.abs(g - o["grad"]) <= 1e-10 * o["grad_scale"]), tag
    else:
        assert abs(ll - o["loglik"]) <= 1e-7 * abs(o["loglik"]), tag
        allowed = 5e-6 * o["grad_term_scale"] + 1e-12 * np.max(o["grad_term_scale"])
        assert np.all(np.abs(g - o["grad"]) <= allowed), tag


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_proposals_match_single_evaluations_and_oracle(flags):
    loc, t = workloads.uniform(6000, seed=31)
    P = workloads.proposals(48, seed=32)
    with engine(loc, t, flags) as e:
        ll, g = e.batchLogLikelihoodAndGradient(P)
        for k in (0, 17, 47):
            e.setParameters(P[k])
            lk, gk = e.getLogLikelihoodAndGradient()
            if flags == FP64:
                assert abs(lk - ll[k]) <= 1e-12 * abs(lk)
                assert np.all(np.abs(gk - g[k]) <= 1e-12 * (np.abs(gk) + 1.0))
            else:
                scale = oracle.oracle_eval(loc, t, P[k], threads=16)["grad_scale"]
                assert abs(lk - ll[k]) <= 1e-13 * abs(lk)
                assert np.all(np.abs(gk - g[k]) <= 1e-11 * scale)
    for k in (3, 29):
        o = oracle.oracle_eval(loc, t, P[k], threads=16)
        check_vs_oracle(ll[k], g[k], o, flags, f"proposal {k}")


@pytest.mark.slow
def test_batched_proposals_config():
    # 256 log-normal (sd 0.3) proposals around the base on N = 20,000 events.
    loc, t = workloads.uniform(20000, seed=2)
    P = workloads.proposals(256, seed=2)
    with engine(loc, t, FP32C) as e32, engine(loc, t, FP64) as e64:
        ll32, g32 = e32.batchLogLikelihoodAndGradient(P)
        ll64, g64 = e64.batchLogLikelihoodAndGradient(P)
    assert np.all(np.abs(ll32 - ll64) <= 1e-8 * np.abs(ll64))
    for k in (0, 128, 255):
        o = oracle.oracle_eval(loc, t, P[k], threads=16)
        check_vs_oracle(ll64[k], g64[k], o, FP64, f"fp64 proposal {k}")
        assert abs(ll32[k] - o["loglik"]) <= 1e-8 * abs(o["loglik"])
        assert np.all(np.abs(g32[k] - o["grad"]) <= 1e-8 * o["grad_scale"] +
                      1e-12 * np.max(o["grad_term_scale"]))


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_multiset_small_sets_vs_oracle(flags):
    sets = workloads.uneven(10, seed=41, lo=100, hi=3000)
    with hb.Multiset(2, [len(t) for _, t, _ in sets], flags, 0) as m:
        for s, (loc, t, _) in enumerate(sets):
            m.setData(s, loc, t)
        ll, g = m.logLikelihoodAndGradient(np.stack([p for _, _, p in sets]))
        _, nb, ns = m.lastLaunchStats()
    assert nb > 0
    for s, (loc, t, p) in enumerate(sets):
        o = oracle.oracle_eval(loc, t, p, threads=16)
        check_vs_oracle(ll[s], g[s], o, flags, f"set {s}")


def test_multiset_equals_single_engines():
    sets = workloads.uneven(5, seed=42, lo=500, hi=8000)
    with hb.Multiset(2, [len(t) for _, t, _ in sets], FP32C, 0) as m:
        for s, (loc, t, _) in enumerate(sets):
            m.setData(s, loc, t)
        ll, g = m.logLikelihoodAndGradient(np.stack([p for _, _, p in sets]))
    for s, (loc, t, p) in enumerate(sets):
        with engine(loc, t, FP32C) as e:
            e.setParameters(p)
            l1, g1 = e.getLogLikelihoodAndGradient()
        # the same sums; the autotuner may pick another sweep shape for the
        # multiset than for one set: other strips (which pairs are summed as
        # the FP32 column sums of the symmetric sweep) and other j-chunks
        assert abs(l1 - ll[s]) <= 1e-9 * abs(l1)
        assert np.all(np.abs(g1 - g[s]) <= 1e-7 * (np.abs(g1) + 1.0))


@pytest.mark.slow
def test_uneven_sets_config():
    # 64 sets, sizes log-uniform in [1,000, 100,000], own log-normal parameters.
    sets = workloads.uneven(64, seed=3)
    sizes = [len(t) for _, t, _ in sets]
    params = np.stack([p for _, _, p in sets])
    out = {}
    for flags in (FP32C, FP64):
        with hb.Multiset(2, sizes, flags, 0) as m:
            for s, (loc, t, _) in enumerate(sets):
                m.setData(s, loc, t)
            out[flags] = m.logLikelihoodAndGradient(params)
    ll32, g32 = out[FP32C]
    ll64, g64 = out[FP64]
    assert np.all(np.abs(ll32 - ll64) <= 1e-8 * np.abs(ll64))
    small = [s for s in np.argsort(sizes)[:3]]
    for s in small:
        loc, t, p = sets[s]
        o = oracle.oracle_eval(loc, t, p, threads=16)
        check_vs_oracle(ll64[s], g64[s], o, FP64, f"set {s}")


def test_multiset_errors():
    with hb.Multiset(2, [100, 200], FP64, 0) as m:
        with pytest.raises(hb.HawkesError) as ei:
            m.logLikelihoodAndGradient(np.ones((2, 6)))
        assert ei.value.status == 7  # set data missing
        with pytest.raises(hb.HawkesError) as ei:
            m.setData(0, np.zeros(150), np.zeros(100))
        assert ei.value.status == 2
        with pytest.raises(hb.HawkesError) as ei:
            m.setData(2, np.zeros(400), np.zeros(200))
        assert ei.value.status == 3


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_multiset_rejected_input_leaves_the_set_unchanged(flags):
    # A set that holds data checks new values while copying them into its
    # host mirror and restores the mirror from the device copy when one is
    # not finite; a set without data checks before copying.  Either way the
    # set keeps its previous events.
    sets = workloads.uneven(3, seed=44, lo=300, hi=2000)
    params = np.stack([p for _, _, p in sets])
    with hb.Multiset(2, [len(t) for _, t, _ in sets], flags, 0) as m:
        bad_loc = np.array(sets[0][0], dtype=np.float64)
        bad_loc.reshape(-1)[7] = np.nan
        with pytest.raises(hb.HawkesError) as ei:
            m.setData(0, bad_loc, sets[0][1])
        assert ei.value.status == 4  # non-finite, before the set had data
        for s, (loc, t, _) in enumerate(sets):
            m.setData(s, loc, t)
        ll0, g0 = m.logLikelihoodAndGradient(params)
        other_loc, other_t = workloads.uniform(len(sets[1][1]), seed=45)
        bad_t = np.array(other_t)
        bad_t[-3] = np.inf
        with pytest.raises(hb.HawkesError) as ei:
            m.setData(1, other_loc, bad_t)  # locations copied, then the times rejected
        assert ei.value.status == 4
        loc2, t2 = workloads.uniform(len(sets[2][1]), seed=46)
        loc2 = np.array(loc2, dtype=np.float64)
        loc2.reshape(-1)[-1] = np.nan
        with pytest.raises(hb.HawkesError) as ei:
            m.setData(2, loc2, t2)  # rejected in the locations
        assert ei.value.status == 4
        ll1, g1 = m.logLikelihoodAndGradient(params)
        assert np.array_equal(ll0, ll1) and np.array_equal(g0, g1)
        # accepted new data still replaces the set
        m.setData(1, other_loc, other_t)
        ll2, _ = m.logLikelihoodAndGradient(params)
        assert ll2[1] != ll0[1] and ll2[0] == ll0[0] and ll2[2] == ll0[2]


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_multiset_degenerate_sizes_vs_oracle(flags):
    # single events, block-boundary sizes, tied and unsorted times, each set at
    # its own parameters, all in one run
    rng = np.random.default_rng(43)
    sizes = [1, 2, 3, 31, 127, 128, 129, 300]
    sets = []
    for k, n in enumerate(sizes):
        loc = rng.uniform(0.0, 20.0, size=(n, 2))
        t = np.sort(rng.uniform(0.0, 8760.0, size=n))
        if k == 6:
            t = np.floor(t / 200.0) * 200.0  # ties
        if k == 7:
            # unsorted; the last time stays the largest, since the model's
            # horizon T is the last time given (as in the reference)
            t = np.append(rng.permutation(t[:-1]), t[-1])
        p = np.asarray(workloads.BASE_PARAMS) * np.exp(0.3 * rng.standard_normal(6))
        sets.append((loc, t, p))
    with hb.Multiset(2, sizes, flags, 0) as m:
        for s, (loc, t, _) in enumerate(sets):
            m.setData(s, loc, t)
        ll, g = m.logLikelihoodAndGradient(np.stack([p for _, _, p in sets]))
    for s, (loc, t, p) in enumerate(sets):
        o = oracle.oracle_eval(loc, t, p, threads=4)
        check_vs_oracle(ll[s], g[s], o, flags, f"set {s} (N={sizes[s]})")
