"""The multi-chain sampler on the CUDA engine: every iteration's K proposals
go through one batched likelihood run (hphc_sampler_run).  The chains must be
the ones the same driver produces with the CPU oracle as its evaluator (same
seed, so the same proposals; the FP64 engine's log-likelihoods agree with the
oracle to ~1e-13, so every accept decision is the same), and the R-style
wrapper must return the reference's shapes."""
import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu


def test_engine_chains_match_oracle_chains():
    loc, t = workloads.uniform(900, seed=41)
    base = np.asarray(workloads.BASE_PARAMS)
    init = np.stack([base * np.exp(0.2 * z) for z in np.random.default_rng(5).standard_normal(
        (6, 6))])
    with hb.CudaHawkes(2, len(t), hb.CUDA, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(base)
        with hb.Sampler(init, radius=0.4, seed=99) as s:
            samples, targets = s.run(e, 80, burnIn=10)
            state = s.state()
        # the engine's own parameters are untouched
        assert abs(e.getSumOfLikContribs() - oracle.oracle_eval(loc, t, base)["loglik"]) <= \
            1e-10 * abs(oracle.oracle_eval(loc, t, base)["loglik"])

    def f(P):
        return np.array([oracle.oracle_eval(loc, t, p, threads=2)["loglik"] for p in P])

    with hb.Sampler(init, radius=0.4, seed=99) as s:
        ref_samples, ref_targets = s.run(f, 80, burnIn=10)
    np.testing.assert_array_equal(samples, ref_samples)
    np.testing.assert_allclose(targets, ref_targets, rtol=1e-10)
    assert np.all(state["accepted"] > 0)


def test_fp32_engine_runs_chains():
    loc, t = workloads.uniform(2000, seed=42)
    base = np.asarray(workloads.BASE_PARAMS)
    with hb.CudaHawkes(2, len(t), hb.CUDA | hb.COMPENSATED, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        with hb.Sampler(np.tile(base, (16, 1)), radius=0.3, seed=1) as s:
            samples, targets = s.run(e, 40)
    assert samples.shape == (16, 40, 6) and np.all(np.isfinite(targets))
    # 16 independent streams: the chains differ
    assert len({tuple(x) for x in samples[:, -1, :]}) > 1


def test_r_style_sampler_wrapper():
    loc, t = workloads.uniform(500, seed=43)
    out = hb.sampler(30, burnIn=5, locations=loc, times=t, radius=2, gpu=1)
    assert out["samples"].shape == (6, 25) and out["target"].shape == (25,)
    assert out["Time"] > 0
    out4 = hb.sampler(12, locations=loc, times=t, chains=4, seed=3)
    assert out4["samples"].shape == (4, 6, 12) and out4["target"].shape == (4, 12)


@pytest.mark.parametrize("flags", [hb.CUDA, hb.CUDA | hb.COMPENSATED], ids=["fp64", "fp32c"])
def test_device_driver_matches_host_driver(flags):
    # The same chains from one replayed CUDA graph per iteration: the same
    # random streams and kernels, differing only in last-bit rounding of the
    # device math library and in the summation order of the device loop's
    # wider work list.
    loc, t = workloads.uniform(1500, seed=44)
    base = np.asarray(workloads.BASE_PARAMS)
    init = np.stack([base * np.exp(0.2 * z) for z in np.random.default_rng(6).standard_normal(
        (8, 6))])
    with hb.CudaHawkes(2, len(t), flags, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        with hb.Sampler(init, radius=0.4, seed=7) as a:
            sh, th = a.run(e, 60, burnIn=5)
            ah = a.state()
        with hb.Sampler(init, radius=0.4, seed=7) as b:
            sd1, td1 = b.run(e, 30, burnIn=5, device=True)
            sd2, td2 = b.run(e, 30, device=True)  # continues the same chains
            bd = b.state()
    np.testing.assert_allclose(np.concatenate([sd1, sd2], axis=1), sh, rtol=1e-9)
    np.testing.assert_allclose(np.concatenate([td1, td2], axis=1), th, rtol=1e-8)
    np.testing.assert_array_equal(bd["accepted"], ah["accepted"])
    np.testing.assert_array_equal(bd["proposed"], ah["proposed"])
    np.testing.assert_allclose(bd["radii"], ah["radii"], rtol=1e-12)


def test_device_driver_rejects_sampled_precisions_and_times_itself():
    import time
    loc, t = workloads.uniform(1000, seed=45)
    base = np.asarray(workloads.BASE_PARAMS)
    with hb.CudaHawkes(2, len(t), hb.CUDA | hb.COMPENSATED, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        with hb.Sampler(base, sampled=(0, 1), seed=1) as s:
            with pytest.raises(hb.HawkesError):
                s.run(e, 5, device=True)
        init = np.tile(base, (16, 1))
        rates = {}
        for device in (False, True):
            with hb.Sampler(init, radius=0.3, seed=2) as s:
                s.run(e, 5, device=device)  # warm-up: autotune, graph
                t0 = time.perf_counter()
                s.run(e, 300, device=device)
                rates[device] = (time.perf_counter() - t0) / 300
    print(f"\nsampler iteration, N=1000, 16 chains: host driver {1e6 * rates[False]:.1f} us, "
          f"device driver {1e6 * rates[True]:.1f} us")
    assert rates[True] < rates[False]
