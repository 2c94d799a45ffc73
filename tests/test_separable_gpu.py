"""Reuse of kept unit sums by parameter group.  The background sums depend on
the events, tauX and tauT only; the self-excitation sums on the events, sigma
and omega; theta and mu0 enter only the finish.  So after an evaluation a
theta or mu0 change needs only the O(N) finish (PATH_KEPT_SUMS) and a sigma or
omega change only the self-excitation terms (PATH_SELF_EXCITATION).  Every
result must equal a sweep-only engine's (NO_INCREMENTAL) to rounding, along a
random-scan sequence like the reference's sampler (R/Untitled.R:318-414,
which keeps tauX and tauT fixed) and for batched proposals; the device-time
entry point must still sweep everything."""
import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

FP64, FP32C = hb.CUDA, hb.CUDA | hb.COMPENSATED


def _engine(loc, t, p, flags):
    e = hb.CudaHawkes(2, len(t), flags, 0)
    e.setTimesData(t)
    e.updateLocations(-1, loc)
    e.setParameters(p)
    return e


def _close(flags, a, b, scale):
    (la, ga), (lb, gb) = a, b
    if flags == FP64:
        assert abs(la - lb) <= 1e-12 * abs(lb)
        assert np.all(np.abs(ga - gb) <= 1e-11 * scale)
    else:  # both within the FP32 mode's accuracy of each other
        assert abs(la - lb) <= 2e-9 * abs(lb)
        assert np.all(np.abs(ga - gb) <= 2e-8 * scale)


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_random_scan_sequence_matches_full_sweeps(flags):
    loc, t = workloads.uniform(8000, seed=30)
    p = np.asarray(workloads.BASE_PARAMS, dtype=float).copy()
    scale = oracle.oracle_eval(loc, t, p, threads=4)["grad_scale"]
    rng = np.random.default_rng(31)
    seen = set()
    with _engine(loc, t, p, flags) as e, _engine(loc, t, p, flags | hb.NO_INCREMENTAL) as ref:
        e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_SWEEP
        for _ in range(24):
            k = int(rng.choice([0, 3, 4, 5]))  # sigma, omega, theta, mu0
            p[k] *= float(np.exp(0.2 * rng.standard_normal()))
            e.setParameters(p)
            ref.setParameters(p)
            got = e.getLogLikelihoodAndGradient()
            path = e.lastEvaluationPath
            seen.add(path)
            assert path == (hb.PATH_SELF_EXCITATION if k in (0, 3) else hb.PATH_KEPT_SUMS)
            _close(flags, got, ref.getLogLikelihoodAndGradient(), scale)
        # P_i from the kept sums of the last step
        np.testing.assert_allclose(e.getProbsSelfExcite(), ref.getProbsSelfExcite(),
                                   rtol=1e-10 if flags == FP64 else 1e-7, atol=1e-13)
        # a tauT change needs the full sweep again
        p[2] *= 1.1
        e.setParameters(p)
        e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_SWEEP
    assert seen == {hb.PATH_SELF_EXCITATION, hb.PATH_KEPT_SUMS}


def test_self_excitation_sweep_evaluates_no_background_term():
    loc, t = workloads.uniform(20000, seed=32)
    p = np.asarray(workloads.BASE_PARAMS, dtype=float).copy()
    with _engine(loc, t, p, FP32C) as e:
        e.getLogLikelihoodAndGradient()
        _, nb_full, ns_full = e.lastLaunchStats()
        p[3] *= 1.3  # omega
        e.setParameters(p)
        e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_SELF_EXCITATION
        _, nb, ns = e.lastLaunchStats()
        # no background term; the self-excitation band is about the full
        # sweep's (omega changed), which had ~18x more background terms (the
        # exact ratio depends on the strip shape the autotuner picks)
        assert nb == 0.0 and 0.9 * ns_full < ns <= 1.1 * ns_full and nb_full > 10 * ns_full


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_batched_proposals_with_fixed_tau_reuse_the_background(flags):
    loc, t = workloads.uniform(6000, seed=33)
    base = np.asarray(workloads.BASE_PARAMS, dtype=float)
    scale = oracle.oracle_eval(loc, t, base, threads=4)["grad_scale"]
    z = np.random.default_rng(34).standard_normal((8, 6))
    z[:, 1:3] = 0.0  # tauX, tauT fixed, as in the reference's sampler
    P = base * np.exp(0.2 * z)
    with _engine(loc, t, base, flags) as e, _engine(loc, t, base, flags | hb.NO_INCREMENTAL) as ref:
        e.getLogLikelihoodAndGradient()
        ll, g = e.batchLogLikelihoodAndGradient(P)
        assert e.lastEvaluationPath == hb.PATH_SELF_EXCITATION
        llr, gr = ref.batchLogLikelihoodAndGradient(P)
        for k in range(len(P)):
            _close(flags, (ll[k], g[k]), (llr[k], gr[k]), scale)
        # the batch keeps proposal 0's sums: a theta change of it is O(N)
        q = P[0].copy()
        q[4] *= 1.2
        e.setParameters(q)
        ref.setParameters(q)
        got = e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS
        _close(flags, got, ref.getLogLikelihoodAndGradient(), scale)
        # proposals that move tauT need the full sweep
        P2 = P.copy()
        P2[3, 2] *= 1.05
        e.batchLogLikelihoodAndGradient(P2)
        assert e.lastEvaluationPath == hb.PATH_SWEEP


def test_device_time_entry_point_always_sweeps_everything():
    loc, t = workloads.uniform(5000, seed=35)
    with _engine(loc, t, workloads.BASE_PARAMS, FP32C) as e:
        for _ in range(3):
            e.enqueueLogLikelihoodAndGradient()
            e.readResults()
            assert e.lastEvaluationPath == hb.PATH_SWEEP
            assert e.lastLaunchStats()[1] > 0  # background terms evaluated


def test_sampler_step_cost_by_path():
    import time
    loc, t = workloads.uniform(100000, seed=36)
    p = np.asarray(workloads.BASE_PARAMS, dtype=float).copy()
    with _engine(loc, t, p, FP32C) as e:
        e.getLogLikelihoodAndGradient()
        times = {}
        for name, k in (("sweep", 2), ("self-excitation", 3), ("kept sums", 4)):
            for _ in range(3):  # warm-up
                p[k] *= 1.001
                e.setParameters(p)
                e.getLogLikelihoodAndGradient()
            t0 = time.perf_counter()
            for _ in range(10):
                p[k] *= 1.001
                e.setParameters(p)
                e.getLogLikelihoodAndGradient()
            times[name] = (time.perf_counter() - t0) / 10 * 1e3
    print(f"\nN=100k FP32-compensated, ms per evaluation: " +
          ", ".join(f"{k} {v:.3f}" for k, v in times.items()))
    assert times["self-excitation"] < 0.25 * times["sweep"]
    assert times["kept sums"] < times["self-excitation"]


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_samplers_with_fixed_tau_reuse_the_background(flags):
    # Chains sharing tauX and tauT: the host driver's batched evaluations and
    # the device driver's replayed iteration both sweep only the
    # self-excitation terms, and must give the same chains.
    loc, t = workloads.uniform(3000, seed=37)
    base = np.asarray(workloads.BASE_PARAMS, dtype=float)
    z = np.random.default_rng(38).standard_normal((8, 6))
    z[:, 1:3] = 0.0
    init = base * np.exp(0.2 * z)
    with _engine(loc, t, base, flags) as e:
        with hb.Sampler(init, radius=0.4, seed=9) as a:
            sh, th = a.run(e, 40, burnIn=5)
        assert e.lastEvaluationPath == hb.PATH_SELF_EXCITATION
        with hb.Sampler(init, radius=0.4, seed=9) as b:
            sd, td = b.run(e, 40, burnIn=5, device=True)
            acc = b.state()["accepted"]
    np.testing.assert_allclose(sd, sh, rtol=1e-9)
    np.testing.assert_allclose(td, th, rtol=1e-8)
    assert np.all(acc > 0)


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_device_loop_band_search_with_blocks_of_equal_times(flags):
    # Times in blocks of 1280 equal values, 2 h apart: the tiles just before a
    # strip share its time (no causal pair, no self-excitation term) while
    # the block before them holds terms.  The device loop's plan lists every
    # earlier tile and finds where to start by bisection on the tile time
    # bounds; it must keep those earlier terms, as the host driver's
    # host-planned bands do.
    n = 6400
    rng = np.random.default_rng(39)
    loc = rng.uniform(0.0, 20.0, size=(n, 2))
    t = (np.arange(n) // 1280) * 2.0
    base = np.asarray(workloads.BASE_PARAMS, dtype=float)
    z = rng.standard_normal((8, 6))
    z[:, 1:3] = 0.0
    init = base * np.exp(0.2 * z)
    with _engine(loc, t, base, flags) as e:
        with hb.Sampler(init, radius=0.4, seed=11) as a:
            sh, th = a.run(e, 30, burnIn=2)
        with hb.Sampler(init, radius=0.4, seed=11) as b:
            sd, td = b.run(e, 30, burnIn=2, device=True)
    np.testing.assert_allclose(sd, sh, rtol=1e-9)
    np.testing.assert_allclose(td, th, rtol=1e-8)
    # and with chains whose tauX, tauT differ (no kept background: the device
    # loop sweeps both kinds of terms over its wide bands)
    init2 = base * np.exp(0.2 * rng.standard_normal((8, 6)))
    with _engine(loc, t, base, flags) as e:
        with hb.Sampler(init2, radius=0.4, seed=12) as a:
            sh, th = a.run(e, 20)
        with hb.Sampler(init2, radius=0.4, seed=12) as b:
            sd, td = b.run(e, 20, device=True)
    np.testing.assert_allclose(sd, sh, rtol=1e-9)
    np.testing.assert_allclose(td, th, rtol=1e-8)


@pytest.mark.parametrize("D", [1, 3])
@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_reuse_in_other_dimensions(flags, D):
    loc, t = workloads.uniform(3000, seed=60 + D, D=D)
    p = np.asarray(workloads.BASE_PARAMS, dtype=float).copy()
    scale = oracle.oracle_eval(loc, t, p, threads=4)["grad_scale"]

    def make(fl):
        e = hb.CudaHawkes(D, len(t), fl, 0)
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(p)
        return e

    with make(flags) as e, make(flags | hb.NO_INCREMENTAL) as ref:
        e.getLogLikelihoodAndGradient()
        for k, f in ((0, 1.2), (4, 0.8), (3, 1.3), (5, 1.1)):
            p[k] *= f
            e.setParameters(p)
            ref.setParameters(p)
            got = e.getLogLikelihoodAndGradient()
            assert e.lastEvaluationPath == (hb.PATH_SELF_EXCITATION if k in (0, 3)
                                            else hb.PATH_KEPT_SUMS)
            _close(flags, got, ref.getLogLikelihoodAndGradient(), scale)
