"""Large inputs through the host's O(N) passes (finite check, copy into the
pinned mirror, dense time ranks).  With times on whole hours (about 34 events
share each hour), a wrong rank would let equal-time pairs count as causal in
the FP32 mode's self-excitation mask, a large error against the FP64 mode,
which tests dt > 0 on the times themselves.  A rejected input must leave the
engine's events as they were."""
import numpy as np
import pytest

import hawkes_b200 as hb
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu


def test_tied_times_at_split_sizes():
    n = 300000
    loc, t = workloads.uniform(n, seed=40)
    t = np.floor(t)  # whole hours: long runs of ties
    p = np.asarray(workloads.BASE_PARAMS)
    out = {}
    for name, flags in (("fp64", hb.CUDA), ("fp32c", hb.CUDA | hb.COMPENSATED)):
        with hb.CudaHawkes(2, n, flags, 0) as e:
            e.setTimesData(t)
            e.updateLocations(-1, loc)
            e.setParameters(p)
            out[name] = e.getLogLikelihoodAndGradient()
            probs = e.getProbsSelfExcite()
            assert np.all(np.isfinite(probs)) and probs.shape == (n,)
    (l64, g64), (l32, g32) = out["fp64"], out["fp32c"]
    assert abs(l32 - l64) <= 1e-8 * abs(l64)
    np.testing.assert_allclose(g32, g64, rtol=1e-6)


def test_rejected_large_input_changes_nothing():
    n = 300000
    loc, t = workloads.uniform(n, seed=41)
    bad = loc.copy()
    bad[n - 7, 1] = np.inf
    with hb.CudaHawkes(2, n, hb.CUDA, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(workloads.BASE_PARAMS)
        ll0 = e.getSumOfLikContribs()
        with pytest.raises(hb.HawkesError) as ei:
            e.updateLocations(-1, bad)
        assert ei.value.status == 4 and str(2 * (n - 7) + 1) in str(ei.value)
        assert e.getSumOfLikContribs() == ll0
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS


def test_ranks_follow_sorted_and_unsorted_times():
    # Sorted times get their dense ranks on the device, unsorted ones from the
    # host: switching between the two on one engine must match fresh engines.
    n = 20000
    loc, t = workloads.uniform(n, seed=42)
    tied = np.floor(t / 3.0) * 3.0
    rng = np.random.default_rng(43)
    perm = rng.permutation(n - 1)  # the last event keeps the latest time (T)
    shuffled_t = np.concatenate([tied[:-1][perm], tied[-1:]])
    shuffled_loc = np.concatenate([loc[:-1][perm], loc[-1:]])
    p = np.asarray(workloads.BASE_PARAMS)
    cases = [(tied, loc), (shuffled_t, shuffled_loc), (t, loc), (tied, loc)]

    def run(e, tt, ll):
        e.setTimesData(tt)
        e.updateLocations(-1, ll)
        e.setParameters(p)
        return e.getLogLikelihoodAndGradient()

    with hb.CudaHawkes(2, n, hb.CUDA | hb.COMPENSATED, 0) as e:
        got = [run(e, tt, ll) for tt, ll in cases]
    for (tt, ll), (lg, gg) in zip(cases, got):
        with hb.CudaHawkes(2, n, hb.CUDA | hb.COMPENSATED, 0) as f:
            lf, gf = run(f, tt, ll)
        assert lg == lf and np.array_equal(gg, gf)
    # the permuted events are the same set: equal up to summation order
    assert abs(got[1][0] - got[0][0]) <= 5e-9 * abs(got[0][0])
