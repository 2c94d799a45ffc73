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
