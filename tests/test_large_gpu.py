"""A million events: ten times the headline size, 1e12 ordered pairs per
evaluation.  The FP32-compensated and FP64 engines must agree to the FP32
mode's accuracy (log-likelihood, gradient, P_i) at that size, where every
count and offset is large (1e6 events, ~7,800 tiles, column sums over a
million rows).  Sweep shapes are fixed so that no autotuning runs."""
import numpy as np
import pytest

import hawkes_b200 as hb
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu


def test_one_million_events_fp32c_matches_fp64():
    n = 1000000
    loc, t = workloads.uniform(n, seed=70)
    p = np.asarray(workloads.BASE_PARAMS)
    out = {}
    for name, flags, shape in (("fp64", hb.CUDA, (2, 32)),
                               ("fp32c", hb.CUDA | hb.COMPENSATED, (4, 64))):
        with hb.CudaHawkes(2, n, flags, 0) as e:
            e.setSweepShape(*shape)
            e.setTimesData(t)
            e.updateLocations(-1, loc)
            e.setParameters(p)
            ll, g = e.getLogLikelihoodAndGradient()
            probs = e.getProbsSelfExcite()
            _, nb, ns = e.lastLaunchStats()
        out[name] = (ll, np.asarray(g), probs)
        assert np.isfinite(ll) and np.all(np.isfinite(g))
        assert probs.shape == (n,) and np.all((probs >= 0) & (probs <= 1))
    (l64, g64, p64), (l32, g32, p32) = out["fp64"], out["fp32c"]
    assert abs(l32 - l64) <= 1e-8 * abs(l64)
    np.testing.assert_allclose(g32, g64, rtol=1e-6)
    assert np.max(np.abs(p32 - p64)) <= 1e-6
