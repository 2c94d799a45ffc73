"""Error propagation and recovery, tested with host-side fakes
(hphc_inject_fault) instead of a GPU fault: an injected failure at the
upload, the graph launch or the completion wait must come back as the mapped
status with "injected" in the message, and the engine's next calls must give
the same bits as an engine that never failed (the kept sums are not trusted
after a failure)."""
import numpy as np
import pytest

import hawkes_b200 as hb
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

STAGES = [(hb.FAULT_UPLOAD, 10), (hb.FAULT_LAUNCH, 6), (hb.FAULT_WAIT, 6)]


def _engine(loc, t, p, flags):
    e = hb.CudaHawkes(2, len(t), flags, 0)
    e.setTimesData(t)
    e.updateLocations(-1, loc)
    e.setParameters(p)
    return e


@pytest.mark.parametrize("flags", [hb.CUDA, hb.CUDA | hb.COMPENSATED], ids=["fp64", "fp32c"])
@pytest.mark.parametrize("stage,status", STAGES, ids=["upload", "launch", "wait"])
def test_injected_fault_is_reported_and_the_engine_recovers(flags, stage, status):
    loc, t = workloads.uniform(3000, seed=20)
    p = workloads.BASE_PARAMS.copy()
    q = p * np.array([1.1, 1.0, 1.0, 0.9, 1.0, 1.05])
    with _engine(loc, t, q, flags) as ref:
        llq, gq = ref.getLogLikelihoodAndGradient()
    with _engine(loc, t, p, flags) as e:
        e.getLogLikelihoodAndGradient()
        e.setParameters(q)  # new parameters: the next call must sweep
        if stage == hb.FAULT_UPLOAD:
            e.updateLocations(-1, loc)  # new events: the next call must upload
        e.injectFault(stage, 1)
        with pytest.raises(hb.HawkesError) as ei:
            e.getLogLikelihoodAndGradient()
        assert ei.value.status == status and "injected" in str(ei.value)
        ll, g = e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_SWEEP
        assert ll == llq and np.array_equal(g, gq)
        pr = e.getProbsSelfExcite()
        assert np.all(np.isfinite(pr))


def test_fault_count_and_clearing():
    loc, t = workloads.uniform(2000, seed=21)
    p = workloads.BASE_PARAMS.copy()
    with _engine(loc, t, p, hb.CUDA | hb.COMPENSATED | hb.NO_INCREMENTAL) as e:
        ll0, _ = e.getLogLikelihoodAndGradient()
        e.injectFault(hb.FAULT_LAUNCH, 2)
        for _ in range(2):
            with pytest.raises(hb.HawkesError):
                e.getLogLikelihoodAndGradient()
        assert e.getLogLikelihoodAndGradient()[0] == ll0
        e.injectFault(hb.FAULT_WAIT, 3)
        e.injectFault(hb.FAULT_WAIT, 0)  # cleared
        assert e.getLogLikelihoodAndGradient()[0] == ll0
        for bad in [(0, 1), (4, 1), (hb.FAULT_LAUNCH, -1)]:
            with pytest.raises(hb.HawkesError) as ei:
                e.injectFault(*bad)
            assert ei.value.status == 3


def test_batched_and_sampler_runs_propagate_and_recover():
    loc, t = workloads.uniform(2000, seed=22)
    base = np.asarray(workloads.BASE_PARAMS)
    P = workloads.proposals(8, seed=5)
    with _engine(loc, t, base, hb.CUDA) as e:
        ll0, g0 = e.batchLogLikelihoodAndGradient(P)
        e.injectFault(hb.FAULT_WAIT, 1)
        with pytest.raises(hb.HawkesError):
            e.batchLogLikelihoodAndGradient(P)
        ll1, g1 = e.batchLogLikelihoodAndGradient(P)
        assert np.array_equal(ll0, ll1) and np.array_equal(g0, g1)
        with hb.Sampler(np.tile(base, (4, 1)), radius=0.3, seed=3) as s:
            e.injectFault(hb.FAULT_LAUNCH, 1)
            with pytest.raises(hb.HawkesError):
                s.run(e, 5)
        with hb.Sampler(np.tile(base, (4, 1)), radius=0.3, seed=3) as s:
            samples, targets = s.run(e, 5)
        assert np.all(np.isfinite(targets))
