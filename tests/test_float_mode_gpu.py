"""The plain single-precision mode (HPHC_FLAG_FLOAT without COMPENSATED)
against the reference's own float engine and its double engine.

The reference's FLOAT flag (src/factory.cpp:34, :45; OpenCLHawkes.hpp:616-630)
computes everything in float: times and coordinates, pair terms, the
per-event sums, log and CDF.  Its results then move with float rounding, and
on data whose times are hours over a year (dcData) the float time
differences also change which near-simultaneous pairs count as causal.  The
CUDA plain FP32 mode follows the same rules: times rounded to FP32 decide
causality, pair terms from FP32 values with the hardware exponential, plain
FP32 sums, the per-event log/CDF/gradient terms in FP32 (event totals are
FP64, in fixed order).

Bars (the fixtures' ref_float_* fields come from the reference float engine;
ref_* from its double engine):
  synthetic cases   log-likelihood within 5e-6 relative of both the reference
                    float and double results; P_i within 2e-3 absolute of the
                    float engine's; gradient within 1e-3 of the oracle's
                    term-level scale (times of up to 8760 h rounded to float
                    are off by up to 2^-11 h, which moves each
                    self-excitation term by up to omega * 2^-11 ~ 5e-4
                    relative at omega = 1).
  dcData            log-likelihood within 5e-6 relative of the reference float
                    engine (which is itself ~3e-4 from double there) and P_i
                    within 2e-3 of the float engine's.
"""
import numpy as np
import pytest

import hawkes_b200 as hb

pytestmark = pytest.mark.gpu

FLOAT = hb.CUDA | hb.FLOAT


def run(c):
    loc = np.asarray(c["loc"], dtype=np.float64)
    with hb.CudaHawkes(loc.shape[1], loc.shape[0], FLOAT, 0) as e:
        assert e.precision == hb.PRECISION_FP32
        e.setTimesData(c["t"])
        e.updateLocations(-1, loc.reshape(-1))
        e.setParameters(c["params"])
        ll, g = e.getLogLikelihoodAndGradient()
        probs = e.getProbsSelfExcite()
    return ll, np.asarray(g), probs


def report(name, c, ll, probs):
    ref32, ref64 = float(c["ref_float_loglik"]), float(c["ref_loglik"])
    r32 = abs(ll - ref32) / abs(ref32)
    r64 = abs(ll - ref64) / abs(ref64)
    p32 = float(np.max(np.abs(probs - c["ref_float_probs"]))) if probs.size else 0.0
    print(f"{name:18s} vs float {r32:.2e}  vs double {r64:.2e}  (reference float vs double "
          f"{abs(ref32 - ref64) / abs(ref64):.2e})  probs vs float {p32:.2e}")
    return r32, r64, p32


def test_float_mode_synthetic(golden_synthetic):
    print()
    for name, c in sorted(golden_synthetic.items()):
        ll, g, probs = run(c)
        r32, r64, p32 = report(name, c, ll, probs)
        assert r32 <= 5e-6 and r64 <= 5e-6, name
        assert p32 <= 2e-3, name
        o_scale = c["grad_term_scale"]
        assert np.all(np.abs(g - c["oracle_grad"]) <= 1e-3 * o_scale + 1e-12), name


def test_float_mode_dcdata(golden_dcdata):
    print()
    for name, c in sorted(golden_dcdata.items()):
        ll, g, probs = run(c)
        r32, r64, p32 = report(name, c, ll, probs)
        assert r32 <= 5e-6, name
        assert p32 <= 2e-3, name


def test_float_flag_is_not_compensated():
    # FLOAT alone: plain FP32; FLOAT | COMPENSATED: the compensated mode.
    with hb.CudaHawkes(2, 10, hb.CUDA | hb.FLOAT | hb.COMPENSATED, 0) as e:
        assert e.precision == hb.PRECISION_FP32_COMP
    with hb.CudaHawkes(2, 10, hb.CUDA | hb.COMPENSATED, 0) as e:
        assert e.precision == hb.PRECISION_FP32_COMP
    with hb.CudaHawkes(2, 10, hb.CUDA | hb.FLOAT, 0) as e:
        assert e.precision == hb.PRECISION_FP32
