"""CPU tests of the oracle (oracle/hawkes_oracle.c) against the golden fixtures
generated from the reference engine, against the reference engine compiled
here (when oracle/_ref is built), and against finite differences."""
import numpy as np
import pytest

import oracle
from hawkes_b200 import workloads


def _cases(golden):
    return sorted(golden.items())


def test_oracle_matches_reference_fixtures(golden_synthetic, golden_dcdata):
    for fixtures in (golden_synthetic, golden_dcdata):
        for name, c in _cases(fixtures):
            o = oracle.oracle_eval(c["loc"], c["t"], c["params"], threads=4)
            ref = float(c["ref_loglik"])
            assert abs(o["loglik"] - ref) <= 1e-13 * abs(ref), name
            np.testing.assert_allclose(o["probs"], c["ref_probs"], rtol=1e-12, atol=1e-15,
                                       err_msg=name)
            np.testing.assert_allclose(o["grad"], c["oracle_grad"], rtol=0,
                                       atol=1e-13 * max(1.0, float(np.max(c["grad_scale"]))),
                                       err_msg=name)


def test_oracle_gradient_matches_reference_finite_differences(golden_synthetic):
    checked = 0
    for name, c in _cases(golden_synthetic):
        if "fd_grad" not in c:
            continue
        # Central differences of the reference loglik with step h = 1e-6 |p_k|:
        # truncation ~h^2 plus rounding noise ~ few eps |L| / h.
        noise = 1e-9 * abs(float(c["ref_loglik"])) / np.abs(c["params"])
        tol = 1e-7 * c["grad_scale"] + noise
        err = np.abs(c["oracle_grad"] - c["fd_grad"])
        assert np.all(err <= tol), (name, err / tol)
        checked += 1
    assert checked >= 15


def test_oracle_is_thread_count_independent():
    loc, t = workloads.uniform(700, seed=5)
    a = oracle.oracle_eval(loc, t, workloads.BASE_PARAMS, threads=1)
    b = oracle.oracle_eval(loc, t, workloads.BASE_PARAMS, threads=7)
    assert a["loglik"] == b["loglik"]
    assert np.array_equal(a["grad"], b["grad"])
    assert np.array_equal(a["probs"], b["probs"])


def test_oracle_single_event_closed_form():
    # N=1: lambda_0 = mu0 a^D b phi(0)^2 = mu0 a^D b / (2 pi); T = t_0 so the
    # compensator is 0 - mu0 (Phi(0) - Phi(-b t_0)).
    from math import erfc, log, pi, sqrt
    p = np.array([1.3, 0.7, 0.02, 1.1, 0.9, 1.7])
    t0 = 5.0
    o = oracle.oracle_eval(np.array([[1.0, 2.0]]), np.array([t0]), p)
    Phi = lambda v: 0.5 * erfc(-v / sqrt(2.0))
    lam = p[5] * p[1] ** 2 * p[2] / (2 * pi)
    expect = log(lam) - p[5] * (Phi(0.0) - Phi(-p[2] * t0)) + 1 * (2 - 1) * log(1 / sqrt(2 * pi))
    assert abs(o["loglik"] - expect) <= 1e-14 * abs(expect)
    assert o["probs"][0] == 0.0


def test_oracle_tie_has_no_self_excitation():
    # Two events at the same time: the strict dt > 0 mask (src/NewHawkes.hpp:540)
    # leaves no self-excitation term.
    loc = np.array([[0.0, 0.0], [0.1, 0.0]])
    t = np.array([3.0, 3.0])
    o = oracle.oracle_eval(loc, t, workloads.BASE_PARAMS)
    assert np.all(o["probs"] == 0.0)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference engine not built here")
def test_oracle_matches_compiled_reference_engine():
    rng = np.random.default_rng(123)
    for D, N in ((2, 400), (3, 257), (1, 129)):
        loc = rng.uniform(0, 10, size=(N, D))
        t = np.sort(rng.uniform(0, 2000, size=N))
        p = workloads.BASE_PARAMS * np.exp(0.3 * rng.standard_normal(6))
        o = oracle.oracle_eval(loc, t, p, threads=3)
        ref = oracle.ref_loglik(loc, t, p)
        assert abs(o["loglik"] - ref) <= 1e-13 * abs(ref)
        np.testing.assert_allclose(o["probs"], oracle.ref_probs(loc, t, p), rtol=1e-12,
                                   atol=1e-15)
        # the reference's "TBB" path (std::thread stub) agrees with its serial path
        assert abs(oracle.ref_loglik(loc, t, p, threads=4) - ref) <= 1e-13 * abs(ref)
