"""The multi-chain Metropolis-Hastings driver (hphc_sampler_*, the restatement
of the reference's R sampler(), R/Untitled.R:254-422) against an independent
Python restatement of the same loop, both fed by the same per-chain
splitmix64 streams and both evaluating the likelihood with the CPU oracle.

These tests call the driver through the C ABI with a caller-supplied batched
evaluator, so they need no GPU; tests/test_sampler_gpu.py runs the driver on
the CUDA engine.
"""
import math

import numpy as np
import pytest

import oracle
from hawkes_b200 import HawkesError, Sampler, log_prior, workloads

MASK64 = (1 << 64) - 1


class SplitMix64:
    """Steele, Lea and Flood (2014)."""

    def __init__(self, state):
        self.state = state & MASK64

    def next(self):
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self):
        return ((self.next() >> 11) + 0.5) * 2.0 ** -53

    def normal(self):
        u1 = self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def rtruncnorm(g, mean, sd):
    """N(mean, sd^2) truncated to [0, inf): Robert (1995)."""
    alpha = -mean / sd
    if alpha <= 0.0:
        while True:
            z = g.normal()
            if z >= alpha:
                return mean + sd * z
    lam = 0.5 * (alpha + math.sqrt(alpha * alpha + 4.0))
    while True:
        z = alpha - math.log(g.uniform()) / lam
        if g.uniform() <= math.exp(-0.5 * (z - lam) ** 2):
            return mean + sd * z


def log_dtruncnorm(x, mean, sd):
    if not x >= 0.0:
        return -math.inf
    z = (x - mean) / sd
    tail = 0.5 * math.erfc((-mean / sd) / math.sqrt(2.0))
    return -0.5 * z * z - math.log(sd) - 0.5 * math.log(2 * math.pi) - math.log(tail)


def reference_loop(init, radius, sampled, seed, loglik, iterations, burn_in):
    """R/Untitled.R:300-414 for each chain, proposals of all chains batched."""
    K = init.shape[0]
    cur = init.copy()
    gens = [SplitMix64(seed ^ ((0x632BE59BD9B4E019 * (k + 1)) & MASK64)) for k in range(K)]
    radii = np.full((K, 6), float(radius))
    acc = np.zeros((K, 6), dtype=int)
    bound = np.full((K, 6), 5, dtype=int)
    count = np.zeros((K, 6), dtype=int)
    U = -loglik(cur) - np.array([log_prior(p) for p in cur])
    samples = np.zeros((K, iterations - burn_in, 6))
    targets = np.zeros((K, iterations - burn_in))
    for it in range(1, iterations + 1):
        prop = cur.copy()
        idx = np.zeros(K, dtype=int)
        former = np.zeros(K)
        for k in range(K):
            n = len(sampled)
            pick = min(int(gens[k].uniform() * n), n - 1)
            idx[k] = sampled[pick]
            former[k] = prop[k, idx[k]]
            prop[k, idx[k]] = rtruncnorm(gens[k], former[k], radii[k, idx[k]])
        ll = loglik(prop)
        for k in range(K):
            i = idx[k]
            r = radii[k, i]
            propU = -ll[k] - log_prior(prop[k])
            curH = U[k] - log_dtruncnorm(prop[k, i], former[k], r)
            propH = propU - log_dtruncnorm(former[k], prop[k, i], r)
            if -propH + curH > math.log(gens[k].uniform()):
                cur[k] = prop[k]
                U[k] = propU
                acc[k, i] += 1
            count[k, i] += 1
            if count[k, i] == bound[k, i]:
                ratio = min(2.0, max(0.5, acc[k, i] / bound[k, i] / 0.44))
                radii[k, i] *= ratio
                count[k, i] = 0
                bound[k, i] = math.ceil(bound[k, i] ** 1.1)
                acc[k, i] = 0
            if it > burn_in:
                samples[k, it - burn_in - 1] = cur[k]
                targets[k, it - burn_in - 1] = U[k]
    return samples, targets, radii


@pytest.fixture(scope="module")
def small_set():
    loc, t = workloads.uniform(150, seed=31)
    return loc, t


def oracle_batch(loc, t):
    def f(P):
        return np.array([oracle.oracle_eval(loc, t, p, threads=1)["loglik"] for p in P])
    return f


def test_driver_matches_restated_reference_loop(small_set):
    loc, t = small_set
    base = np.asarray(workloads.BASE_PARAMS)
    init = np.stack([base, base * np.array([1.3, 1, 1, 0.8, 0.9, 1.2]), base * 0.7])
    f = oracle_batch(loc, t)
    with Sampler(init, radius=0.5, seed=12345) as s:
        samples, targets = s.run(f, 120, burnIn=20)
        st = s.state()
    ref_s, ref_t, ref_r = reference_loop(init, 0.5, (0, 3, 4, 5), 12345, f, 120, 20)
    np.testing.assert_allclose(samples, ref_s, rtol=1e-13, atol=0)
    np.testing.assert_allclose(targets, ref_t, rtol=1e-12, atol=0)
    np.testing.assert_allclose(st["radii"], ref_r, rtol=1e-13)
    # tauX and tauT are never proposed (sample(c(1,4:6)), R/Untitled.R:328)
    assert np.all(samples[:, :, 1:3] == init[:, None, 1:3])
    assert np.all(st["proposed"] == 120)
    assert np.all((st["accepted"] > 0) & (st["accepted"] < 120))


def test_runs_continue_the_same_chains(small_set):
    loc, t = small_set
    f = oracle_batch(loc, t)
    init = np.asarray(workloads.BASE_PARAMS)
    with Sampler(init, radius=1.0, seed=7) as a:
        whole, _ = a.run(f, 60)
    with Sampler(init, radius=1.0, seed=7) as b:
        first, _ = b.run(f, 25)
        second, _ = b.run(f, 35)
    np.testing.assert_array_equal(np.concatenate([first, second], axis=1), whole)


def test_sampled_set_and_seed(small_set):
    loc, t = small_set
    f = oracle_batch(loc, t)
    init = np.asarray(workloads.BASE_PARAMS)
    with Sampler(init, radius=0.3, sampled=(1, 2), seed=3) as s:
        x, _ = s.run(f, 30)
    assert np.all(x[0, :, [0, 3, 4, 5]] == init[[0, 3, 4, 5], None])
    with Sampler(init, radius=0.3, seed=3) as a, Sampler(init, radius=0.3, seed=4) as b:
        xa, _ = a.run(f, 30)
        xb, _ = b.run(f, 30)
    assert not np.array_equal(xa, xb)


def test_invalid_arguments_and_evaluator_errors(small_set):
    with pytest.raises(HawkesError):
        Sampler(np.asarray(workloads.BASE_PARAMS), radius=0.0)
    with pytest.raises(HawkesError):
        Sampler(-np.asarray(workloads.BASE_PARAMS))
    with Sampler(np.asarray(workloads.BASE_PARAMS)) as s:
        with pytest.raises(HawkesError):
            s.run(lambda P: np.zeros(len(P)), 5, burnIn=6)

        def broken(P):
            raise ValueError("evaluator failed")
        with pytest.raises(ValueError):
            s.run(broken, 3)
