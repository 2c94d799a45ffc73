"""Accuracy at the headline size: N = 100,000 events (20 x 20 km box, times
U[0, 8760) h sorted, seed 5, base parameters) against the committed oracle
fixture tests/golden/headline_n100k.npz (made by make_headline.py; the
oracle's log-likelihood there agrees with the reference CPU engine's,
src/NewHawkes.hpp:636-660, to 6e-15, and its P_i subset with the reference's
src/NewHawkes.hpp:662-719 to 2e-14).

Bars
  FP64 plain        log-likelihood relative 1e-10; gradient 1e-10 of |g_k|
                    for every component; P_i 1e-10 absolute.
  FP32-compensated  log-likelihood relative 1e-8; gradient 1e-8 of |g_k| for
                    every component (componentwise) and 1e-8 of its
                    per-event scale sum_i |per-event contribution|; P_i 1e-5
                    absolute.
"""
import os

import numpy as np
import pytest

import hawkes_b200 as hb
from hawkes_b200 import workloads

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                       "headline_n100k.npz")


@pytest.fixture(scope="module")
def headline():
    z = np.load(FIXTURE)
    N, seed = int(z["N"]), int(z["seed"])
    loc, t = workloads.uniform(N, seed=seed)
    ck = np.array([t.sum(), t[0], t[-1], loc[:, 0].sum(), loc[:, 1].sum()])
    assert np.allclose(ck, z["input_checksums"], rtol=1e-14, atol=0), \
        "the generator no longer reproduces the fixture's events"
    return loc, t, z


def evaluate(loc, t, p, flags):
    with hb.CudaHawkes(2, len(t), flags, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(p)
        ll, g = e.getLogLikelihoodAndGradient()
        probs = e.getProbsSelfExcite()
    return ll, np.asarray(g), probs


def errors(tag, ll, g, probs, z):
    llo, go = float(z["oracle_loglik"]), z["oracle_grad"]
    rel = abs(ll - llo) / abs(llo)
    comp = np.abs(g - go) / np.abs(go)
    scale = np.abs(g - go) / z["grad_scale"]
    pe = np.max(np.abs(probs[z["probs_index"]] - z["oracle_probs"]))
    print(f"\n{tag}: loglik rel {rel:.3e}\n  grad err/|g_k|       "
          f"{np.array2string(comp, precision=2)}\n  grad err/event-scale "
          f"{np.array2string(scale, precision=2)}\n  probs max abs {pe:.3e}")
    return rel, comp, scale, pe


def test_fixture_is_pinned_to_the_reference(headline):
    _, _, z = headline
    assert abs(float(z["ref_loglik"]) - float(z["oracle_loglik"])) <= 1e-13 * abs(
        float(z["ref_loglik"]))
    assert np.max(np.abs(z["ref_probs"] - z["oracle_probs"])) <= 1e-12


def test_fp64_plain_at_headline_size(headline):
    loc, t, z = headline
    rel, comp, _, pe = errors("fp64", *evaluate(loc, t, z["params"], hb.CUDA), z)
    assert rel <= 1e-10
    assert np.all(comp <= 1e-10)
    assert pe <= 1e-10


def test_fp32_compensated_at_headline_size(headline):
    loc, t, z = headline
    rel, comp, scale, pe = errors("fp32c", *evaluate(loc, t, z["params"],
                                                     hb.CUDA | hb.COMPENSATED), z)
    assert rel <= 1e-8
    assert np.all(comp <= 1e-8), "componentwise gradient error above 1e-8"
    assert np.all(scale <= 1e-8)
    assert pe <= 1e-5
