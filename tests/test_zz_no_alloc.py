"""GPU test of hphc_loglik_grad_fp64_static, the entry point for callers that
cannot allocate GPU memory while they run (a host framework that owns all
device memory through its own pool or cap, a real-time loop that cannot take
an allocation's synchronisation, a process with a fixed GPU memory budget).
It keeps all of its scratch in one static device array inside the library, so
the caller passes only device inputs and an output buffer.

The test calls it through the C ABI on device buffers the test allocates,
twice in a row on different event sets (the shared static scratch must not
carry anything from one call into the next) and once more on the first set,
and compares every result with the engine entry point
(hphc_get_log_likelihood_and_gradient, FP64 mode) within the FP64 tolerance
of the parity tests, and the first one also with the oracle.  A set with
unsorted and tied times checks the same against the engine.  This file is
collected last so that a failing run that stops at the first failure has
already run every other test.
"""
import ctypes
import os

import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import _native, workloads

pytestmark = pytest.mark.gpu

_dp = ctypes.POINTER(ctypes.c_double)


def engine_result(loc, t, p):
    with hb.CudaHawkes(loc.shape[1], loc.shape[0], hb.CUDA, 0) as e:
        e.setTimesData(t)
        e.updateLocations(-1, loc)
        e.setParameters(p)
        return e.getLogLikelihoodAndGradient()


def static_result(torch, loc, t, p):
    dev_loc = torch.tensor(np.ascontiguousarray(loc).reshape(-1), dtype=torch.float64,
                           device="cuda")
    dev_t = torch.tensor(t, dtype=torch.float64, device="cuda")
    out = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")
    params = np.ascontiguousarray(p, dtype=np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    st = _native.lib.hphc_loglik_grad_fp64_static(
        loc.shape[1], loc.shape[0], ctypes.c_void_p(dev_loc.data_ptr()),
        ctypes.c_void_p(dev_t.data_ptr()), params.ctypes.data_as(_dp),
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert st == 0, _native.lib.hphc_status_string(st).decode()
    host = out.cpu().numpy()
    return float(host[0]), host[1:7].copy()


def close(a, b):
    ll_a, g_a = a
    ll_b, g_b = b
    assert abs(ll_a - ll_b) <= 1e-12 * abs(ll_b)
    assert np.all(np.abs(g_a - g_b) <= 1e-10 * (np.abs(g_b) + 1e-6 * np.max(np.abs(g_b))))


def test_static_scratch_entry_point_matches_engine():
    torch = pytest.importorskip("torch")
    loc_a, t_a = workloads.uniform(3000, seed=21)
    p_a = workloads.BASE_PARAMS
    loc_b, t_b = workloads.uniform(1700, seed=22, D=3)
    p_b = workloads.BASE_PARAMS * np.array([1.2, 0.9, 1.1, 0.7, 1.3, 0.8])

    first_a = static_result(torch, loc_a, t_a, p_a)
    close(first_a, engine_result(loc_a, t_a, p_a))
    second_b = static_result(torch, loc_b, t_b, p_b)
    close(second_b, engine_result(loc_b, t_b, p_b))
    again_a = static_result(torch, loc_a, t_a, p_a)
    assert again_a[0] == first_a[0] and np.array_equal(again_a[1], first_a[1])

    o = oracle.oracle_eval(loc_a, t_a, p_a, threads=max(1, os.cpu_count() or 1))
    assert abs(first_a[0] - o["loglik"]) <= 1e-10 * abs(o["loglik"])
    assert np.all(np.abs(first_a[1] - o["grad"]) <= 1e-10 * o["grad_scale"])


def test_static_scratch_unsorted_and_tied_times():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(23)
    loc = rng.uniform(0.0, 20.0, size=(1500, 2))
    t = rng.integers(0, 300, size=1500).astype(np.float64) * 5.0  # many exact ties
    m = int(np.argmax(t))
    t[m], t[-1] = t[-1], t[m]  # unsorted, the latest time last (T = t[N-1])
    p = workloads.BASE_PARAMS * np.array([0.8, 1.1, 1.4, 0.9, 1.2, 1.0])
    close(static_result(torch, loc, t, p), engine_result(loc, t, p))


def test_static_scratch_rejects_oversized_problems():
    torch = pytest.importorskip("torch")
    small = torch.zeros(8, dtype=torch.float64, device="cuda")
    params = np.ascontiguousarray(workloads.BASE_PARAMS)
    st = _native.lib.hphc_loglik_grad_fp64_static(
        2, 10_000_000, ctypes.c_void_p(small.data_ptr()), ctypes.c_void_p(small.data_ptr()),
        params.ctypes.data_as(_dp), ctypes.c_void_p(small.data_ptr()), None)
    assert st == 11  # HPHC_ERR_SCRATCH_TOO_SMALL, decided before any device work
