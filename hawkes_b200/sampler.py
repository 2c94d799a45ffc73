"""Multi-chain Metropolis-Hastings sampler over the Hawkes parameters.

:class:`Sampler` wraps the C ABI's ``hphc_sampler_*`` (include/hphc.h), the
restatement of the reference's R ``sampler()`` (R/Untitled.R:254-422) for K
independent chains whose proposals are evaluated together in one batched
likelihood run per iteration.  :func:`sampler` mirrors the R function's
signature and return value; :func:`Potential` mirrors ``Potential()``
(R/Untitled.R:225-231).
"""
from __future__ import annotations

import ctypes
import math
import time
from typing import Callable, Optional

import numpy as np

from . import _native
from .engine import CudaHawkes, Engine, HawkesError, engineInitial, getLogLikelihood

_lib = _native.lib
_dp = ctypes.POINTER(ctypes.c_double)

# Parameters the reference proposes: sample(c(1,4:6)) (R/Untitled.R:328),
# i.e. sigmaXprec, omega, theta, mu0 (0-based 0, 3, 4, 5).
REFERENCE_SAMPLED = (0, 3, 4, 5)
BASE_PARAMS = (1.0, 1.0 / 1.6, 1.0 / (14 * 24), 1.0, 1.0, 1.0)


def _log_truncnorm(x: float, mean: float, sd: float) -> float:
    if not x >= 0.0:
        return -math.inf
    z = (x - mean) / sd
    tail = 0.5 * math.erfc((-mean / sd) / math.sqrt(2.0))
    return -0.5 * z * z - math.log(sd) - 0.5 * math.log(2.0 * math.pi) - math.log(tail)


def log_prior(params) -> float:
    """Log prior of the reference's Potential (R/Untitled.R:226-227):
    independent normals truncated to (0, inf), sd 10 for the first five
    parameters and sd 1 for mu0."""
    p = np.asarray(params, dtype=np.float64).reshape(-1)
    return sum(_log_truncnorm(float(p[k]), 0.0, 10.0) for k in range(5)) + \
        _log_truncnorm(float(p[5]), 0.0, 1.0)


def Potential(engine: Engine, parameters) -> float:
    """-logL - log prior at the engine's current parameters (R/Untitled.R:225-231)."""
    return -getLogLikelihood(engine) - log_prior(parameters)


class Sampler:
    """K chains of the reference's random-scan Metropolis-Hastings sampler.

    initialParams: 6 values (one chain) or K x 6.  radius: initial proposal sd
    of every parameter.  sampled: parameter indices proposed from (default the
    reference's sigma, omega, theta, mu0).  seed: seeds one splitmix64 stream
    per chain.  State is kept between :meth:`run` calls.
    """

    def __init__(self, initialParams, radius: float = 2.0, sampled=REFERENCE_SAMPLED,
                 seed: int = 0):
        p = np.ascontiguousarray(np.asarray(initialParams, dtype=np.float64).reshape(-1, 6))
        mask = 0
        for q in sampled:
            mask |= 1 << int(q)
        h = ctypes.c_void_p()
        st = _lib.hphc_sampler_create(p.shape[0], p.ctypes.data_as(_dp), float(radius), mask,
                                      ctypes.c_ulonglong(int(seed) & (2 ** 64 - 1)),
                                      ctypes.byref(h))
        if st != 0:
            raise HawkesError(st, "hphc_sampler_create: " + _lib.hphc_status_string(st).decode())
        self._h = h
        self.numChains = p.shape[0]

    def _check(self, st: int, what: str) -> None:
        if st != 0:
            msg = (_lib.hphc_sampler_last_error(self._h).decode() or
                   _lib.hphc_status_string(st).decode())
            raise HawkesError(st, f"{what}: {msg}")

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.hphc_sampler_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, evaluator, iterations: int, burnIn: int = 0, device: bool = False):
        """Run every chain; returns (samples [K, iterations - burnIn, 6],
        targets [K, iterations - burnIn]).

        evaluator: a :class:`CudaHawkes` engine (its batched entry point
        evaluates the K proposals in one run) or a callable mapping a K x 6
        array of parameter vectors to K log-likelihoods.  device=True (engine
        only) runs every iteration on the GPU from one captured CUDA graph."""
        M = int(iterations) - int(burnIn)
        samples = np.zeros((self.numChains, max(M, 0), 6))
        targets = np.zeros((self.numChains, max(M, 0)))
        if isinstance(evaluator, CudaHawkes):
            fn = _lib.hphc_sampler_run_device if device else _lib.hphc_sampler_run
            st = fn(self._h, evaluator._h, int(iterations), int(burnIn),
                    samples.ctypes.data_as(_dp), targets.ctypes.data_as(_dp))
        elif device:
            raise HawkesError(3, "run: device=True needs a CudaHawkes engine")
        else:
            st = self._run_callable(evaluator, iterations, burnIn, samples, targets)
        self._check(st, "run")
        return samples, targets

    def _run_callable(self, fn: Callable, iterations, burnIn, samples, targets) -> int:
        failure = []

        def cb(_user, params, K, out):
            try:
                p = np.ctypeslib.as_array(params, shape=(K, 6)).copy()
                ll = np.asarray(fn(p), dtype=np.float64).reshape(K)
                ctypes.memmove(out, ll.ctypes.data, K * 8)
                return 0
            except Exception as exc:  # reported after the run returns
                failure.append(exc)
                return 3

        cfn = _native.BATCH_LOGLIK_FN(cb)
        st = _lib.hphc_sampler_run_with(self._h, ctypes.cast(cfn, ctypes.c_void_p), None,
                                        int(iterations), int(burnIn),
                                        samples.ctypes.data_as(_dp), targets.ctypes.data_as(_dp))
        if failure:
            raise failure[0]
        return st

    def state(self) -> dict:
        K = self.numChains
        params = np.zeros((K, 6))
        pot = np.zeros(K)
        radii = np.zeros((K, 6))
        acc = (ctypes.c_longlong * K)()
        prop = (ctypes.c_longlong * K)()
        self._check(_lib.hphc_sampler_get_state(self._h, params.ctypes.data_as(_dp),
                                                pot.ctypes.data_as(_dp),
                                                radii.ctypes.data_as(_dp), acc, prop), "state")
        return {"params": params, "potential": pot, "radii": radii,
                "accepted": np.array(acc[:], dtype=np.int64),
                "proposed": np.array(prop[:], dtype=np.int64)}


def sampler(n_iter: int, burnIn: int = 0, locations=None, times=None, radius: float = 2.0,
            params=BASE_PARAMS, latentDimension: int = 2, threads: int = 1, simd: int = 0,
            gpu: int = 1, single: int = 0, chains: int = 1, seed: int = 0,
            on_device: bool = False) -> dict:
    """The reference's ``sampler()`` (R/Untitled.R:254-422) on the CUDA engine.

    Returns {"samples": 6 x (n_iter - burnIn) (chains x 6 x ... for
    chains > 1), "target": the potentials (same leading shape), "Time":
    seconds of the sampling loop}.  ``threads`` and ``simd`` are accepted for
    signature compatibility and ignored; ``gpu`` is the device number as in
    ``createEngine``; ``single`` selects the FP32-compensated mode; ``chains``
    runs that many independent chains from ``params`` (each with its own
    random stream), their proposals evaluated together; ``on_device`` runs the
    iterations as one replayed CUDA graph (tauX and tauT stay fixed, as in the
    reference's sampler)."""
    if locations is None:
        raise HawkesError(3, "No locations found.")
    if times is None:
        raise HawkesError(3, "No times found.")
    loc = np.asarray(locations, dtype=np.float64)
    N = loc.shape[0]
    eng = engineInitial(loc, N, latentDimension, times, params, threads, simd, gpu, single)
    init = np.tile(np.asarray(params, dtype=np.float64).reshape(1, 6), (int(chains), 1))
    with Sampler(init, radius=radius, seed=seed) as s:
        t0 = time.perf_counter()
        samples, targets = s.run(eng["engine"], n_iter, burnIn, device=on_device)
        elapsed = time.perf_counter() - t0
    eng["engine"].close()
    samples = np.transpose(samples, (0, 2, 1))  # chains x 6 x M, as ParametersSaved
    if chains == 1:
        return {"samples": samples[0], "target": targets[0], "Time": elapsed}
    return {"samples": samples, "target": targets, "Time": elapsed}
