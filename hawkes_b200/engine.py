"""Python host interface of the B200 Hawkes likelihood engine.

Two layers, both thin wrappers over the C ABI in include/hphc.h:

* :class:`CudaHawkes` mirrors the reference engine interface
  ``hph::AbstractHawkes`` (src/AbstractHawkes.hpp:32-60) method for method:
  ``setTimesData``, ``updateLocations``, ``setParameters``,
  ``getSumOfLikContribs``, ``getLogLikelihoodGradient`` (commented out in the
  reference at src/AbstractHawkes.hpp:44), ``getProbsSelfExcite``,
  ``storeState``/``restoreState``/``acceptState`` and
  ``getInternalDimension``.  Construction mirrors ``hph::factory``
  (src/factory.cpp:32) with the GPU slot selected.

* Module functions mirror the reference's R API (R/hph.R:10-110,
  src/hpHawkes.cpp:59-151): ``createEngine``, ``setTimesData``,
  ``updateLocations`` (an N x D matrix, row-major as R/hph.R:103 arranges it),
  ``setParameters``, ``getLogLikelihood``, ``getProbsSelfExcite`` and the
  gradient the reference does not expose.  They raise the same messages as the
  R functions ("locations not set", "times not set", "parameters not set",
  "Invalid data size").

Every call goes to the CUDA library; errors raise :class:`HawkesError` with the
engine's message.
"""
from __future__ import annotations

import ctypes
import time
from typing import Optional

import numpy as np

from . import _native

_lib = _native.lib
_dp = ctypes.POINTER(ctypes.c_double)

# hph::Flags (src/flags.h:6-13) and the two bits added for the CUDA engine.
FLOAT = 1 << 2
TBB = 1 << 3
OPENCL = 1 << 4
SSE = 1 << 5
AVX = 1 << 6
AVX512 = 1 << 7
CUDA = 1 << 8
COMPENSATED = 1 << 9
NO_UNDERFLOW_SKIP = 1 << 10
FP32_FAST_EXP = 1 << 11
FP32_SPACE_HILO = 1 << 12
ORDERED = 1 << 13       # both orders of every background pair, either precision
FP32_ORDERED = ORDERED  # earlier name of the same bit
NO_INCREMENTAL = 1 << 14
NO_FAST_TAIL = 1 << 15  # one exponential for every term, the far tail included
NO_TAIL_TRUNCATION = 1 << 16  # skip background tile pairs only where every term underflows

# Fault-injection stages (CudaHawkes.injectFault).
FAULT_UPLOAD = 1
FAULT_LAUNCH = 2
FAULT_WAIT = 3

# How an evaluation was computed (CudaHawkes.lastEvaluationPath).
PATH_SWEEP = 0
PATH_INCREMENTAL = 1
PATH_KEPT_SUMS = 2
PATH_SELF_EXCITATION = 3

PRECISION_FP64 = 0
PRECISION_FP32_COMP = 1
PRECISION_FP32 = 2  # FP32 throughout: the reference's single precision (FLOAT alone)

# Parameter order of NewHawkes::setParameters (src/NewHawkes.hpp:331-339).
PARAMETER_NAMES = ("sigmaXprec", "tauXprec", "tauTprec", "omega", "theta", "mu0")


class HawkesError(RuntimeError):
    """A non-zero status from the CUDA engine."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def _as_f64(a, name: str) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    return arr


class CudaHawkes:
    """The CUDA engine behind the reference's ``hph::AbstractHawkes`` interface."""

    def __init__(self, embeddingDimension: int, locationCount: int, flags: int = CUDA,
                 device: int = 0):
        h = ctypes.c_void_p()
        st = _lib.hphc_create(int(embeddingDimension), int(locationCount), int(flags),
                              int(device), ctypes.byref(h))
        if st != 0:
            raise HawkesError(st, "hphc_create: " + _lib.hphc_status_string(st).decode())
        self._h = h
        self.embeddingDimension = int(embeddingDimension)
        self.locationCount = int(locationCount)
        self.flags = int(flags)
        self.device = int(device)

    # -- plumbing -------------------------------------------------------------
    def _check(self, st: int, what: str) -> None:
        if st != 0:
            msg = _lib.hphc_last_error(self._h).decode() or _lib.hphc_status_string(st).decode()
            raise HawkesError(st, f"{what}: {msg}")

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.hphc_destroy(self._h)
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

    # -- hph::AbstractHawkes ----------------------------------------------------
    def setTimesData(self, data) -> None:
        arr = _as_f64(data, "times")
        self._check(_lib.hphc_set_times_data(self._h, arr.ctypes.data_as(_dp), arr.size),
                    "setTimesData")

    def updateLocations(self, locationIndex: int, location) -> None:
        arr = _as_f64(location, "locations")
        self._check(_lib.hphc_update_locations(self._h, int(locationIndex),
                                               arr.ctypes.data_as(_dp), arr.size),
                    "updateLocations")

    def setParameters(self, data) -> None:
        arr = _as_f64(data, "parameters")
        self._check(_lib.hphc_set_parameters(self._h, arr.ctypes.data_as(_dp), arr.size),
                    "setParameters")

    def getSumOfLikContribs(self) -> float:
        out = ctypes.c_double()
        self._check(_lib.hphc_get_sum_of_lik_contribs(self._h, ctypes.byref(out)),
                    "getSumOfLikContribs")
        return out.value

    def getLogLikelihoodGradient(self) -> np.ndarray:
        out = np.zeros(6)
        self._check(_lib.hphc_get_log_likelihood_gradient(self._h, out.ctypes.data_as(_dp), 6),
                    "getLogLikelihoodGradient")
        return out

    def getLogLikelihoodAndGradient(self):
        ll = ctypes.c_double()
        g = np.zeros(6)
        self._check(_lib.hphc_get_log_likelihood_and_gradient(self._h, ctypes.byref(ll),
                                                              g.ctypes.data_as(_dp), 6),
                    "getLogLikelihoodAndGradient")
        return ll.value, g

    def getProbsSelfExcite(self) -> np.ndarray:
        out = np.zeros(self.locationCount)
        self._check(_lib.hphc_get_probs_self_excite(self._h, out.ctypes.data_as(_dp), out.size),
                    "getProbsSelfExcite")
        return out

    def storeState(self) -> None:
        self._check(_lib.hphc_store_state(self._h), "storeState")

    def restoreState(self) -> None:
        self._check(_lib.hphc_restore_state(self._h), "restoreState")

    def acceptState(self) -> None:
        self._check(_lib.hphc_accept_state(self._h), "acceptState")

    def getInternalDimension(self) -> int:
        out = ctypes.c_int()
        self._check(_lib.hphc_get_internal_dimension(self._h, ctypes.byref(out)),
                    "getInternalDimension")
        return out.value

    # -- additions ------------------------------------------------------------
    def batchLogLikelihoodAndGradient(self, params):
        """Log-likelihood and gradient for K parameter vectors (K x 6)."""
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1, 6))
        K = p.shape[0]
        ll = np.zeros(K)
        g = np.zeros((K, 6))
        self._check(_lib.hphc_batch_log_likelihood_and_gradient(
            self._h, p.ctypes.data_as(_dp), K, ll.ctypes.data_as(_dp), g.ctypes.data_as(_dp)),
            "batchLogLikelihoodAndGradient")
        return ll, g

    @property
    def precision(self) -> int:
        out = ctypes.c_int()
        self._check(_lib.hphc_get_precision(self._h, ctypes.byref(out)), "getPrecision")
        return out.value

    @property
    def stream(self) -> int:
        """The engine's cudaStream_t as an integer handle."""
        out = ctypes.c_void_p()
        self._check(_lib.hphc_get_stream(self._h, ctypes.byref(out)), "getStream")
        return int(out.value or 0)

    def enqueueLogLikelihoodAndGradient(self) -> None:
        self._check(_lib.hphc_enqueue_log_likelihood_and_gradient(self._h),
                    "enqueueLogLikelihoodAndGradient")

    def readResults(self):
        ll = ctypes.c_double()
        g = np.zeros(6)
        self._check(_lib.hphc_read_results(self._h, ctypes.byref(ll), g.ctypes.data_as(_dp), 6),
                    "readResults")
        return ll.value, g

    def setSweepShape(self, eventsPerThread: int = 0, itemsPerSM: int = 0) -> None:
        """Fix the sweep shape (0 = autotune that dimension)."""
        self._check(_lib.hphc_set_sweep_shape(self._h, int(eventsPerThread), int(itemsPerSM)),
                    "setSweepShape")

    def sweepShape(self):
        r = ctypes.c_int()
        i = ctypes.c_int()
        self._check(_lib.hphc_get_sweep_shape(self._h, ctypes.byref(r), ctypes.byref(i)),
                    "sweepShape")
        return r.value, i.value

    def setKernelTiming(self, enable: bool = True) -> None:
        self._check(_lib.hphc_set_kernel_timing(self._h, int(bool(enable))), "setKernelTiming")

    def kernelTimes(self):
        """(sweep ms, finish ms, step ms) of the last evaluation made with kernel
        timing on; the step spans table upload, record build, sweep, finish and
        result copy on the device."""
        a = ctypes.c_float()
        b = ctypes.c_float()
        c = ctypes.c_float()
        self._check(_lib.hphc_get_kernel_times(self._h, ctypes.byref(a), ctypes.byref(b),
                                               ctypes.byref(c)), "kernelTimes")
        return a.value, b.value, c.value

    def lastLaunchStats(self):
        """(kernel launches, background terms evaluated, self-excitation terms
        evaluated) of the last evaluation."""
        n = ctypes.c_int()
        nb = ctypes.c_double()
        ns = ctypes.c_double()
        self._check(_lib.hphc_get_last_launch_stats(self._h, ctypes.byref(n), ctypes.byref(nb),
                                                    ctypes.byref(ns)), "lastLaunchStats")
        return n.value, nb.value, ns.value

    def lastLaunchEvals(self):
        """Background exponentials the last evaluation computed (a pair
        evaluated once for both of its events counts once)."""
        v = ctypes.c_double()
        self._check(_lib.hphc_get_last_launch_evals(self._h, ctypes.byref(v)), "lastLaunchEvals")
        return v.value

    def injectFault(self, stage: int, count: int = 1) -> None:
        """Make the next `count` calls that reach `stage` (FAULT_UPLOAD,
        FAULT_LAUNCH, FAULT_WAIT) fail there with a stand-in CUDA error; the
        engine stays usable.  count 0 clears."""
        self._check(_lib.hphc_inject_fault(self._h, int(stage), int(count)), "injectFault")

    # -- sharded evaluation (hawkes_b200.shard) --------------------------------
    def sweepShard(self, rank: int, world: int, devicePart: int) -> None:
        """Rank `rank` of `world`: write this rank's share of every event's six
        unit pair sums at the current parameters to the device buffer at
        address devicePart (6 N doubles on the engine's device)."""
        self._check(_lib.hphc_sweep_shard(self._h, int(rank), int(world),
                                          ctypes.c_void_p(int(devicePart)),
                                          6 * self.locationCount), "sweepShard")

    def setUnitSums(self, deviceParts: int, numParts: int) -> None:
        """Add numParts shares (back to back at device address deviceParts,
        share r from rank r) in rank order and keep them as the sums at the
        current parameters; the next evaluation runs only the O(N) finish."""
        self._check(_lib.hphc_set_unit_sums(self._h, ctypes.c_void_p(int(deviceParts)),
                                            int(numParts),
                                            int(numParts) * 6 * self.locationCount),
                    "setUnitSums")

    @property
    def lastEvaluationPath(self) -> int:
        """PATH_SWEEP, PATH_INCREMENTAL or PATH_KEPT_SUMS for the last evaluation."""
        v = ctypes.c_int()
        self._check(_lib.hphc_get_last_evaluation_path(self._h, ctypes.byref(v)),
                    "lastEvaluationPath")
        return v.value


class Multiset:
    """Many independent event sets of uneven size, each evaluated at its own
    parameter vector in one run (hphc_multiset_* in include/hphc.h)."""

    def __init__(self, embeddingDimension: int, setSizes, flags: int = CUDA, device: int = 0):
        sizes = (ctypes.c_int * len(setSizes))(*[int(n) for n in setSizes])
        h = ctypes.c_void_p()
        st = _lib.hphc_multiset_create(int(embeddingDimension), len(setSizes), sizes, int(flags),
                                       int(device), ctypes.byref(h))
        if st != 0:
            raise HawkesError(st, "hphc_multiset_create: " +
                              _lib.hphc_status_string(st).decode())
        self._h = h
        self.embeddingDimension = int(embeddingDimension)
        self.setSizes = [int(n) for n in setSizes]

    def _check(self, st: int, what: str) -> None:
        if st != 0:
            msg = (_lib.hphc_multiset_last_error(self._h).decode() or
                   _lib.hphc_status_string(st).decode())
            raise HawkesError(st, f"{what}: {msg}")

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.hphc_multiset_destroy(self._h)
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

    def setData(self, set_index: int, locations, times) -> None:
        loc = _as_f64(locations, "locations")
        t = _as_f64(times, "times")
        self._check(_lib.hphc_multiset_set_data(self._h, int(set_index), loc.ctypes.data_as(_dp),
                                                loc.size, t.ctypes.data_as(_dp), t.size),
                    "setData")

    def logLikelihoodAndGradient(self, params):
        """params: numSets x 6 -> (loglik[numSets], gradient[numSets, 6])."""
        S = len(self.setSizes)
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(S, 6))
        ll = np.zeros(S)
        g = np.zeros((S, 6))
        self._check(_lib.hphc_multiset_log_likelihood_and_gradient(
            self._h, p.ctypes.data_as(_dp), ll.ctypes.data_as(_dp), g.ctypes.data_as(_dp)),
            "logLikelihoodAndGradient")
        return ll, g

    def setKernelTiming(self, enable: bool = True) -> None:
        self._check(_lib.hphc_multiset_set_kernel_timing(self._h, int(bool(enable))),
                    "setKernelTiming")

    def kernelTimes(self):
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        self._check(_lib.hphc_multiset_get_kernel_times(self._h, ctypes.byref(a),
                                                        ctypes.byref(b), ctypes.byref(c)),
                    "kernelTimes")
        return a.value, b.value, c.value

    def lastLaunchStats(self):
        n, nb, ns = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        self._check(_lib.hphc_multiset_get_last_launch_stats(self._h, ctypes.byref(n),
                                                             ctypes.byref(nb), ctypes.byref(ns)),
                    "lastLaunchStats")
        return n.value, nb.value, ns.value

    def lastLaunchEvals(self):
        v = ctypes.c_double()
        self._check(_lib.hphc_multiset_get_last_launch_evals(self._h, ctypes.byref(v)),
                    "lastLaunchEvals")
        return v.value


def factory(embeddingDimension: int, locationCount: int, flags: int, device: int = 0,
            threads: int = 0) -> CudaHawkes:
    """``hph::factory`` (src/factory.cpp:32) restricted to its GPU slot.

    ``OPENCL`` or ``CUDA`` in flags selects the CUDA engine; ``FLOAT`` (the
    reference's single-precision request) selects FP32 throughout, as the
    reference's float engine; ``COMPENSATED`` selects the FP32-compensated mode
    (FP32 pair terms, compensated sums, FP64 reductions).
    ``threads`` is accepted for signature compatibility and ignored.
    """
    if not flags & (OPENCL | CUDA):
        raise HawkesError(5, "factory: this package provides only the GPU engine; "
                             "set the OPENCL or CUDA flag")
    return CudaHawkes(embeddingDimension, locationCount, flags | CUDA, device)


# ---------------------------------------------------------------- R mirror --

class Engine(dict):
    """The list ``createEngine`` returns in R (src/hpHawkes.cpp:97-106)."""


def createEngine(embeddingDimension: int, locationCount: int, tbb: int = 0, simd: int = 0,
                 gpu: int = 1, single: bool = False, compensated: bool = False) -> Engine:
    """``createEngine`` (src/hpHawkes.cpp:59-109) with the GPU path selected.

    ``gpu`` is the device number as in the R glue (``deviceNumber = gpu``,
    src/hpHawkes.cpp:68); out-of-range numbers fall back to device 0 as the
    OpenCL engine falls back to the default device.  ``single`` selects the
    reference's single precision (FP32 throughout); ``compensated`` (not in
    the R glue) the FP32-compensated mode.
    """
    if gpu <= 0:
        raise HawkesError(5, "createEngine: the CUDA engine needs gpu > 0")
    flags = OPENCL | CUDA
    if single:
        flags |= FLOAT
    if compensated:
        flags |= COMPENSATED
    eng = CudaHawkes(embeddingDimension, locationCount, flags, gpu)
    return Engine(engine=eng, embeddingDimension=embeddingDimension,
                  locationCount=locationCount, timesInitialized=False,
                  locationsInitialized=False, threads=0, deviceNumber=gpu, flags=flags,
                  parameters=None)


def updateLocations(engine: Engine, locations) -> Engine:
    """R/hph.R:102-110: an N x D matrix, sent row-major."""
    loc = np.asarray(locations, dtype=np.float64)
    flat = np.ascontiguousarray(loc).reshape(-1)
    if flat.size != engine["locationCount"] * engine["embeddingDimension"]:
        raise HawkesError(2, "Invalid data size")
    engine["engine"].updateLocations(-1, flat)
    engine["locationsInitialized"] = True
    return engine


def setTimesData(engine: Engine, data) -> Engine:
    """R/hph.R:83-91."""
    t = np.asarray(data, dtype=np.float64).reshape(-1)
    if t.size != engine["locationCount"]:
        raise HawkesError(2, "Invalid data size")
    engine["engine"].setTimesData(t)
    engine["timesInitialized"] = True
    return engine


def setParameters(engine: Engine, parameters) -> Engine:
    """R/hph.R:68-72."""
    engine["engine"].setParameters(parameters)
    engine["parameters"] = np.asarray(parameters, dtype=np.float64).copy()
    return engine


def _check_ready(engine: Engine) -> None:
    # R/hph.R:12-22
    if not engine["locationsInitialized"]:
        raise HawkesError(7, "locations not set")
    if not engine["timesInitialized"]:
        raise HawkesError(7, "times not set")
    if engine.get("parameters") is None:
        raise HawkesError(7, "parameters not set")


def getLogLikelihood(engine: Engine) -> float:
    """R/hph.R:10-31."""
    _check_ready(engine)
    return engine["engine"].getSumOfLikContribs()


def getProbsSelfExcite(engine: Engine) -> np.ndarray:
    """R/hph.R:41-57."""
    _check_ready(engine)
    return engine["engine"].getProbsSelfExcite()


def getGradient(engine: Engine) -> np.ndarray:
    """Gradient of the log-likelihood (the reference's commented-out
    ``.getLogLikelihoodGradient``, src/hpHawkes.cpp:124-130)."""
    _check_ready(engine)
    return engine["engine"].getLogLikelihoodGradient()


def engineInitial(locations, N: int, P: int, times, parameters, threads: int = 0, simd: int = 0,
                  gpu: int = 1, single: bool = False) -> Engine:
    """R/Untitled.R:193-212: create, set locations, times and parameters."""
    engine = createEngine(P, N, threads, simd, gpu, single)
    engine = updateLocations(engine, locations)
    engine = setTimesData(engine, times)
    engine = setParameters(engine, parameters)
    return engine


def timeTest(locationCount: int = 5000, maxIts: int = 1, threads: int = 0, simd: int = 0,
             gpu: int = 1, single: int = 0, r: bool = False, seed: int = 666) -> float:
    """``timeTest()`` (R/Untitled.R:132-175): seconds taken by ``maxIts``
    log-likelihood evaluations of a random problem in two dimensions
    (standard normal locations, times 1..N, parameters drawn from Exp(1)),
    with numpy's generator seeded by ``seed`` in place of R's.

    Every evaluation is the full computation, as the reference recomputes
    each time: the engine is made with ``NO_INCREMENTAL`` so that repeated
    calls at unchanged parameters do not reuse kept sums.  ``r=True`` (the
    naive R implementation) is not part of this package; ``threads`` and
    ``simd`` are accepted for signature compatibility.
    """
    if r:
        raise HawkesError(5, "timeTest: the naive R implementation is not part of this package")
    if gpu <= 0:
        raise HawkesError(5, "timeTest: the CUDA engine needs gpu > 0")
    rng = np.random.default_rng(seed)
    n = int(locationCount)
    locations = rng.standard_normal((n, 2))
    times = np.arange(1, n + 1, dtype=np.float64)
    params = rng.exponential(1.0, size=6)
    flags = OPENCL | CUDA | NO_INCREMENTAL | (FLOAT if single else 0)
    with CudaHawkes(2, n, flags, gpu) as eng:
        eng.updateLocations(-1, locations)
        eng.setTimesData(times)
        eng.setParameters(params)
        t0 = time.perf_counter()
        for _ in range(int(maxIts)):
            eng.getSumOfLikContribs()
        elapsed = time.perf_counter() - t0
    print(f"{elapsed:.6f}")
    return elapsed
