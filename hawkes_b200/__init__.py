"""B200-native engine for the hpHawkes spatio-temporal Hawkes log-likelihood.

The compute path is libhawkes_b200.so (hand-written sm_100a CUDA kernels behind
the C ABI in include/hphc.h); this package is its Python host interface.
"""
from .engine import (  # noqa: F401
    AVX, AVX512, COMPENSATED, CUDA, FLOAT, FP32_FAST_EXP, FP32_ORDERED, FP32_SPACE_HILO, ORDERED,
    FAULT_LAUNCH, FAULT_UPLOAD, FAULT_WAIT, NO_FAST_TAIL, NO_INCREMENTAL, NO_TAIL_TRUNCATION,
    NO_UNDERFLOW_SKIP,
    OPENCL, PARAMETER_NAMES, PATH_INCREMENTAL, PATH_KEPT_SUMS, PATH_SELF_EXCITATION,
    PATH_SWEEP,
    PRECISION_FP32, PRECISION_FP32_COMP, PRECISION_FP64, SSE, TBB, CudaHawkes, Engine, HawkesError, Multiset,
    createEngine, engineInitial, factory, getGradient, getLogLikelihood, getProbsSelfExcite,
    setParameters, setTimesData, timeTest, updateLocations)
from .sampler import Potential, Sampler, log_prior, sampler  # noqa: F401

__all__ = [
    "CudaHawkes", "Engine", "HawkesError", "Multiset", "factory", "createEngine", "engineInitial",
    "updateLocations", "setTimesData", "setParameters", "getLogLikelihood",
    "getProbsSelfExcite", "getGradient", "timeTest", "PARAMETER_NAMES", "Sampler", "sampler",
    "Potential",
    "log_prior",
]
