"""ctypes binding of libhawkes_b200.so (the C ABI declared in include/hphc.h).

The library is built in-tree by ``hawkes_b200/csrc/Makefile`` (or
``__graft_entry__.build()``).  There is no CPU fallback: if the library is
missing or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libhawkes_b200.so")

# Every entry point declared in include/hphc.h, with its ctypes signature.
_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_int_p = ctypes.POINTER(ctypes.c_int)
_handle = ctypes.c_void_p

SIGNATURES = {
    "hphc_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_void_p)]),
    "hphc_destroy": (None, [_handle]),
    "hphc_last_error": (ctypes.c_char_p, [_handle]),
    "hphc_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "hphc_set_times_data": (ctypes.c_int, [_handle, _c_double_p, ctypes.c_size_t]),
    "hphc_update_locations": (ctypes.c_int, [_handle, ctypes.c_int, _c_double_p, ctypes.c_size_t]),
    "hphc_set_parameters": (ctypes.c_int, [_handle, _c_double_p, ctypes.c_size_t]),
    "hphc_get_sum_of_lik_contribs": (ctypes.c_int, [_handle, _c_double_p]),
    "hphc_get_log_likelihood_gradient": (ctypes.c_int, [_handle, _c_double_p, ctypes.c_size_t]),
    "hphc_get_log_likelihood_and_gradient": (ctypes.c_int, [_handle, _c_double_p, _c_double_p,
                                                            ctypes.c_size_t]),
    "hphc_get_probs_self_excite": (ctypes.c_int, [_handle, _c_double_p, ctypes.c_size_t]),
    "hphc_store_state": (ctypes.c_int, [_handle]),
    "hphc_restore_state": (ctypes.c_int, [_handle]),
    "hphc_accept_state": (ctypes.c_int, [_handle]),
    "hphc_get_internal_dimension": (ctypes.c_int, [_handle, _c_int_p]),
    "hphc_batch_log_likelihood_and_gradient": (ctypes.c_int, [_handle, _c_double_p, ctypes.c_int,
                                                              _c_double_p, _c_double_p]),
    "hphc_get_precision": (ctypes.c_int, [_handle, _c_int_p]),
    "hphc_get_stream": (ctypes.c_int, [_handle, ctypes.POINTER(ctypes.c_void_p)]),
    "hphc_enqueue_log_likelihood_and_gradient": (ctypes.c_int, [_handle]),
    "hphc_read_results": (ctypes.c_int, [_handle, _c_double_p, _c_double_p, ctypes.c_size_t]),
    "hphc_get_last_launch_stats": (ctypes.c_int, [_handle, _c_int_p, _c_double_p, _c_double_p]),
    "hphc_get_last_launch_evals": (ctypes.c_int, [_handle, _c_double_p]),
    "hphc_get_last_evaluation_path": (ctypes.c_int, [_handle, _c_int_p]),
    "hphc_loglik_grad_fp64_static": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                    ctypes.c_void_p, _c_double_p,
                                                    ctypes.c_void_p, ctypes.c_void_p]),
    "hphc_sweep_shard": (ctypes.c_int, [_handle, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_size_t]),
    "hphc_set_unit_sums": (ctypes.c_int, [_handle, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_size_t]),
    "hphc_inject_fault": (ctypes.c_int, [_handle, ctypes.c_int, ctypes.c_int]),
    "hphc_eval_exponentials": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                              ctypes.c_size_t, ctypes.POINTER(ctypes.c_float),
                                              ctypes.POINTER(ctypes.c_float)]),
    "hphc_set_kernel_timing": (ctypes.c_int, [_handle, ctypes.c_int]),
    "hphc_set_sweep_shape": (ctypes.c_int, [_handle, ctypes.c_int, ctypes.c_int]),
    "hphc_get_sweep_shape": (ctypes.c_int, [_handle, _c_int_p, _c_int_p]),
    "hphc_get_kernel_times": (ctypes.c_int, [_handle, ctypes.POINTER(ctypes.c_float),
                                             ctypes.POINTER(ctypes.c_float),
                                             ctypes.POINTER(ctypes.c_float)]),
    "hphc_multiset_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _c_int_p, ctypes.c_long,
                                            ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "hphc_multiset_destroy": (None, [_handle]),
    "hphc_multiset_last_error": (ctypes.c_char_p, [_handle]),
    "hphc_multiset_set_data": (ctypes.c_int, [_handle, ctypes.c_int, _c_double_p, ctypes.c_size_t,
                                              _c_double_p, ctypes.c_size_t]),
    "hphc_multiset_log_likelihood_and_gradient": (ctypes.c_int, [_handle, _c_double_p, _c_double_p,
                                                                 _c_double_p]),
    "hphc_multiset_set_kernel_timing": (ctypes.c_int, [_handle, ctypes.c_int]),
    "hphc_multiset_get_kernel_times": (ctypes.c_int, [_handle, ctypes.POINTER(ctypes.c_float),
                                                      ctypes.POINTER(ctypes.c_float),
                                                      ctypes.POINTER(ctypes.c_float)]),
    "hphc_multiset_get_last_launch_evals": (ctypes.c_int, [_handle, _c_double_p]),
    "hphc_multiset_get_last_launch_stats": (ctypes.c_int, [_handle, _c_int_p, _c_double_p,
                                                           _c_double_p]),
    "hphc_sampler_create": (ctypes.c_int, [ctypes.c_int, _c_double_p, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_ulonglong,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "hphc_sampler_destroy": (None, [_handle]),
    "hphc_sampler_last_error": (ctypes.c_char_p, [_handle]),
    "hphc_sampler_run": (ctypes.c_int, [_handle, _handle, ctypes.c_int, ctypes.c_int, _c_double_p,
                                        _c_double_p]),
    "hphc_sampler_run_device": (ctypes.c_int, [_handle, _handle, ctypes.c_int, ctypes.c_int,
                                               _c_double_p, _c_double_p]),
    "hphc_sampler_run_with": (ctypes.c_int, [_handle, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_int, _c_double_p,
                                             _c_double_p]),
    "hphc_sampler_get_state": (ctypes.c_int, [_handle, _c_double_p, _c_double_p, _c_double_p,
                                              ctypes.POINTER(ctypes.c_longlong),
                                              ctypes.POINTER(ctypes.c_longlong)]),
}

# Signature of hphc_batch_loglik_fn (a batched log-likelihood evaluator).
BATCH_LOGLIK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, _c_double_p, ctypes.c_int,
                                   _c_double_p)


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIBRARY_PATH):
        raise ImportError(
            f"{LIBRARY_PATH} is missing: build it with `make -C hawkes_b200/csrc` "
            "(the CUDA engine has no CPU fallback)")
    lib = ctypes.CDLL(LIBRARY_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()
