"""ORACLE -- test infrastructure only.

Python bindings of the two CPU checkers:

* ``liboracle.so`` -- the plain-C restatement in hawkes_oracle.c (log-likelihood,
  analytic gradient, probabilities; long-double accumulation), always built;
* ``_ref/libhawkes_ref.so`` -- the reference hpHawkes CPU engine compiled from
  its own sources (src/NewHawkes.hpp, src/factory.cpp) by oracle/Makefile.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this package, and only to check or time against it.  The product
(hawkes_b200/) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhawkes_ref.so")
REF_BENCHMARK = os.path.join(HERE, "_ref", "benchmark_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_oracle = None
_ref = None


def build(reference_src: str | None = None) -> None:
    """Build liboracle.so, and the reference artefacts when the reference's
    src/ directory is given (argument, else the HAWKES_REF_SRC environment
    variable) and exists."""
    subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)
    src = reference_src or os.environ.get("HAWKES_REF_SRC", "")
    if src and os.path.isdir(src):
        subprocess.run(["make", "-C", HERE, "ref", f"REF_SRC={src}"], check=True,
                       stdout=subprocess.DEVNULL)


def _oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.hawkes_oracle_eval.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                           ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.hawkes_oracle_eval.restype = ctypes.c_int
        lib.hawkes_oracle_pair_sums.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                                ctypes.c_int, _dp]
        lib.hawkes_oracle_pair_sums.restype = ctypes.c_int
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB} not built (needs the reference sources)")
        lib = ctypes.CDLL(REF_LIB)
        lib.ref_create.restype = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int]
        lib.ref_variant.restype = ctypes.c_char_p
        lib.ref_variant.argtypes = [ctypes.c_void_p]
        lib.ref_destroy.argtypes = [ctypes.c_void_p]
        for f in ("ref_set_times_data", "ref_set_parameters"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, _dp, ctypes.c_size_t]
        lib.ref_update_locations.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_size_t]
        lib.ref_get_sum_of_lik_contribs.restype = ctypes.c_double
        lib.ref_get_sum_of_lik_contribs.argtypes = [ctypes.c_void_p]
        lib.ref_get_probs_self_excite.argtypes = [ctypes.c_void_p, _dp, ctypes.c_size_t]
        lib.ref_store_state.argtypes = [ctypes.c_void_p]
        lib.ref_restore_state.argtypes = [ctypes.c_void_p]
        lib.ref_get_internal_dimension.argtypes = [ctypes.c_void_p]
        lib.ref_get_internal_dimension.restype = ctypes.c_int
        _ref = lib
    return _ref


FLAG_FLOAT = 1 << 2
FLAG_TBB = 1 << 3


class RefEngine:
    """The reference NewHawkes engine (serial by default; TBB-stub threads
    when ``threads`` > 0)."""

    def __init__(self, D: int, N: int, threads: int = 0, single: bool = False):
        lib = _ref_lib()
        flags = (FLAG_TBB if threads > 0 else 0) | (FLAG_FLOAT if single else 0)
        self._lib = lib
        self._h = lib.ref_create(D, N, flags, threads)
        if not self._h:
            raise RuntimeError("reference engine construction failed")
        self.D, self.N = D, N
        self.variant = lib.ref_variant(self._h).decode()

    def close(self):
        if self._h:
            self._lib.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_data(self, loc, times):
        loc = np.ascontiguousarray(loc, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(times, dtype=np.float64)
        self._lib.ref_set_times_data(self._h, t.ctypes.data_as(_dp), t.size)
        self._lib.ref_update_locations(self._h, -1, loc.ctypes.data_as(_dp), loc.size)

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        self._lib.ref_set_parameters(self._h, p.ctypes.data_as(_dp), p.size)

    def loglik(self) -> float:
        return self._lib.ref_get_sum_of_lik_contribs(self._h)

    def probs(self) -> np.ndarray:
        out = np.zeros(self.N)
        self._lib.ref_get_probs_self_excite(self._h, out.ctypes.data_as(_dp), self.N)
        return out


def ref_loglik(loc, times, params, threads: int = 0) -> float:
    loc = np.asarray(loc, dtype=np.float64)
    e = RefEngine(loc.shape[1], loc.shape[0], threads)
    e.set_data(loc, times)
    e.set_parameters(params)
    v = e.loglik()
    e.close()
    return v


def ref_probs(loc, times, params, threads: int = 0) -> np.ndarray:
    loc = np.asarray(loc, dtype=np.float64)
    e = RefEngine(loc.shape[1], loc.shape[0], threads)
    e.set_data(loc, times)
    e.set_parameters(params)
    v = e.probs()
    e.close()
    return v


def oracle_eval(loc, times, params, threads: int = 1) -> dict:
    """Log-likelihood, gradient, two gradient scales, probabilities and rates
    from the C restatement.

    grad_scale[k]      = sum_i |per-event contribution to d logL / d p_k|
    grad_term_scale[k] = sum_i of |each additive term| of that contribution
                         (e.g. |D/sigma S_i| + |sigma S_i d^2| for sigma): the
                         condition scale of the sum, which bounds what any
                         working precision can resolve."""
    loc = np.ascontiguousarray(loc, dtype=np.float64)
    t = np.ascontiguousarray(times, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    N, D = loc.shape
    ll = ctypes.c_double()
    g = np.zeros(6)
    ga = np.zeros(6)
    gm = np.zeros(6)
    probs = np.zeros(N)
    lam = np.zeros(N)
    st = _oracle_lib().hawkes_oracle_eval(D, N, loc.ctypes.data_as(_dp), t.ctypes.data_as(_dp),
                                          p.ctypes.data_as(_dp), int(threads), ctypes.byref(ll),
                                          g.ctypes.data_as(_dp), ga.ctypes.data_as(_dp),
                                          gm.ctypes.data_as(_dp), probs.ctypes.data_as(_dp),
                                          lam.ctypes.data_as(_dp))
    if st != 0:
        raise ValueError("oracle: bad arguments")
    return {"loglik": ll.value, "grad": g, "grad_scale": ga, "grad_term_scale": gm,
            "probs": probs, "lam": lam}


def oracle_pair_sums(loc, times, params, threads: int = 1) -> np.ndarray:
    """N x 6 unit pair sums (see hawkes_oracle_pair_sums)."""
    loc = np.ascontiguousarray(loc, dtype=np.float64)
    t = np.ascontiguousarray(times, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    N, D = loc.shape
    out = np.zeros((N, 6))
    st = _oracle_lib().hawkes_oracle_pair_sums(D, N, loc.ctypes.data_as(_dp),
                                               t.ctypes.data_as(_dp), p.ctypes.data_as(_dp),
                                               int(threads), out.ctypes.data_as(_dp))
    if st != 0:
        raise ValueError("oracle: bad arguments")
    return out
