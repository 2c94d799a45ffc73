"""CPU tests of the C ABI boundary: the library loads, exports every entry
point include/hphc.h declares, and validates arguments that need no device."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hphc.h")
LIB = os.path.join(ROOT, "hawkes_b200", "libhawkes_b200.so")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hphc_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_interface():
    names = declared_functions()
    for required in ("hphc_create", "hphc_destroy", "hphc_set_times_data",
                     "hphc_update_locations", "hphc_set_parameters",
                     "hphc_get_sum_of_lik_contribs", "hphc_get_log_likelihood_gradient",
                     "hphc_get_probs_self_excite", "hphc_store_state", "hphc_restore_state",
                     "hphc_accept_state", "hphc_get_internal_dimension"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    from hawkes_b200 import _native
    assert set(declared_functions()) <= set(_native.SIGNATURES)


def test_status_strings():
    from hawkes_b200._native import lib
    for code in range(0, 12):
        s = lib.hphc_status_string(code).decode()
        assert s and s != "unknown status"
    assert lib.hphc_status_string(99).decode() == "unknown status"


def test_create_validates_before_touching_a_device():
    from hawkes_b200._native import lib
    h = ctypes.c_void_p()
    assert lib.hphc_create(0, 10, 0, 0, ctypes.byref(h)) == 5   # D < 1: unsupported
    assert lib.hphc_create(9, 10, 0, 0, ctypes.byref(h)) == 5   # D > 8: unsupported
    assert lib.hphc_create(2, 0, 0, 0, ctypes.byref(h)) == 3    # N < 1: bad argument
    assert lib.hphc_create(2, 10, 0, 0, None) == 3              # null out
    assert not h.value


def test_null_handle_is_rejected_everywhere():
    from hawkes_b200._native import lib
    d = ctypes.c_double()
    buf = (ctypes.c_double * 6)()
    assert lib.hphc_set_times_data(None, buf, 6) == 1
    assert lib.hphc_update_locations(None, -1, buf, 6) == 1
    assert lib.hphc_set_parameters(None, buf, 6) == 1
    assert lib.hphc_get_sum_of_lik_contribs(None, ctypes.byref(d)) == 1
    assert lib.hphc_get_log_likelihood_gradient(None, buf, 6) == 1
    assert lib.hphc_get_probs_self_excite(None, buf, 6) == 1
    assert lib.hphc_store_state(None) == 1
    assert lib.hphc_restore_state(None) == 1
    assert lib.hphc_accept_state(None) == 1
    lib.hphc_destroy(None)  # no-op
    assert lib.hphc_last_error(None).decode() == "invalid handle"


def _has_gpu():
    from hawkes_b200._native import lib
    h = ctypes.c_void_p()
    st = lib.hphc_create(2, 4, 0, 0, ctypes.byref(h))
    if st == 0:
        lib.hphc_destroy(h)
    return st == 0


def test_no_device_is_reported_not_faked():
    if _has_gpu():
        pytest.skip("a GPU is visible")
    import hawkes_b200 as hb
    with pytest.raises(hb.HawkesError) as ei:
        hb.CudaHawkes(2, 100, hb.CUDA)
    assert ei.value.status == 9


def test_python_factory_and_r_mirror_validation():
    import hawkes_b200 as hb
    with pytest.raises(hb.HawkesError):
        hb.factory(2, 10, 0)  # no GPU flag: this package only provides the GPU engine
    with pytest.raises(hb.HawkesError):
        hb.createEngine(2, 10, gpu=0)
