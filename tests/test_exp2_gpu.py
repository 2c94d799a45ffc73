"""The two exponentials of the FP32 sweep, evaluated on the device
(hphc_eval_exponentials) and checked against FP64 exp2:

* the software exponential 2^-s (Cody-Waite reduction, degree-7 polynomial
  fitted by tests/fit_exp2.py, exact power of two): relative error at most
  8e-8 (the 6.3e-8 of FP32 Horner evaluation plus the polynomial's 3.4e-10),
  mean below 2e-10 in magnitude over a dense grid of s in [0, 125.5], and
  exactly +0 from s = 127 on (the tile-level underflow skip relies on it);
* the hardware ex2.approx.ftz used for far-tail background terms (each at
  most 2^-10 of an event's own term, s in [10, 91]): relative error below
  2^-21 everywhere, a mean between -8e-8 and -2e-8, and the same mean (to
  5e-9) as over [0, 16), where the engine measures the bias it divides out.
"""
import ctypes

import numpy as np
import pytest

from hawkes_b200 import _native

pytestmark = pytest.mark.gpu

_fp = ctypes.POINTER(ctypes.c_float)


def device_exponentials(s):
    s = np.ascontiguousarray(s, dtype=np.float32)
    poly = np.empty_like(s)
    hw = np.empty_like(s)
    st = _native.lib.hphc_eval_exponentials(0, s.ctypes.data_as(_fp), s.size,
                                            poly.ctypes.data_as(_fp), hw.ctypes.data_as(_fp))
    assert st == 0, _native.lib.hphc_status_string(st).decode()
    return poly, hw


def rel_error(y, s):
    exact = np.exp2(-s.astype(np.float64))
    return y.astype(np.float64) / exact - 1.0


def test_polynomial_exponential():
    grid = np.linspace(0.0, 125.5, 1 << 22).astype(np.float32)
    ints = np.arange(0, 126).astype(np.float32)
    halves = ints + np.float32(0.5)
    s = np.concatenate([grid, ints, halves[:-1]])
    poly, _ = device_exponentials(s)
    e = rel_error(poly, s)
    print(f"\npolynomial: max |rel| {np.abs(e).max():.3e}, mean {e[:grid.size].mean():+.3e}")
    assert np.abs(e).max() <= 8e-8
    assert abs(e[:grid.size].mean()) <= 2e-10
    under = np.concatenate([np.linspace(127.0, 300.0, 4097), [1e6, 3e38]]).astype(np.float32)
    pu, _ = device_exponentials(under)
    assert np.all(pu == 0.0)


def test_hardware_exponential_far_tail():
    far = np.linspace(10.0, 91.0, 1 << 21).astype(np.float32)
    near = np.linspace(0.0, 16.0, 1 << 21, endpoint=False).astype(np.float32)
    _, hf = device_exponentials(far)
    _, hn = device_exponentials(near)
    ef, en = rel_error(hf, far), rel_error(hn, near)
    print(f"\nex2.approx: far max |rel| {np.abs(ef).max():.3e} mean {ef.mean():+.3e}; "
          f"[0,16) mean {en.mean():+.3e}")
    assert np.abs(ef).max() <= 2.0 ** -21
    assert -8e-8 <= ef.mean() <= -2e-8
    assert abs(ef.mean() - en.mean()) <= 5e-9
