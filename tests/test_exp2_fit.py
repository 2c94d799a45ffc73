"""The FP32 software exponential's coefficients (hawkes_b200/csrc/hphc_sweep.cuh,
kP1..kP7) are the output of tests/fit_exp2.py, and that fit meets the error it
states: with the FP32 coefficients, max relative error below 4e-10 in FP64
evaluation and below 6.5e-8 with every Horner step rounded to FP32 (the
rounding of the last step alone is up to 6e-8), mean below 1e-10 in
magnitude."""
import os
import re

import numpy as np

import fit_exp2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KERNELS = os.path.join(ROOT, "hawkes_b200", "csrc", "hphc_sweep.cuh")


def kernel_coefficients():
    src = open(KERNELS).read()
    found = dict(re.findall(r"constexpr float kP(\d) = (0x[0-9a-fA-F.]+p[-+]?\d+)f;", src))
    return np.array([1.0] + [float.fromhex(found[str(k)]) for k in range(1, 8)])


def test_kernel_coefficients_are_the_fit():
    c = kernel_coefficients()
    fitted = fit_exp2.fit_fp32(7).astype(np.float32).astype(np.float64)
    assert np.array_equal(c, fitted), (c, fitted)


def test_fit_error_bounds():
    c32 = kernel_coefficients().astype(np.float32)
    x = np.linspace(-0.5, 0.5, 200001)
    e64 = np.polynomial.polynomial.polyval(x, c32.astype(np.float64)) / np.exp2(x) - 1.0
    x32 = x.astype(np.float32)
    e32 = fit_exp2.horner32(c32, x32).astype(np.float64) / np.exp2(x32.astype(np.float64)) - 1.0
    assert np.abs(e64).max() < 4e-10
    assert abs(e64.mean()) < 1e-10
    assert np.abs(e32).max() < 6.5e-8
    assert abs(e32.mean()) < 1e-10
