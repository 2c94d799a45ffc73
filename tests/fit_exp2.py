"""Fit the polynomial used by the FP32 software exponential (hawkes_b200/csrc/hphc_sweep.cuh).

    python tests/fit_exp2.py [degree]

2^x is evaluated as 2^n * p(f) with n = round(x), f = x - n in [-1/2, 1/2]
(Cody-Waite range reduction, W. J. Cody and W. Waite, "Software Manual for the
Elementary Functions", 1980).  p is fitted here to 2^f in relative error: a
weighted least-squares fit at Chebyshev nodes followed by Remez-style
re-weighting (Lawson's algorithm) towards the minimax solution.  The printed
coefficients are rounded to FP32 and the resulting error is checked on a dense
grid in FP64 and with FP32 Horner evaluation (each step rounded to FP32).
"""
import sys

import numpy as np


def fit(deg: int, iters: int = 60, fixed=()):
    """Coefficients c_0..c_deg; the first len(fixed) are held at the given
    values and the rest fitted (relative error, near-minimax)."""
    m = 4000
    k = np.arange(m)
    f = 0.5 * np.cos(np.pi * (k + 0.5) / m)  # Chebyshev nodes on [-1/2, 1/2]
    target = np.exp2(f)
    nf = len(fixed)
    V = np.vander(f, deg + 1, increasing=True)
    rhs0 = target - (V[:, :nf] @ np.asarray(fixed, dtype=np.float64) if nf else 0.0)
    w = np.ones(m)
    c = None
    for _ in range(iters):  # Lawson: multiplicative weight update towards minimax
        A = V[:, nf:] * (w / target)[:, None]
        c, *_ = np.linalg.lstsq(A, rhs0 * w / target, rcond=None)
        full = np.concatenate([np.asarray(fixed, dtype=np.float64), c])
        err = np.abs(V @ full / target - 1.0)
        w = w * (err / err.max() + 1e-3)
        w /= w.sum()
    return np.concatenate([np.asarray(fixed, dtype=np.float64), c])


def fit_fp32(deg: int):
    """Sequential rounding: c_0 = 1 exactly, then each coefficient is rounded
    to FP32 and the higher ones are refitted to absorb its rounding error."""
    fixed = [1.0]
    for _ in range(1, deg + 1):
        c = fit(deg, fixed=fixed)
        fixed.append(float(np.float32(c[len(fixed)])))
    return np.asarray(fixed)


def horner32(c32, f32):
    p = np.float32(c32[-1]) * np.ones_like(f32)
    for ck in c32[-2::-1]:
        p = (p.astype(np.float64) * f32.astype(np.float64) + np.float64(ck)).astype(np.float32)
    return p


def main():
    deg = int(sys.argv[1]) if len(sys.argv) > 1 else 7
    c32 = fit_fp32(deg).astype(np.float32)
    x = np.linspace(-0.5, 0.5, 200001)
    exact = np.exp2(x)
    e64 = np.polynomial.polynomial.polyval(x, c32.astype(np.float64)) / exact - 1.0
    x32 = x.astype(np.float32)
    e32 = horner32(c32, x32).astype(np.float64) / np.exp2(x32.astype(np.float64)) - 1.0
    print(f"degree {deg}: FP32 coefficients, FP64 evaluation max rel err {np.abs(e64).max():.3e}"
          f" (mean {e64.mean():+.2e}); FP32 Horner max {np.abs(e32).max():.3e}"
          f" mean {e32.mean():+.2e}")
    for i, v in enumerate(c32):
        print(f"  c{i} = {float(v).hex()}  ({float(v):.9e})")


if __name__ == "__main__":
    main()
