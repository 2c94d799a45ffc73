"""Seeded synthetic event sets with the shapes of the benchmark workloads.

No public dataset is involved: every workload is drawn with
``numpy.random.default_rng(seed)`` in FP64, D = 2 unless stated.

* ``uniform``   -- N events, locations i.i.d. U[0, box)^D km, times i.i.d.
                   U[0, horizon) h sorted ascending.
* ``proposals`` -- K parameter vectors ``base * exp(sd * z)``, z ~ N(0, I_6),
                   the batched-proposal workload.
* ``uneven``    -- S independent uniform sets with sizes log-uniform in
                   [lo, hi], each with its own log-normal parameter vector.
* ``clustered`` -- a Hawkes branching process: homogeneous Poisson background
                   in a box over [0, horizon) with an oversample, Poisson(m)
                   offspring per event, recursively, offsets N(0, s^2 I) km and
                   Exp(rate) h; events past the horizon are dropped, the rest
                   sorted by time and the first N kept.

BASE_PARAMS are the reference's default sampler parameters
(R/Untitled.R:259, README.md:74-79): sigma = 1, tauX = 1/1.6, tauT = 1/(14*24),
omega = 1, theta = 1, mu0 = 1.
"""
from __future__ import annotations

import numpy as np

BASE_PARAMS = np.array([1.0, 1.0 / 1.6, 1.0 / (14 * 24), 1.0, 1.0, 1.0])


def uniform(N: int, seed: int, D: int = 2, box: float = 20.0, horizon: float = 8760.0,
            rng: np.random.Generator | None = None):
    """(locations N x D, times N sorted)."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    loc = rng.uniform(0.0, box, size=(N, D))
    t = np.sort(rng.uniform(0.0, horizon, size=N))
    return loc, t


def proposals(K: int, seed: int, base=BASE_PARAMS, sd: float = 0.3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    z = rng.standard_normal(size=(K, 6))
    return np.asarray(base)[None, :] * np.exp(sd * z)


def uneven(S: int, seed: int, lo: int = 1000, hi: int = 100000, D: int = 2, base=BASE_PARAMS,
           sd: float = 0.3):
    """List of (locations, times, params) for S sets."""
    rng = np.random.default_rng(seed)
    sizes = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=S))).astype(int)
    sets = []
    for n in sizes:
        loc, t = uniform(int(n), 0, D=D, rng=rng)
        p = np.asarray(base) * np.exp(sd * rng.standard_normal(6))
        sets.append((loc, t, p))
    return sets


def clustered(N: int = 500000, seed: int = 4, background: int = 250000,
              oversample: float = 0.04, box: float = 50.0, horizon: float = 8760.0,
              mean_offspring: float = 0.5, offset_sd: float = 0.5, rate: float = 1.0):
    """(locations N x 2, times N sorted) from the branching process."""
    rng = np.random.default_rng(seed)
    nb = int(round(background * (1.0 + oversample)))
    px = rng.uniform(0.0, box, size=(nb, 2))
    pt = rng.uniform(0.0, horizon, size=nb)
    xs, ts = [px], [pt]
    while pt.size:
        k = rng.poisson(mean_offspring, size=pt.size)
        idx = np.repeat(np.arange(pt.size), k)
        cx = px[idx] + rng.normal(0.0, offset_sd, size=(idx.size, 2))
        ct = pt[idx] + rng.exponential(1.0 / rate, size=idx.size)
        keep = ct < horizon
        px, pt = cx[keep], ct[keep]
        xs.append(px)
        ts.append(pt)
    x = np.concatenate(xs)
    t = np.concatenate(ts)
    order = np.argsort(t, kind="stable")[:N]
    return np.ascontiguousarray(x[order]), np.ascontiguousarray(t[order])
