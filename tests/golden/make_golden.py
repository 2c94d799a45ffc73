"""Generate the golden parity fixtures in tests/golden/ (run in a container
that has the reference sources; the fixtures are committed).

    python tests/golden/make_golden.py --reference <reference checkout>

(or HAWKES_REF set to the checkout).

Every expected log-likelihood and probability vector comes from the reference
hpHawkes CPU engine itself (src/NewHawkes.hpp, serial DOUBLE path), compiled
from its sources by oracle/Makefile into oracle/_ref/libhawkes_ref.so; the
``ref_float_*`` fields come from the same engine's single-precision path
(FLOAT, src/factory.cpp:45: every pair term, sum, log and CDF in float).  The
reference has no live gradient; expected gradients are the oracle's analytic
gradient (oracle/hawkes_oracle.c), stored together with central finite
differences of the reference engine's log-likelihood that pin it.

Cases (inputs are stored with the outputs, so no generator has to be
re-run to check them):
  c1_uniform   N=1000, D=2, 20x20 km box, times U[0,8760) h sorted, seed 0,
               base parameters (sigma=1, tauX=1/1.6, tauT=1/336, omega=1,
               theta=1, mu0=1).
  edge_N<n>    N in {1,2,3,31,32,33,127,128,129,255,256,257,511,513}, D=2.
  ties         N=200, times drawn from 40 distinct integers (many exact ties).
  unsorted     N=300, times not sorted, the latest one last (T = t[N-1] as the
               reference defines it).
  dim<d>       D in {1,3,4,8}, N=150.
  params<k>    N=500, five log-normal parameter vectors around the base.
  dcdata_*     the reference's own data file data/dcData.RData (5022 DC
               gunfire events: X, Y in km, Time in hours), README parameters
               c(1, 1/1.6, 1/(14*24), 1, 1, 1) and one perturbed vector.
"""
from __future__ import annotations

import argparse
import gzip
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from hawkes_b200 import workloads  # noqa: E402

BASE = workloads.BASE_PARAMS


def read_rdata_columns(path: str) -> dict:
    """Minimal reader for the R XDR (version 2) serialization of a data frame
    of REALSXP columns, as stored in data/dcData.RData.  Returns the columns
    by name."""
    buf = gzip.open(path).read()
    assert buf[:5] == b"RDX2\n", "not an RDX2 file"
    cols = []
    names = None
    pos = 0
    while True:
        # REALSXP (type 14) headers followed by a 32-bit length.
        k = buf.find(struct.pack(">i", 14), pos)
        if k < 0:
            break
        # flags word: type in the low byte; we look for the exact flags 0x0000000e
        n = struct.unpack(">i", buf[k + 4:k + 8])[0]
        if n > 1000 and k + 8 + 8 * n <= len(buf):
            cols.append(np.frombuffer(buf[k + 8:k + 8 + 8 * n], dtype=">f8").astype(np.float64))
            pos = k + 8 + 8 * n
        else:
            pos = k + 4
    # names attribute: STRSXP (type 16) of length len(cols), CHARSXPs follow
    k = buf.find(struct.pack(">i", 16) + struct.pack(">i", len(cols)), pos - 1)
    if k >= 0:
        p = k + 8
        names = []
        for _ in range(len(cols)):
            p += 4  # CHARSXP flags
            ln = struct.unpack(">i", buf[p:p + 4])[0]
            p += 4
            names.append(buf[p:p + ln].decode())
            p += ln
    if names is None:
        names = [f"V{i}" for i in range(len(cols))]
    return dict(zip(names, cols))


def reference_outputs(loc, t, p, single=False):
    eng = oracle.RefEngine(loc.shape[1], loc.shape[0], threads=0, single=single)
    eng.set_data(loc, t)
    eng.set_parameters(p)
    ll = eng.loglik()
    pr = eng.probs()
    variant = eng.variant
    eng.close()
    return ll, pr, variant


def fd_gradient(loc, t, p, rel_step=1e-6):
    eng = oracle.RefEngine(loc.shape[1], loc.shape[0], threads=0)
    eng.set_data(loc, t)
    g = np.zeros(6)
    for k in range(6):
        h = rel_step * abs(p[k])
        q = p.copy()
        q[k] = p[k] + h
        eng.set_parameters(q)
        up = eng.loglik()
        q[k] = p[k] - h
        eng.set_parameters(q)
        dn = eng.loglik()
        g[k] = (up - dn) / (2 * h)
    eng.close()
    return g


def case(name, loc, t, p, store, fd=True):
    loc = np.ascontiguousarray(loc, dtype=np.float64)
    t = np.ascontiguousarray(t, dtype=np.float64)
    p = np.asarray(p, dtype=np.float64)
    ll, pr, variant = reference_outputs(loc, t, p)
    ll32, pr32, _ = reference_outputs(loc, t, p, single=True)
    o = oracle.oracle_eval(loc, t, p, threads=8)
    entry = {
        "loc": loc, "t": t, "params": p,
        "ref_loglik": np.float64(ll), "ref_probs": pr,
        "ref_float_loglik": np.float64(ll32), "ref_float_probs": pr32,
        "oracle_grad": o["grad"], "grad_scale": o["grad_scale"],
        "grad_term_scale": o["grad_term_scale"],
    }
    if fd:
        entry["fd_grad"] = fd_gradient(loc, t, p)
    store[name] = entry
    print(f"{name:14s} N={len(t):5d} D={loc.shape[1]} ref logL={ll:.12f} "
          f"(oracle rel {abs(o['loglik'] - ll) / max(abs(ll), 1e-300):.1e}) [{variant}]")


def save(store, fname):
    flat = {}
    for name, entry in store.items():
        for k, v in entry.items():
            flat[f"{name}__{k}"] = v
    np.savez_compressed(os.path.join(HERE, fname), **flat)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("HAWKES_REF", ""),
                    help="the reference checkout (its src/ and data/ are read)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("--reference (or HAWKES_REF) is required")
    oracle.build(os.path.join(args.reference, "src"))

    synth = {}
    loc, t = workloads.uniform(1000, seed=0)
    case("c1_uniform", loc, t, BASE, synth)
    for n in (1, 2, 3, 31, 32, 33, 127, 128, 129, 255, 256, 257, 511, 513):
        loc, t = workloads.uniform(n, seed=n)
        case(f"edge_N{n}", loc, t, BASE, synth, fd=n <= 257)
    rng = np.random.default_rng(77)
    loc = rng.uniform(0, 20, size=(200, 2))
    t = np.sort(rng.integers(0, 40, size=200).astype(np.float64) * 3.0)
    case("ties", loc, t, BASE, synth)
    rng = np.random.default_rng(78)
    loc = rng.uniform(0, 20, size=(300, 2))
    t = rng.uniform(0, 8760, size=300)
    m = int(np.argmax(t))
    t[m], t[-1] = t[-1], t[m]  # unsorted, but T = t[N-1] is the latest time
    case("unsorted", loc, t, BASE, synth)
    for d in (1, 3, 4, 8):
        loc, t = workloads.uniform(150, seed=100 + d, D=d)
        case(f"dim{d}", loc, t, BASE, synth)
    loc, t = workloads.uniform(500, seed=9)
    for k, p in enumerate(workloads.proposals(5, seed=11)):
        case(f"params{k}", loc, t, p, synth)
    save(synth, "synthetic.npz")

    dc = read_rdata_columns(os.path.join(args.reference, "data", "dcData.RData"))
    x, y, tt = dc["X"], dc["Y"], dc["Time"]
    loc = np.stack([x, y], axis=1)
    real = {}
    case("dcdata_readme", loc, tt, BASE, real, fd=False)
    case("dcdata_perturbed", loc, tt, BASE * np.array([1.3, 0.8, 1.5, 0.5, 0.4, 2.0]), real,
         fd=False)
    save(real, "dcdata.npz")


if __name__ == "__main__":
    main()
