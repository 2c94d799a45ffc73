"""GPU parity tests: the CUDA engine (through the C ABI) against the reference
engine's outputs (golden fixtures) and the oracle.

Tolerances
  FP64 plain        log-likelihood relative 1e-10; probabilities 1e-10 absolute;
                    gradient 1e-10 of its absolute scale (sum over events of
                    |per-event contribution|, per component).
  FP32-compensated  at the small fixture sizes: log-likelihood relative 1e-7,
                    gradient 5e-6 of its term-level scale (sum over events of
                    |each additive term| of the contribution, e.g.
                    |D/sigma S_i| + |sigma S_i d^2|), probabilities 2e-5 absolute.
                    (The 1e-8 target is checked at N=50,000 in
                    test_accuracy_gpu.py.)
"""
import ctypes

import numpy as np
import pytest

import hawkes_b200 as hb
import oracle
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

FP64 = hb.CUDA
FP32C = hb.CUDA | hb.COMPENSATED
FP32F = hb.CUDA | hb.COMPENSATED | hb.FP32_FAST_EXP
FP32O = hb.CUDA | hb.COMPENSATED | hb.ORDERED
FP64O = hb.CUDA | hb.ORDERED
TOL = {FP64: dict(ll=1e-10, grad=1e-10, probs=1e-10),
       FP64O: dict(ll=1e-10, grad=1e-10, probs=1e-10),
       FP32C: dict(ll=1e-7, grad=5e-6, probs=2e-5),
       FP32F: dict(ll=1e-7, grad=5e-6, probs=2e-5),
       FP32O: dict(ll=1e-7, grad=5e-6, probs=2e-5)}
MODES = [FP64, FP64O, FP32C, FP32F, FP32O]
IDS = ["fp64", "fp64_ordered", "fp32c", "fp32c_fast", "fp32c_ordered"]


def engine(loc, t, p, flags):
    loc = np.asarray(loc, dtype=np.float64)
    e = hb.CudaHawkes(loc.shape[1], loc.shape[0], flags, 0)
    e.setTimesData(t)
    e.updateLocations(-1, loc.reshape(-1))
    e.setParameters(p)
    return e


def check_case(name, c, flags):
    tol = TOL[flags]
    with engine(c["loc"], c["t"], c["params"], flags) as e:
        ll, g = e.getLogLikelihoodAndGradient()
        probs = e.getProbsSelfExcite()
        ll2 = e.getSumOfLikContribs()
        g2 = e.getLogLikelihoodGradient()
    ref = float(c["ref_loglik"])
    assert abs(ll - ref) <= tol["ll"] * abs(ref), (name, ll, ref)
    assert ll == ll2 and np.array_equal(g, g2), name
    # FP64: against the per-event scale; FP32: against the term-level scale
    # (the condition scale of the sum, which is what FP32 pair terms resolve)
    fp64 = flags in (FP64, FP64O)
    key = "grad_scale" if fp64 else "grad_term_scale"
    scale = np.maximum(c[key], 1e-300)
    allowed = tol["grad"] * scale
    if not fp64:
        # An FP32 exponent e (log2 units, |e| <= 126) carries an absolute
        # error ~|e| 2^-23, so a pair term far out in its kernel is resolved
        # only to ~1e-6 relative, and terms below 2^-126 flush to zero.  A
        # component made only of such terms (d/d sigma, d/d omega when events
        # are sparse in time; d/d sigma ~ 1e-23 in the 8-D case) is checked
        # against an absolute floor of 1e-12 of the largest component scale.
        allowed = allowed + 1e-12 * np.max(c[key])
    gerr = np.abs(g - c["oracle_grad"]) / allowed
    assert np.all(gerr <= 1.0), (name, gerr)
    perr = np.max(np.abs(probs - c["ref_probs"]))
    assert perr <= tol["probs"], (name, perr)


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_golden_synthetic(golden_synthetic, flags):
    for name, c in sorted(golden_synthetic.items()):
        check_case(name, c, flags)


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_golden_dcdata(golden_dcdata, flags):
    for name, c in sorted(golden_dcdata.items()):
        check_case(name, c, flags)


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_random_cases_against_oracle(flags):
    rng = np.random.default_rng(2024)
    for trial in range(6):
        D = int(rng.integers(1, 9))
        N = int(rng.integers(1, 1500))
        loc = rng.uniform(0, 15, size=(N, D))
        t = np.sort(rng.uniform(0, 3000, size=N))
        p = workloads.BASE_PARAMS * np.exp(0.4 * rng.standard_normal(6))
        o = oracle.oracle_eval(loc, t, p, threads=8)
        c = {"loc": loc, "t": t, "params": p, "ref_loglik": o["loglik"],
             "ref_probs": o["probs"], "oracle_grad": o["grad"], "grad_scale": o["grad_scale"],
             "grad_term_scale": o["grad_term_scale"]}
        check_case(f"trial{trial}_D{D}_N{N}", c, flags)


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_block_boundary_sizes_against_oracle(flags):
    # Event counts at tile (128) and strip (256 events at R = 2, 512 at R = 4)
    # boundaries, with tie-heavy times: the last partial tile and strip, the
    # padding rows and columns, and (FP32 modes) the spatial row order of the
    # full strips, at both strip heights.
    rng = np.random.default_rng(131)
    shapes = [(1, 16), (2, 16)] if flags == FP64 else [(2, 16), (4, 16)]
    for N in (1, 2, 127, 128, 129, 255, 256, 257, 511, 512, 513):
        loc = rng.uniform(0, 6, size=(N, 2))
        t = np.sort(np.round(rng.uniform(0, 400, size=N), 0))  # many exact ties
        p = workloads.BASE_PARAMS * np.array([1.0, 1.0, 4.0, 1.0, 1.0, 1.0])
        o = oracle.oracle_eval(loc, t, p, threads=8)
        tol = TOL[flags]
        key = "grad_scale" if flags == FP64 else "grad_term_scale"
        allowed = tol["grad"] * np.maximum(o[key], 1e-300) + \
            (0.0 if flags == FP64 else 1e-12 * np.max(o[key]))
        for shape in shapes:
            with engine(loc, t, p, flags) as e:
                e.setSweepShape(*shape)
                ll, g = e.getLogLikelihoodAndGradient()
                probs = e.getProbsSelfExcite()
            tag = (N, shape)
            assert abs(ll - o["loglik"]) <= tol["ll"] * abs(o["loglik"]), tag
            assert np.all(np.abs(np.asarray(g) - o["grad"]) <= allowed), tag
            assert np.max(np.abs(probs - o["probs"])) <= tol["probs"], tag


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_wide_kernels_against_oracle(flags):
    # Self-excitation kernels wider than the background's: a small sigma
    # (wide in space) and a small omega (slow decay) make single terms of the
    # sums S d'^2 and S dt' exceed 1 in record units, so the compensated row
    # sums start from a larger power-of-two offset there (here 8 and 2 for
    # S d'^2 in the first two cases, 2 for S dt' in the last).
    rng = np.random.default_rng(91)
    for N, D, scale in ((1200, 2, (0.2, 1.0, 1.0, 0.05, 1.0, 1.0)),
                        (900, 3, (0.35, 1.0, 2.0, 0.2, 0.5, 2.0)),
                        (800, 2, (0.5, 1.0, 1.0, 5e-4, 1.0, 1.0))):
        loc = rng.uniform(0, 12, size=(N, D))
        t = np.sort(rng.uniform(0, 2000, size=N))
        p = workloads.BASE_PARAMS * np.array(scale)
        o = oracle.oracle_eval(loc, t, p, threads=8)
        c = {"loc": loc, "t": t, "params": p, "ref_loglik": o["loglik"],
             "ref_probs": o["probs"], "oracle_grad": o["grad"], "grad_scale": o["grad_scale"],
             "grad_term_scale": o["grad_term_scale"]}
        check_case(f"wide_D{D}_N{N}", c, flags)


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_unsorted_times_against_oracle(flags):
    # Times in no particular order (the last one is the largest, so T bounds
    # them): every tile pair may hold self-excitation terms in either order.
    rng = np.random.default_rng(77)
    for N, D in ((1000, 2), (700, 3)):
        loc = rng.uniform(0, 10, size=(N, D))
        t = rng.uniform(0, 500, size=N)
        k = int(np.argmax(t))
        t[[k, N - 1]] = t[[N - 1, k]]
        t[: N // 3] = np.sort(t[: N // 3])  # partly sorted, partly not
        p = workloads.BASE_PARAMS * np.array([1.0, 1.0, 3.0, 1.0, 1.0, 1.0])
        o = oracle.oracle_eval(loc, t, p, threads=8)
        c = {"loc": loc, "t": t, "params": p, "ref_loglik": o["loglik"],
             "ref_probs": o["probs"], "oracle_grad": o["grad"], "grad_scale": o["grad_scale"],
             "grad_term_scale": o["grad_term_scale"]}
        check_case(f"unsorted_D{D}_N{N}", c, flags)


@pytest.mark.parametrize("sym,ordered", [(FP32C, FP32O), (FP64, FP64O)], ids=["fp32c", "fp64"])
def test_symmetric_sweep_halves_background_work(sym, ordered):
    # Each background pair with an earlier tile is evaluated once for both
    # events: the same terms are accounted for with about half the exponentials.
    loc, t = workloads.uniform(30000, seed=21)
    p = workloads.BASE_PARAMS
    with engine(loc, t, p, sym) as s, engine(loc, t, p, ordered) as o:
        for e in (s, o):
            e.setSweepShape(2, 16)
        ls, gs = s.getLogLikelihoodAndGradient()
        lo, go = o.getLogLikelihoodAndGradient()
        _, nbs, nss = s.lastLaunchStats()
        _, nbo, nso = o.lastLaunchStats()
        evs, evo = s.lastLaunchEvals(), o.lastLaunchEvals()
    # The tile-level skip is decided per (strip, tile); a pair's other order
    # is decided from the other event's strip, so the two modes may account
    # for slightly different sets of exactly-zero terms.
    assert abs(nbs - nbo) <= 0.01 * nbo and nss == nso
    assert evo == nbo and evs < 0.55 * evo
    if sym == FP64:  # the FP64 column sums are exact to FP64 rounding
        assert abs(ls - lo) <= 1e-13 * abs(lo)
        assert np.all(np.abs(gs - go) <= 1e-11 * (np.abs(go) + 1.0))
    assert abs(ls - lo) <= 1e-9 * abs(lo)


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_underflow_skip_is_bit_exact_in_fp64(flags):
    # Tile pairs whose terms all underflow are skipped; evaluating them anyway
    # must give identical bits in FP64.  In the FP32 modes a tile pair that
    # carries self-excitation terms takes its coordinate differences from hi +
    # lo parts (background-only pairs from hi parts, each event's coordinates
    # then off by up to half an FP32 ulp): evaluating the underflowed
    # self-excitation pairs gives their background terms the exact
    # coordinates.  Measured: 7e-12 on the log-likelihood, 6e-8 on the
    # strongly cancelling d/d tauT component, 7e-8 on P_i.
    loc, t = workloads.uniform(20000, seed=7)
    p = workloads.BASE_PARAMS
    with engine(loc, t, p, flags | hb.NO_TAIL_TRUNCATION) as a, \
            engine(loc, t, p, flags | hb.NO_UNDERFLOW_SKIP) as b:
        a.setSweepShape(2, 16)  # same summation order in both
        b.setSweepShape(2, 16)
        la, ga = a.getLogLikelihoodAndGradient()
        lb, gb = b.getLogLikelihoodAndGradient()
        # stats of the sweeps (the probabilities below come from the kept sums)
        _, nba, nsa = a.lastLaunchStats()
        _, nbb, nsb = b.lastLaunchStats()
        pa, pb = a.getProbsSelfExcite(), b.getProbsSelfExcite()
    if not flags & hb.COMPENSATED:
        assert la == lb and np.array_equal(ga, gb) and np.array_equal(pa, pb)
    else:
        assert abs(la - lb) <= 5e-11 * abs(lb)
        assert np.all(np.abs(ga - gb) <= 2e-7 * np.abs(gb) + 1e-12)
        assert np.max(np.abs(pa - pb)) <= 2e-7
    assert nba + nsa < nbb + nsb  # the skip did remove work
    assert nbb == 20000.0 ** 2  # without it every background term is evaluated


@pytest.mark.parametrize("flags", MODES, ids=IDS)
def test_tail_truncation_is_below_fp64_rounding(flags):
    # Background tile pairs whose terms are all below 2^-91 of an event's own
    # term are skipped by default: each event's sums move by under 2^-60.
    loc, t = workloads.uniform(20000, seed=7)
    p = workloads.BASE_PARAMS
    with engine(loc, t, p, flags) as a, engine(loc, t, p, flags | hb.NO_TAIL_TRUNCATION) as b:
        a.setSweepShape(2, 16)
        b.setSweepShape(2, 16)
        la, ga = a.getLogLikelihoodAndGradient()
        lb, gb = b.getLogLikelihoodAndGradient()
        _, nba, nsa = a.lastLaunchStats()
        _, nbb, nsb = b.lastLaunchStats()
        pa, pb = a.getProbsSelfExcite(), b.getProbsSelfExcite()
    assert abs(la - lb) <= 1e-14 * abs(lb)
    assert np.all(np.abs(ga - gb) <= 1e-12 * np.max(np.abs(gb)))
    assert np.all(np.abs(pa - pb) <= 1e-15)
    assert nsa == nsb  # the self-excitation sums keep the underflow skip only
    # times span 8760 h and b = 1/336 per hour: pairs more than 11.2 / b =
    # 3774 h apart are cut (FP32 underflow alone cuts at 13.3 / b, FP64 never)
    gap = np.abs(t[:, None] - t[None, ::50])
    assert nba < np.mean(gap < 3774 * 1.1) * 20000.0 ** 2
    assert nba < nbb


@pytest.mark.parametrize("flags", [FP64, FP32C, FP32O], ids=["fp64", "fp32c", "fp32c_ordered"])
def test_repeatable_bits(flags):
    loc, t = workloads.uniform(5000, seed=8)
    with engine(loc, t, workloads.BASE_PARAMS, flags) as e:
        r1 = e.getLogLikelihoodAndGradient()
        r2 = e.getLogLikelihoodAndGradient()
    assert r1[0] == r2[0] and np.array_equal(r1[1], r2[1])


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_sweep_shapes_agree(flags):
    # The FP64 sums and the FP32-compensated row sums (exact errors from a
    # power-of-two start) do not depend on the j-chunks, so shapes with the
    # same events per thread R agree to rounding.  In the FP32 mode another R
    # makes other strips: the tile-pair decisions (software or far-tail
    # exponential, the truncated tail) and the pairs left to the symmetric
    # sweep's FP32 column sums change, so those results differ within the
    # mode's own error against the oracle (measured R = 2 against R = 4:
    # 3.3e-11 on the log-likelihood, 3.0e-9 of the per-event scale on the
    # gradient, mostly from the far-tail tile pairs that the wider strips
    # classify as near; bars 2e-10 and half the mode's 1e-8).
    loc, t = workloads.uniform(20000, seed=13)
    p = workloads.BASE_PARAMS
    scale = oracle.oracle_eval(loc, t, p, threads=16)["grad_scale"]
    shapes = [(1, 8), (1, 64), (2, 8), (2, 64)] if flags == FP64 else \
        [(2, 8), (2, 64), (4, 8), (4, 64)]
    out = {}
    with engine(loc, t, p, flags | hb.NO_INCREMENTAL) as e:
        for shape in shapes:
            e.setSweepShape(*shape)
            ll, g = e.getLogLikelihoodAndGradient()
            out[shape] = (ll, np.asarray(g))
    ll0, g0 = out[shapes[0]]
    for shape, (ll, g) in out.items():
        same_r = shape[0] == shapes[0][0]
        if flags == FP64:
            assert abs(ll - ll0) <= 1e-13 * abs(ll0), shape
            assert np.all(np.abs(g - g0) <= 1e-12 * scale), shape
        else:
            print(shape, f"loglik {abs(ll - ll0) / abs(ll0):.2e}",
                  f"grad/event-scale {np.max(np.abs(g - g0) / scale):.2e}")
            assert abs(ll - ll0) <= (1e-13 if same_r else 2e-10) * abs(ll0), shape
            assert np.all(np.abs(g - g0) <= (1e-12 if same_r else 5e-9) * scale), shape


def test_single_row_updates_equal_full_update():
    loc, t = workloads.uniform(777, seed=9)
    p = workloads.BASE_PARAMS
    with engine(loc, t, p, FP64) as full:
        want = full.getLogLikelihoodAndGradient()
    e = hb.CudaHawkes(2, 777, FP64, 0)
    e.setTimesData(t)
    for i in range(777):  # as the reference CLI does (src/benchmark.cpp:167-171)
        e.updateLocations(i, loc[i])
    e.setParameters(p)
    got = e.getLogLikelihoodAndGradient()
    e.close()
    assert got[0] == want[0] and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_store_restore_state(flags):
    loc, t = workloads.uniform(3000, seed=10)
    p = workloads.BASE_PARAMS
    with engine(loc, t, p, flags) as e:
        first = e.getLogLikelihoodAndGradient()
        e.storeState()
        moved = loc.copy()
        moved[17] += 0.5
        e.updateLocations(17, moved[17])
        e.setParameters(p * 1.1)
        second = e.getLogLikelihoodAndGradient()
        assert second[0] != first[0]
        e.restoreState()
        third = e.getLogLikelihoodAndGradient()
        assert third[0] == first[0] and np.array_equal(third[1], first[1])
        e.acceptState()
        e.storeState()
        e.updateLocations(-1, moved)
        e.acceptState()  # keep the proposal
        fourth = e.getLogLikelihoodAndGradient()
    with engine(moved, t, p, flags) as f:
        assert f.getLogLikelihoodAndGradient()[0] == fourth[0]


def test_batch_equals_single_evaluations():
    loc, t = workloads.uniform(4000, seed=12)
    P = workloads.proposals(5, seed=13)
    with engine(loc, t, workloads.BASE_PARAMS, FP32C) as e:
        ll, g = e.batchLogLikelihoodAndGradient(P)
        for k in range(5):
            e.setParameters(P[k])
            lk, gk = e.getLogLikelihoodAndGradient()
            # one run of 5 problems vs 5 runs: only the FP64 chunk-sum order differs
            assert abs(lk - ll[k]) <= 1e-12 * abs(lk)
            assert np.all(np.abs(gk - g[k]) <= 1e-12 * (np.abs(gk) + 1.0))


def test_argument_errors_on_a_live_engine():
    with hb.CudaHawkes(2, 10, FP64, 0) as e:
        with pytest.raises(hb.HawkesError) as ei:
            e.setTimesData(np.zeros(9))
        assert ei.value.status == 2
        with pytest.raises(hb.HawkesError) as ei:
            e.updateLocations(-1, np.zeros(19))
        assert ei.value.status == 2
        with pytest.raises(hb.HawkesError) as ei:
            e.updateLocations(10, np.zeros(2))
        assert ei.value.status == 3
        with pytest.raises(hb.HawkesError) as ei:
            e.setParameters(np.ones(5))
        assert ei.value.status == 2
        bad = np.zeros(10)
        bad[3] = np.nan
        with pytest.raises(hb.HawkesError) as ei:
            e.setTimesData(bad)
        assert ei.value.status == 4
        assert e.getInternalDimension() == 2


def test_r_mirror_call_sequence():
    # The sequence R's engineInitial / getLogLikelihood / getProbsSelfExcite
    # make (R/Untitled.R:193-212, R/hph.R:10-57), through the Python mirror.
    loc, t = workloads.uniform(600, seed=14)
    eng = hb.createEngine(2, 600, gpu=1, single=False)
    with pytest.raises(hb.HawkesError, match="locations not set"):
        hb.getLogLikelihood(eng)
    eng = hb.engineInitial(loc, 600, 2, t, workloads.BASE_PARAMS)
    o = oracle.oracle_eval(loc, t, workloads.BASE_PARAMS, threads=4)
    assert abs(hb.getLogLikelihood(eng) - o["loglik"]) <= 1e-10 * abs(o["loglik"])
    assert np.max(np.abs(hb.getProbsSelfExcite(eng) - o["probs"])) <= 1e-10
    g = hb.getGradient(eng)
    assert np.all(np.abs(g - o["grad"]) <= 1e-10 * o["grad_scale"])


def test_r_time_test():
    # timeTest() (R/Untitled.R:132-175): elapsed seconds of full evaluations
    s = hb.timeTest(locationCount=2000, maxIts=3, gpu=1)
    assert 0.0 < s < 60.0
    assert 0.0 < hb.timeTest(locationCount=1000, maxIts=2, gpu=1, single=1) < 60.0
    with pytest.raises(hb.HawkesError):
        hb.timeTest(locationCount=100, r=True)
    with pytest.raises(hb.HawkesError):
        hb.timeTest(locationCount=100, gpu=0)


@pytest.mark.parametrize("flags", [FP64, FP32C], ids=["fp64", "fp32c"])
def test_tail_truncation_at_random_parameters(flags):
    # Parameters spread log-normally (sd 1) around the base, so the time
    # kernel ranges from wide (little cut) to sharp (most tile pairs cut).
    loc, t = workloads.uniform(6000, seed=11)
    rng = np.random.default_rng(12)
    for k in range(6):
        p = workloads.BASE_PARAMS * np.exp(rng.normal(0.0, 1.0, 6))
        with engine(loc, t, p, flags) as a, engine(loc, t, p, flags | hb.NO_TAIL_TRUNCATION) as b:
            a.setSweepShape(2, 16)
            b.setSweepShape(2, 16)
            la, ga = a.getLogLikelihoodAndGradient()
            lb, gb = b.getLogLikelihoodAndGradient()
            pa, pb = a.getProbsSelfExcite(), b.getProbsSelfExcite()
        assert abs(la - lb) <= 1e-14 * abs(lb), k
        assert np.all(np.abs(ga - gb) <= 1e-12 * np.max(np.abs(gb))), k
        assert np.all(np.abs(pa - pb) <= 1e-15), k
