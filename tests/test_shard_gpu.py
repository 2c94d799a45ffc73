"""Sharded evaluation on the CUDA engine (hphc_sweep_shard +
hphc_set_unit_sums).  One GPU stands in for `world` of them: every rank's
share is swept in turn on the same device into its slot of one buffer, as the
all-gather would leave it, and the rank-ordered sum must give the unsharded
log-likelihood, gradient and P_i (to rounding of the regrouped FP64 sums);
the ranks' work must partition the unsharded sweep's pair terms exactly.  The
ShardedHawkes host class then runs over a one-rank NCCL process group."""
import os
import subprocess
import sys

import numpy as np
import pytest

import hawkes_b200 as hb
from hawkes_b200 import workloads

pytestmark = pytest.mark.gpu

MODES = [hb.CUDA, hb.CUDA | hb.ORDERED, hb.CUDA | hb.COMPENSATED,
         hb.CUDA | hb.COMPENSATED | hb.ORDERED]
IDS = ["fp64", "fp64_ordered", "fp32c", "fp32c_ordered"]


def _engine(loc, t, p, flags):
    e = hb.CudaHawkes(2, len(t), flags, 0)
    e.setTimesData(t)
    e.updateLocations(-1, loc)
    e.setParameters(p)
    return e


@pytest.mark.parametrize("flags", MODES, ids=IDS)
@pytest.mark.parametrize("world", [2, 3, 8])
def test_shares_add_up_to_the_unsharded_sweep(flags, world):
    import torch
    loc, t = workloads.uniform(20000, seed=9)
    p = workloads.BASE_PARAMS
    # one strip height for both engines: the tile-level causality test, and
    # so the count of self-excitation terms evaluated, depends on it
    shape = (2, 16) if not flags & hb.COMPENSATED else (4, 16)
    with _engine(loc, t, p, flags) as ref:
        ref.setSweepShape(*shape)
        ll0, g0 = ref.getLogLikelihoodAndGradient()
        _, nb0, ns0 = ref.lastLaunchStats()  # of the sweep (P_i come from the kept sums)
        pr0 = ref.getProbsSelfExcite()
    n = 6 * len(t)
    buf = torch.empty(world * n, dtype=torch.float64, device="cuda:0")
    with _engine(loc, t, p, flags) as e:
        e.setSweepShape(*shape)
        nb = ns = 0.0
        for r in range(world):
            e.sweepShard(r, world, buf[r * n:].data_ptr())
            _, b, s = e.lastLaunchStats()
            assert b > 0.0
            nb, ns = nb + b, ns + s
        assert (nb, ns) == (nb0, ns0)  # the ranks' work partitions the sweep
        e.setUnitSums(buf.data_ptr(), world)
        ll, g = e.getLogLikelihoodAndGradient()
        assert e.lastEvaluationPath == hb.PATH_KEPT_SUMS
        pr = e.getProbsSelfExcite()
    if not flags & hb.COMPENSATED:
        assert abs(ll - ll0) <= 1e-12 * abs(ll0)
        np.testing.assert_allclose(g, g0, rtol=1e-10, atol=1e-12 * np.abs(g0).max())
        np.testing.assert_allclose(pr, pr0, rtol=1e-11, atol=1e-14)
    else:
        # a rank's strips are cut into other j-chunks than in the unsharded
        # sweep; the compensated FP32 sums restart per chunk with exact
        # errors (measured: 2e-16 on the log-likelihood, 1e-12 on the gradient,
        # 6e-13 absolute on P_i)
        assert abs(ll - ll0) <= 1e-13 * abs(ll0)
        np.testing.assert_allclose(g, g0, rtol=1e-10, atol=1e-12 * np.abs(g0).max())
        np.testing.assert_allclose(pr, pr0, rtol=1e-10, atol=2e-12)


def test_shard_arguments_are_checked():
    import torch
    loc, t = workloads.uniform(3000, seed=10)
    p = workloads.BASE_PARAMS
    n = 6 * len(t)
    buf = torch.zeros(2 * n, dtype=torch.float64, device="cuda:0")
    host = np.zeros(2 * n)
    with _engine(loc, t, p, hb.CUDA | hb.COMPENSATED) as e:
        for bad in [(2, 2), (-1, 2), (0, 0)]:
            with pytest.raises(hb.HawkesError):
                e.sweepShard(*bad, buf.data_ptr())
        with pytest.raises(hb.HawkesError):  # host memory is not a device buffer
            e.sweepShard(0, 2, host.ctypes.data)
        with pytest.raises(hb.HawkesError):  # no share swept yet
            e.setUnitSums(buf.data_ptr(), 2)
        e.sweepShard(0, 2, buf.data_ptr())
        e.setParameters(p * 1.01)
        with pytest.raises(hb.HawkesError):  # parameters changed since the sweep
            e.setUnitSums(buf.data_ptr(), 2)
        e.setParameters(p)
        e.sweepShard(1, 2, buf[n:].data_ptr())
        e.updateLocations(-1, loc + 0.5)
        with pytest.raises(hb.HawkesError):  # events changed since the sweep
            e.setUnitSums(buf.data_ptr(), 2)
        e.updateLocations(-1, loc)
        # still usable after the refusals
        ll, _ = e.getLogLikelihoodAndGradient()
        assert np.isfinite(ll)
    with _engine(loc, t, p, hb.CUDA | hb.NO_INCREMENTAL) as e:
        e.sweepShard(0, 1, buf.data_ptr())
        with pytest.raises(hb.HawkesError):  # this engine keeps no sums
            e.setUnitSums(buf.data_ptr(), 1)


_NCCL_SCRIPT = r"""
import datetime, os, sys
sys.path.insert(0, os.environ["REPO"])
import numpy as np, torch, torch.distributed as dist
import hawkes_b200 as hb
from hawkes_b200 import workloads
from hawkes_b200.shard import ShardedHawkes
torch.cuda.set_device(0)
dist.init_process_group("nccl", init_method="tcp://127.0.0.1:" + os.environ["PORT"], rank=0,
                        world_size=1, timeout=datetime.timedelta(seconds=60),
                        device_id=torch.device("cuda", 0))
loc, t = workloads.uniform(8000, seed=11)
p = workloads.BASE_PARAMS
out = []
for flags in (hb.CUDA, hb.CUDA | hb.COMPENSATED):
    with hb.CudaHawkes(2, len(t), flags, 0) as a, hb.CudaHawkes(2, len(t), flags, 0) as b:
        for e in (a, b):
            e.setTimesData(t); e.updateLocations(-1, loc); e.setParameters(p)
        ll0, g0 = a.getLogLikelihoodAndGradient()
        sh = ShardedHawkes(b)
        ll, g = sh.getLogLikelihoodAndGradient()
        pr = sh.getProbsSelfExcite()
        assert abs(ll - ll0) <= 1e-12 * abs(ll0), (ll, ll0)
        assert np.allclose(g, g0, rtol=1e-10, atol=0), (g, g0)
        assert np.allclose(pr, a.getProbsSelfExcite(), rtol=1e-11, atol=1e-14)
dist.destroy_process_group()
print("sharded ok")
"""


def test_sharded_hawkes_over_a_one_rank_nccl_group():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, REPO=root, PORT=str(port))
    r = subprocess.run([sys.executable, "-c", _NCCL_SCRIPT], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and "sharded ok" in r.stdout, r.stdout + r.stderr
