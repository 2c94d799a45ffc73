"""The host side of the sharded evaluation (hawkes_b200.shard) on CPU: gloo
ranks run ShardedHawkes over a stand-in engine whose share of the unit sums
is a seeded array per rank.  Every rank must receive every share, in rank
order, and so hold the same sums and results; a single process needs no
process group."""
import ctypes
import os
import socket

import numpy as np
import pytest

N = 37  # events of the stand-in engine: shares of 6 N doubles


def _share(rank):
    return np.random.default_rng(100 + rank).standard_normal(6 * N)


class StandInEngine:
    """The two sharding calls of CudaHawkes on host memory (plain pointers),
    with the rank-ordered sum of hphc_set_unit_sums."""

    def __init__(self):
        self.locationCount = N
        self.device = 0
        self.parts = None
        self.kept = None

    def sweepShard(self, rank, world, ptr):
        a = np.ctypeslib.as_array((ctypes.c_double * (6 * N)).from_address(ptr))
        a[:] = _share(rank)

    def setUnitSums(self, ptr, nparts):
        a = np.ctypeslib.as_array((ctypes.c_double * (nparts * 6 * N)).from_address(ptr))
        self.parts = a.reshape(nparts, 6 * N).copy()
        s = self.parts[0].copy()
        for r in range(1, nparts):
            s += self.parts[r]
        self.kept = s

    def getLogLikelihoodAndGradient(self):
        return float(self.kept.sum()), self.kept[:6].copy()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from hawkes_b200.shard import ShardedHawkes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    eng = StandInEngine()
    sh = ShardedHawkes(eng, device="cpu")
    ll, g = sh.getLogLikelihoodAndGradient()
    shares = sh.shares()
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, (sh.rank, sh.world, eng.parts, ll, g, shares)))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_every_share_in_rank_order(world):
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=10) for _ in procs)
    expect = np.stack([_share(r) for r in range(world)])
    total = expect[0].copy()
    for r in range(1, world):
        total += expect[r]
    for r in range(world):
        rank, w, parts, ll, g, shares = res[r]
        assert (rank, w) == (r, world)
        np.testing.assert_array_equal(parts, expect)
        np.testing.assert_array_equal(shares.reshape(world, -1), expect)
        assert ll == float(total.sum())
        np.testing.assert_array_equal(g, total[:6])
    # the same bits on every rank
    assert len({res[r][3] for r in range(world)}) == 1


def test_single_process_is_a_world_of_one():
    pytest.importorskip("torch")
    from hawkes_b200.shard import ShardedHawkes
    eng = StandInEngine()
    sh = ShardedHawkes(eng, device="cpu")
    assert (sh.rank, sh.world) == (0, 1)
    ll, g = sh.getLogLikelihoodAndGradient()
    np.testing.assert_array_equal(eng.parts[0], _share(0))
    assert ll == float(_share(0).sum())
