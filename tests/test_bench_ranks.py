"""The multi-process side of bench.py on CPU: two gloo ranks take the
barrier and the max-over-ranks reduction bench.py applies to its device times
(the same Ranks class, backend "gloo" instead of "nccl"), and the whole-job
rate is the units of all ranks over the slowest rank's time."""
import os
import socket

import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    ranks = bench.Ranks(world, "gloo", torch.device("cpu"), timeout_s=60)
    ranks.barrier()
    # rank-dependent device times: rank 1 is the slow one in the first entry
    got = ranks.max([1.0 + rank, 10.0 - rank, 0.25])
    ranks.barrier()
    ranks.close()
    out.put((rank, got))


def test_two_gloo_ranks_take_the_slowest_time():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    results = dict(q.get(timeout=10) for _ in procs)
    assert results[0] == results[1] == [2.0, 10.0, 0.25]


def test_single_rank_needs_no_process_group():
    torch = pytest.importorskip("torch")
    r = bench.Ranks(1, "gloo", torch.device("cpu"))
    assert r.max([3.0, 4.0]) == [3.0, 4.0]
    r.barrier()
    r.close()


def test_whole_job_rate():
    # 2 ranks x 1e10 pair-evals each over the slowest rank's 5 ms
    assert bench.whole_job_rate(2, 1e10, 5.0) == pytest.approx(4e12)
