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


_REF_ARM = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1", "--n", "2000"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit:
    pass
maps = open("/proc/self/maps").read()
libs = sorted({l.split()[-1] for l in maps.splitlines() if l.split()[-1].endswith(".so")
               and ("/oracle/" in l or "/hawkes_b200/" in l)})
print("MAPPED " + json.dumps(libs))
"""


def test_reference_arm_line_and_libraries():
    # The reference arm prints one JSON line with the contract's keys and maps
    # the reference engine's library only, never the CUDA engine's.
    import json
    import subprocess
    import sys

    import oracle
    if not oracle.ref_available():
        pytest.skip("reference engine (oracle/_ref) not built")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _REF_ARM], cwd=root, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    line = json.loads(lines[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup",
                "ms_per_step", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
    mapped = json.loads([l for l in r.stdout.splitlines() if l.startswith("MAPPED ")][-1][7:])
    assert any(m.endswith("oracle/_ref/libhawkes_ref.so") for m in mapped), mapped
    assert not any("libhawkes_b200" in m for m in mapped), mapped
