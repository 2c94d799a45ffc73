"""The persistent autotune cache (HPHC_TUNE_CACHE, a JSON-lines file): a
process that tunes a new shape appends a line for this device, and a later
process reads it instead of timing the candidates.  The second process is
given an edited line whose shape the tuner never tries (1 item per SM), so
finding that shape in use shows the cache was read."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.environ["REPO"])
import hawkes_b200 as hb
from hawkes_b200 import workloads
loc, t = workloads.uniform(20000, seed=23)
with hb.CudaHawkes(2, len(t), hb.CUDA | hb.COMPENSATED, 0) as e:
    e.setTimesData(t); e.updateLocations(-1, loc); e.setParameters(workloads.BASE_PARAMS)
    ll, _ = e.getLogLikelihoodAndGradient()
    print(json.dumps({"shape": e.sweepShape(), "ll": ll}))
"""


def _run(cache):
    env = dict(os.environ, REPO=ROOT, HPHC_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", _SCRIPT], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_tuned_shape_is_written_and_read_back(tmp_path):
    import torch
    cache = tmp_path / "tune.jsonl"
    first = _run(cache)
    lines = [json.loads(x) for x in cache.read_text().splitlines()]
    assert len(lines) == 1
    line = lines[0]
    assert line["v"] == 1 and line["device"] == torch.cuda.get_device_name(0)
    assert line["sms"] == torch.cuda.get_device_properties(0).multi_processor_count
    assert [line["R"], line["items"]] == first["shape"] and line["D"] == 2
    # a process with the cached shape does not tune again (no new line)
    second = _run(cache)
    assert second["shape"] == first["shape"] and second["ll"] == first["ll"]
    assert len(cache.read_text().splitlines()) == 1
    # an edited shape the tuner never tries is taken from the file
    edited = dict(line, items=1)
    other = dict(line, device="another device", items=8)
    cache.write_text("not json\n" + json.dumps(other) + "\n" + json.dumps(edited) + "\n")
    third = _run(cache)
    assert third["shape"] == [line["R"], 1]
    # other j-chunk bounds: the FP32-compensated sums restart per chunk with
    # exact errors, so the log-likelihood moves by ~1e-15 relative
    assert abs(third["ll"] - first["ll"]) <= 1e-13 * abs(first["ll"])
