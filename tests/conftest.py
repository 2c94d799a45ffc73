import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def load_golden(fname: str) -> dict:
    """{case: {field: array}} from a fixture written by make_golden.py."""
    data = np.load(os.path.join(GOLDEN, fname))
    cases = {}
    for key in data.files:
        name, field = key.split("__", 1)
        cases.setdefault(name, {})[field] = data[key]
    return cases


@pytest.fixture(scope="session")
def golden_synthetic():
    return load_golden("synthetic.npz")


@pytest.fixture(scope="session")
def golden_dcdata():
    return load_golden("dcdata.npz")


@pytest.fixture(scope="session")
def events_50k():
    """The accuracy workload: N = 50,000 uniform events (seed 1), base
    parameters, and the oracle's log-likelihood, gradient and scales."""
    import oracle
    from hawkes_b200 import workloads
    loc, t = workloads.uniform(50000, seed=1)
    p = workloads.BASE_PARAMS.copy()
    o = oracle.oracle_eval(loc, t, p, threads=max(1, os.cpu_count() or 1))
    return loc, t, p, o
