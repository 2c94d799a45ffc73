"""The reference's own command-line benchmark (src/benchmark.cpp, compiled
unmodified into oracle/_ref/benchmark_ref with its factory's GPU slot filled
by this engine through hawkes_b200/integration/factory_shim.cpp) run twice on
the same seeded data: on its CPU path (the reference NewHawkes engine) and on
its --gpu path, which hph::factory sends to the CUDA engine.  The printed
averages must agree to the precision the CLI prints: AvgProbSE to its six
significant digits, and AvgLogLik exactly, up to one unit (the CLI
accumulates the log-likelihoods into an int, src/benchmark.cpp:174, so a value
within rounding of an integer boundary may truncate differently)."""
import os
import re
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu


def run_cli(args, cwd):
    out = subprocess.run([oracle.REF_BENCHMARK] + args, cwd=cwd, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    ll = float(re.search(r"AvgLogLik = (\S+)", out.stdout).group(1))
    pse = float(re.search(r"AvgProbSE = (\S+)", out.stdout).group(1))
    return ll, pse, out.stdout + out.stderr


@pytest.mark.skipif(not os.path.exists(oracle.REF_BENCHMARK),
                    reason="reference CLI not built (needs the reference sources at build time)")
@pytest.mark.parametrize("dim,n", [(2, 3000), (3, 1500)])
def test_reference_cli_gpu_slot_matches_its_cpu_engine(tmp_path, dim, n):
    args = ["--locations", str(n), "--iterations", "2", "--dimension", str(dim)]
    cpu_ll, cpu_pse, cpu_out = run_cli(args, tmp_path)
    gpu_ll, gpu_pse, gpu_out = run_cli(["--gpu", "1"] + args, tmp_path)
    assert "Running on CPU" in cpu_out and "Running on GPU" in gpu_out
    assert "CUDA (sm_100a), DOUBLE" in gpu_out  # the engine the factory built
    assert abs(gpu_ll - cpu_ll) <= 1.0
    assert abs(gpu_pse - cpu_pse) <= 1.5e-6 * abs(cpu_pse)
