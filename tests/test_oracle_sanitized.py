"""The oracle under AddressSanitizer and UndefinedBehaviorSanitizer: the C
restatement every parity test trusts, compiled with both sanitizers (in
pytest's temporary directory) and driven through its edge cases by
oracle/sanitize_check.c.  Any out-of-bounds access, leak of uninitialised
memory into a result, or undefined arithmetic aborts the run."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _compilers():
    seen = []
    for cc in (os.environ.get("CC"), "gcc", "cc", "/usr/bin/gcc", "clang"):
        path = shutil.which(cc) if cc else None
        if path and path not in seen:
            seen.append(path)
    return seen


def test_oracle_is_clean_under_asan_and_ubsan(tmp_path):
    exe = tmp_path / "sanitize_check"
    errors = []
    for cc in _compilers():  # the first compiler that has the sanitizer runtimes
        build = subprocess.run(
            [cc, "-O1", "-g", "-std=c11", "-fsanitize=address,undefined",
             "-fno-sanitize-recover=all", "-fno-omit-frame-pointer",
             os.path.join(ROOT, "oracle", "hawkes_oracle.c"),
             os.path.join(ROOT, "oracle", "sanitize_check.c"),
             "-o", str(exe), "-lm", "-lpthread"], capture_output=True, text=True, timeout=300)
        if build.returncode == 0:
            break
        errors.append(f"{cc}: {build.stderr.strip()[-300:]}")
    else:
        pytest.skip("no C compiler with ASan/UBSan runtimes: " + " | ".join(errors))
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    env.pop("LD_PRELOAD", None)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600, env=env)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
