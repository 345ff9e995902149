"""The oracle under AddressSanitizer and UndefinedBehaviorSanitizer (host only).

`make -C oracle sanitize` builds oracle/sanitize_main.cpp with tebd_oracle.cpp, undefined
behaviour fatal, and the driver runs every extern "C" entry point of the oracle on small
inputs.  Any out-of-bounds access, use after free, leak or undefined behaviour makes the run
exit non-zero.  Skipped only when no compiler with the sanitizer runtimes is present.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_is_clean_under_asan_and_ubsan():
    mk = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "sanitize"], capture_output=True, text=True)
    if mk.returncode != 0:
        if "asan" in mk.stderr or "sanitize" in mk.stderr:
            pytest.skip(f"no sanitizer runtime: {mk.stderr.strip().splitlines()[-1]}")
        raise AssertionError(mk.stderr)
    exe = os.path.join(ROOT, "oracle", "build", "oracle_sanitize")
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=env)
    assert run.returncode == 0, run.stderr[-4000:]
    assert "sanitize ok" in run.stdout
    assert "runtime error" not in run.stderr
