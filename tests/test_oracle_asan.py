"""The oracle (oracle/rppb_oracle.c) under AddressSanitizer and UndefinedBehaviorSanitizer: a C driver
(tests/asan/oracle_asan_driver.c) runs every restated op on edge-case batches (lengths 0, 1, 2, shorter
than the window, longer than the NSR reset interval; centred and not; NFT and NTF; every border,
normalisation axis and padding mode) in buffers of exactly the descriptors' sizes.  The parity tests
trust the oracle's outputs, so it must neither read nor write outside the caller's tensors."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "asan", "_build")


def test_oracle_memory_safe_under_asan():
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc absent")
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "oracle_asan_driver")
    cmd = [cc, "-std=gnu11", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=all", "-ffp-contract=off", os.path.join(ROOT, "oracle", "rppb_oracle.c"),
           os.path.join(ROOT, "tests", "asan", "oracle_asan_driver.c"), "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "sanitize" in r.stderr and ("cannot find" in r.stderr or "not supported" in r.stderr):
        pytest.skip("sanitizer runtime unavailable: " + r.stderr.strip().splitlines()[-1])
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=env)
    assert run.returncode == 0 and "oracle asan ok" in run.stdout, run.stdout + run.stderr
