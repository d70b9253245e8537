"""The parity suites against the bounds-checked library (librppb_checked.so).

In that library every global load and store of the kernels is checked against the device regions of
the call that launched it, and a call with an access outside them returns an error status
(include/rppb_frontend.h, rpp_b200/csrc/check.cu).  Running the parity suites against it in a child
process (RPPB_LIBRARY=checked) shows that every kernel stays inside the caller's tensors as their
descriptors describe them, the per-sample tensors, the workspace and the handle's tables, on every
case those suites cover, with the same outputs; tests/test_gpu_checked_fuzz.py adds seeded random valid
calls of every entry point.  tests/test_gpu_checked_hooks.py, run in the same child process, shows that
the checks do fire.  Outside this check: the tensor-core kernels' TMA loads
(their reach is bounded by the tensor maps, which the driver validates), and the serving thread's
copy kernels, which run outside any call.
"""
import os
import subprocess
import sys

import pytest

from rpp_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITES = ["tests/test_gpu_ops.py", "tests/test_gpu_normalize_nd.py", "tests/test_gpu_frontend.py",
          "tests/test_gpu_frontend_tc.py", "tests/test_gpu_tc.py", "tests/test_gpu_parity_reference.py",
          "tests/test_gpu_edges.py", "tests/test_gpu_parity_fuzz.py", "tests/test_gpu_checked_hooks.py",
          "tests/test_gpu_checked_fuzz.py"]


@pytest.mark.gpu
def test_parity_suites_under_the_checked_library():
    assert os.path.isfile(lib.CHECKED_LIB_PATH), "build it with `python -m rpp_b200.build --checked`"
    env = dict(os.environ, RPPB_LIBRARY="checked")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"] + SUITES,
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    tail = r.stdout[-4000:] + r.stderr[-2000:]
    assert r.returncode == 0, tail
    assert " passed" in r.stdout and "skipped" not in r.stdout.splitlines()[-1], tail
