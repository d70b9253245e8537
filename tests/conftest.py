import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built librppb.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle, build_oracle
    build_oracle()
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference's own host library; built here when the sources are present."""
    from oracle import Reference, build_reference, reference_lib_path
    if not os.path.isfile(reference_lib_path()):
        build_reference()
    if not os.path.isfile(reference_lib_path()):
        pytest.skip("reference host library not built (reference sources absent)")
    return Reference(threads=min(8, os.cpu_count() or 1))


@pytest.fixture(scope="session")
def reference_or_none():
    """The reference's host library when it is built (or buildable), else None."""
    from oracle import Reference, build_reference, reference_lib_path
    if not os.path.isfile(reference_lib_path()):
        try:
            build_reference()
        except Exception:
            return None
    if not os.path.isfile(reference_lib_path()):
        return None
    return Reference(threads=min(8, os.cpu_count() or 1))


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_audio_qa.npz"))


@pytest.fixture(scope="session")
def gpu():
    """CUDA device + handle on the current torch stream; fails (not skips) without the library."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu-marked test needs a CUDA device")
    from rpp_b200 import lib
    lib.load()
    h = lib.Handle(batch_size=1, stream=torch.cuda.current_stream().cuda_stream)
    yield h
    torch.cuda.synchronize()
    h.close()
