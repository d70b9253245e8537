"""rppt_to_decibels_gpu_static — the allocation-free to_decibels — through the C ABI.

Some callers cannot allocate device memory (a fixed device-memory budget owned by another runtime, a
real-time thread that must not block in cudaMalloc, code with no rppHandle_t).  This entry point
serves them with scratch held in a fixed array inside the library.  The test checks, on calls in a
row with different batches (the shared array keeps the previous call's contents), that its output is
bit for bit the handle-based rppt_to_decibels_gpu output (both run the same kernels with the same
arguments; a maximum left over from the previous call would show as a difference), and that a batch
above the array's limit is refused.  It needs no other test to run first.
"""
import ctypes

import numpy as np
import pytest
import torch

from rpp_b200 import audio, lib
from rpp_b200.types import RppStatus, audio_desc, spectra_desc

pytestmark = pytest.mark.gpu


def call_static(src, sdesc, dst, ddesc, dims, cutoff, mult, ref, stream):
    L = lib.load()
    return L.rppt_to_decibels_gpu_static(src.data_ptr(), ctypes.byref(sdesc), dst.data_ptr(), ctypes.byref(ddesc),
                                         dims.data_ptr(), float(cutoff), float(mult), float(ref),
                                         ctypes.c_void_p(stream))


def one_case(h, stream, n, H, W, seed, ref_mag, two_d):
    r = np.random.Generator(np.random.PCG64(seed))
    if two_d:
        x = (r.random((n, H, W)) ** 3).astype(np.float32) * float(seed)
        wh = np.stack([r.integers(1, W + 1, n), r.integers(1, H + 1, n)], 1).astype(np.int32)
        desc = spectra_desc(n, H, W)
    else:
        x = (r.normal(0, 1, (n, H * W)) ** 2).astype(np.float32)
        wh = np.stack([np.ones(n, np.int32), r.integers(1, H * W + 1, n)], 1).astype(np.int32)
        desc = audio_desc(n, H * W)
    xd = torch.from_numpy(x).cuda()
    dims = torch.from_numpy(wh).cuda()
    expect = torch.full_like(xd, -7.0)
    got = torch.full_like(xd, -7.0)
    assert audio.to_decibels(xd, desc, expect, desc, dims, -80.0, 10.0, ref_mag, h) == RppStatus.RPP_SUCCESS
    assert call_static(xd, desc, got, desc, dims, -80.0, 10.0, ref_mag, stream) == RppStatus.RPP_SUCCESS
    torch.cuda.synchronize()
    e, g = expect.cpu().numpy(), got.cpu().numpy()
    assert np.array_equal(e == -7.0, g == -7.0)       # same elements written
    assert np.array_equal(g, e)                       # same bits


def test_static_to_decibels_matches_handle_path():
    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    stream = torch.cuda.current_stream().cuda_stream
    h = lib.Handle(batch_size=1, stream=stream)
    try:
        # two calls in a row: the second one's per-sample maxima must not inherit the first one's
        one_case(h, stream, n=64, H=128, W=400, seed=3, ref_mag=0.0, two_d=True)
        one_case(h, stream, n=40, H=128, W=300, seed=1, ref_mag=0.0, two_d=True)
        one_case(h, stream, n=16, H=50, W=200, seed=5, ref_mag=0.0, two_d=False)
        one_case(h, stream, n=8, H=20, W=30, seed=6, ref_mag=2.0, two_d=True)
        # above the fixed scratch: refused, nothing launched
        n = 8193
        x = torch.zeros((n, 4), device="cuda")
        dims = torch.ones((n, 2), dtype=torch.int32, device="cuda")
        d = audio_desc(n, 4)
        assert call_static(x, d, x, d, dims, -80.0, 10.0, 0.0, stream) == \
            RppStatus.RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE
        torch.cuda.synchronize()
    finally:
        h.close()
