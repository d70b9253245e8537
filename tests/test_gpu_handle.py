"""Handle entry points of include/rpp.h beyond create/destroy/stream: rppSetAllocator (a counting
allocator through the C ABI), rppEnableProfiling / rppGetKernelTime, and the roi read of
rppt_normalize_gpu after earlier work on the stream wrote it."""
import ctypes

import numpy as np
import pytest
import torch

from rpp_b200 import audio, lib, synth
from rpp_b200.types import RppStatus, audio_desc, frontend_params, generic_desc, spectra_desc
from gpu_util import dev, host, canvas

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS

ALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)
FREE = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)


def _fused(h, x, lens):
    n, L = x.shape
    F = lens // 160 + 1
    mf = int(F.max())
    out = canvas((n, 128, mf))
    assert audio.frontend(dev(x), audio_desc(n, L), out, spectra_desc(n, 128, mf), dev(lens),
                          dev(np.full(n, 0.97, np.float32)), frontend_params(), h) == OK
    return host(out)


def test_set_allocator_routes_every_device_block(gpu):
    """Every device block of a handle with a custom allocator comes from it (workspace, cached tables,
    the device error word), the results do not change, and destroying the handle returns each block."""
    L = lib.load()
    live, calls = {}, {"alloc": 0, "free": 0}

    def alloc(ctx, size):
        t = torch.empty(int(size), dtype=torch.uint8, device="cuda")
        live[t.data_ptr()] = t
        calls["alloc"] += 1
        return t.data_ptr()

    def free(ctx, p):
        calls["free"] += 1
        live.pop(p)

    a_cb, f_cb = ALLOC(alloc), FREE(free)
    x, lens = synth.gapped_clips(n=6, max_len=40000)
    expect = _fused(gpu, x, lens)
    h = lib.Handle(batch_size=6, stream=torch.cuda.current_stream().cuda_stream)
    try:
        assert L.rppSetAllocator(h.ptr, ctypes.cast(a_cb, ctypes.c_void_p), ctypes.cast(f_cb, ctypes.c_void_p),
                                 None) == 0
        got = _fused(h, x, lens)
        assert audio.device_error(h) == 0
        assert calls["alloc"] >= 3   # workspace + at least one table + the error word
        assert len(live) == calls["alloc"] - calls["free"]
        np.testing.assert_array_equal(got, expect)
        # back to cudaMalloc: the custom workspace is returned at once, tables stay until destroy
        before = calls["free"]
        assert L.rppSetAllocator(h.ptr, None, None, None) == 0
        assert calls["free"] == before + 1
        np.testing.assert_array_equal(_fused(h, x, lens), expect)
    finally:
        h.close()
    torch.cuda.synchronize()
    assert calls["alloc"] == calls["free"] and not live


def test_kernel_time_and_profiling(gpu):
    L = lib.load()
    h = lib.Handle(batch_size=4, stream=torch.cuda.current_stream().cuda_stream)
    try:
        t = ctypes.c_float(-1.0)
        x, lens = synth.gapped_clips(n=4, max_len=64000)
        _fused(h, x, lens)
        assert L.rppGetKernelTime(h.ptr, ctypes.byref(t)) == 0
        assert t.value == 0.0          # profiling off: no time recorded
        assert L.rppEnableProfiling(h.ptr, True) == 0
        _fused(h, x, lens)
        assert L.rppGetKernelTime(h.ptr, ctypes.byref(t)) == 0
        assert 0.0 < t.value < 1000.0   # the call's device time in ms
        assert L.rppEnableProfiling(h.ptr, False) == 0
        assert L.rppGetKernelTime(h.ptr, ctypes.byref(t)) == 0
        assert t.value == 0.0
        assert L.rppGetKernelTime(h.ptr, None) != 0
    finally:
        h.close()


@pytest.mark.parametrize("space", ["device", "pinned"])
def test_normalize_reads_roi_written_by_earlier_stream_work(gpu, oracle, space):
    """The roi tensor is filled by a copy queued on the handle stream just before the call (behind a
    long kernel), so reading it without waiting for the stream would see the stale values."""
    r = np.random.Generator(np.random.PCG64(5))
    n, rows, cols = 3, 16, 200
    x = r.normal(0, 1, (n, rows, cols)).astype(np.float32)
    roi = np.array([[0, 0, rows, 150], [0, 0, 9, 200], [0, 0, rows, 37]], np.uint32)
    stale = np.array([[0, 0, 1, 1]] * n, np.uint32)
    s = torch.cuda.current_stream()
    src_roi = dev(roi.view(np.int32))
    if space == "device":
        roi_t = dev(stale.view(np.int32))
    else:
        roi_t = torch.from_numpy(stale.view(np.int32).copy()).pin_memory()
    # a slow kernel ahead of the copy: the roi arrives well after the call is made
    big = torch.randn((4096, 4096), device="cuda")
    for _ in range(8):
        big = big @ big.T * 1e-4
    with torch.cuda.stream(s):
        roi_t.copy_(src_roi, non_blocking=True)
    d = generic_desc((n, rows, cols))
    out = canvas((n, rows, cols))
    mean = torch.zeros(n * rows, device="cuda")
    std = torch.zeros(n * rows, device="cuda")
    assert audio.normalize(dev(x), d, out, d, 2, mean, std, 3, 1.0, 0.0, roi_t, gpu) == OK
    got = host(out)
    exp = np.zeros_like(x)
    m_ref = np.zeros(n * rows, np.float32)
    s_ref = np.zeros(n * rows, np.float32)
    oracle.normalize_2d(x, exp, 2, m_ref, s_ref, 3, 1.0, 0.0, roi.ravel())
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-5)
