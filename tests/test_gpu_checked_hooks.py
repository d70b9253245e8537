"""The bounds-checked library (librppb_checked.so) catching accesses outside a call's regions.

These run only against that library (RPPB_LIBRARY=checked); tests/test_gpu_checked.py starts them in a
child process together with the parity suites.  Nothing here touches memory out of bounds: the write
test shortens the destination the library registers (the reported store is in bounds and is skipped),
and the read test describes a source shorter than its lengths while the buffer behind it is larger
(the reported loads read the library's dummy instead).  The library redirects every flagged access.
"""
import os

import numpy as np
import pytest
import torch

from rpp_b200 import audio, lib
from rpp_b200.types import RppStatus, audio_desc
from gpu_util import dev, host, canvas

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("RPPB_LIBRARY") != "checked",
                                 reason="runs against librppb_checked.so (tests/test_gpu_checked.py)")]


def preemph_case(n=3, L=1000, seed=5):
    r = np.random.Generator(np.random.PCG64(seed))
    x = r.normal(0, 0.3, (n, L)).astype(np.float32)
    lens = np.array([L, L // 2, 7], np.int32)[:n]
    coeff = np.full(n, 0.97, np.float32)
    return x, lens, coeff


def test_write_past_the_destination_is_reported(gpu, oracle):
    x, lens, coeff = preemph_case()
    n, L = x.shape
    lens[-1] = L   # the last clip fills its row, so its last store is the tensor's last element
    ref = np.full_like(x, -7.0)
    oracle.pre_emphasis(x, ref, lens, coeff, 0)
    # the destination registered one float short of its descriptor
    assert lib.load().rppb_check_shrink_next_destination(4) == 0
    out = canvas(x.shape, -7.0)
    st = audio.pre_emphasis_filter(dev(x), audio_desc(n, L), out, audio_desc(n, L), dev(lens), dev(coeff), 0, gpu)
    assert st == RppStatus.RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH, st
    msg = lib.last_error()
    assert "write of" in msg and "preemph.cu" in msg, msg
    got = host(out)
    np.testing.assert_array_equal(got.ravel()[:-4], ref.ravel()[:-4])   # the stores before the last vector landed
    assert (got.ravel()[-4:] == -7.0).all() or got.ravel()[-1] == -7.0  # the flagged store was skipped
    # the record was read and cleared: the same call without the hook succeeds
    out2 = canvas(x.shape, -7.0)
    st = audio.pre_emphasis_filter(dev(x), audio_desc(n, L), out2, audio_desc(n, L), dev(lens), dev(coeff), 0, gpu)
    assert st == RppStatus.RPP_SUCCESS, lib.last_error()
    np.testing.assert_array_equal(host(out2), ref)


def test_read_past_the_source_is_reported(gpu):
    x, lens, coeff = preemph_case()
    n, L = x.shape
    # the source described as n rows of L samples, the last clip's length 64 samples past its row; the
    # buffer holds 256 floats more than the descriptor describes
    buf = torch.zeros(n * L + 256, device="cuda")
    buf[: n * L] = torch.from_numpy(x.ravel()).cuda()
    lens[-1] = L + 64
    dst = torch.full((n, L + 128), -7.0, device="cuda")
    st = audio.pre_emphasis_filter(buf, audio_desc(n, L), dst, audio_desc(n, L + 128), dev(lens), dev(coeff), 0,
                                   gpu)
    assert st == RppStatus.RPP_ERROR_OUT_OF_BOUND_SRC_ROI, st
    msg = lib.last_error()
    assert "read of" in msg and "preemph.cu" in msg, msg
