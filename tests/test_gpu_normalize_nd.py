"""rppt_normalize_gpu beyond the 2-D F32 audio case: F32 3-D (every axis mask; NHWC -> NHWC,
NHWC -> NCHW, the 16-channel rows, NCHW -> NCHW writing zeros), F32 ranks 1 and 4, and U8 / F16 /
I8 at ranks 2-4, against the oracle (bit-exact to the reference host library where that library
is defined: the cases of tests/test_oracle_vs_reference.py).

Computed means match bit for bit (the same halving-tree sums, in the same order, onto the same
starting values); inverse std devs within 2e-6 (CUDA's correctly rounded rsqrt against the
reference's refined SSE/AVX estimate), so the outputs are exact where the std dev is given and
within that error otherwise: 1e-5 for F32, one unit for U8 / I8 after truncation, 2e-3 relative
for F16 after rounding."""
import numpy as np
import pytest
import torch

from rpp_b200 import audio
from rpp_b200.types import RppStatus, RpptDataType, RpptLayout, generic_desc
from gpu_util import dev, host
from test_oracle_vs_reference import NORM3D, NORMINT, NORMND, normalize_nd_case

pytestmark = pytest.mark.gpu
DT = {np.dtype(np.float32): RpptDataType.F32, np.dtype(np.float16): RpptDataType.F16,
      np.dtype(np.uint8): RpptDataType.U8, np.dtype(np.int8): RpptDataType.I8}


def run_both(gpu, oracle, src, dst_shape, mask, mean, std, compute, scale, shift, roi, sl=0, dl=0):
    exp = np.full(dst_shape, 7, src.dtype)
    m_ref, s_ref = mean.copy(), std.copy()
    oracle.normalize_nd(src, exp, mask, m_ref, s_ref, compute, scale, shift, roi, sl, dl)
    sd = generic_desc(src.shape, DT[src.dtype], sl)
    dd = generic_desc(dst_shape, DT[src.dtype], dl)
    out = dev(np.full(dst_shape, 7, src.dtype))
    m_gpu, s_gpu = dev(mean.copy()), dev(std.copy())
    st = audio.normalize(dev(src), sd, out, dd, mask, m_gpu, s_gpu, compute, scale, shift, roi, gpu)
    assert st == RppStatus.RPP_SUCCESS, st
    return host(out), exp, host(m_gpu), m_ref, host(s_gpu), s_ref


def check(got, exp, compute, dtype):
    if compute in (0, 1):
        np.testing.assert_array_equal(got, exp)
    elif dtype == np.float32:
        np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-5)
    elif dtype == np.float16:
        np.testing.assert_allclose(got.astype(np.float32), exp.astype(np.float32), rtol=2e-3, atol=2e-3)
    else:
        assert np.abs(got.astype(np.int32) - exp.astype(np.int32)).max() <= 1


def check_stats(m, m_ref, s, s_ref, compute):
    if compute & 1:
        np.testing.assert_array_equal(m, m_ref)
    if compute & 2:
        np.testing.assert_allclose(s, s_ref, rtol=2e-6, atol=0)


@pytest.mark.parametrize("case", range(len(NORM3D)))
@pytest.mark.parametrize("compute", [0, 1, 2, 3])
def test_normalize_f32_3d(gpu, oracle, case, compute):
    sl, dl, mask = NORM3D[case]
    r = np.random.Generator(np.random.PCG64(400 + case * 4 + compute))
    shp = (3, 19, 23, 3) if sl == 1 else (3, 3, 19, 23)
    src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, np.float32, begin_fits=mask in (1, 2, 4, 5))
    dshape = shp if dl == sl else (3, 3, 19, 23)
    got, exp, m, m_ref, s, s_ref = run_both(gpu, oracle, src, dshape, mask, mean, std, compute, 1.5, 0.25, roi, sl,
                                            dl)
    check(got, exp, compute, np.float32)
    check_stats(m, m_ref, s, s_ref, compute)


def test_normalize_f32_3d_16_channels(gpu, oracle):
    r = np.random.Generator(np.random.PCG64(440))
    src, roi, mean, std = normalize_nd_case(r, (2, 9, 11, 16), 3, 3, np.float32)
    got, exp, m, m_ref, s, s_ref = run_both(gpu, oracle, src, (2, 9, 11, 16), 3, mean, std, 3, 2.0, -1.0, roi, 1, 1)
    check(got, exp, 3, np.float32)
    check_stats(m, m_ref, s, s_ref, 3)


@pytest.mark.parametrize("case", range(len(NORMND)))
@pytest.mark.parametrize("compute", [0, 1, 2, 3])
def test_normalize_f32_nd(gpu, oracle, case, compute):
    shp, mask = NORMND[case]
    r = np.random.Generator(np.random.PCG64(460 + case * 4 + compute))
    src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, np.float32, begin_fits=case == 2)
    got, exp, m, m_ref, s, s_ref = run_both(gpu, oracle, src, shp, mask, mean, std, compute, 1.5, 0.25, roi)
    check(got, exp, compute, np.float32)
    check_stats(m, m_ref, s, s_ref, compute)


@pytest.mark.parametrize("case", range(len(NORMINT)))
@pytest.mark.parametrize("compute", [0, 1, 3])
@pytest.mark.parametrize("dtype", [np.uint8, np.int8, np.float16])
def test_normalize_other_types(gpu, oracle, case, compute, dtype):
    """U8, I8 (signed values, negative ones included) and F16 through the N-D branch."""
    shp, mask = NORMINT[case]
    r = np.random.Generator(np.random.PCG64(500 + case * 4 + compute))
    if dtype == np.float16:
        src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, np.float32)
        src = src.astype(np.float16)
        scale, shift = 1.5, 0.25
    else:
        src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, dtype)
        if dtype == np.int8:
            src = (src.astype(np.int16) - 64).astype(np.int8)   # -64 .. 63
            if compute == 0:
                mean = mean - 64
        scale, shift = (15.0, 0.0) if dtype == np.int8 else (20.0, 128.0)
        if compute == 0:
            scale = 15.0
        if compute == 1:
            std[:] = 0.5   # the caller's std dev array is the multiplier as given
    got, exp, m, m_ref, s, s_ref = run_both(gpu, oracle, src, shp, mask, mean, std, compute, scale, shift, roi)
    check(got, exp, compute, dtype)
    check_stats(m, m_ref, s, s_ref, compute)


def test_normalize_nd_accumulates_onto_caller_statistics(gpu, oracle):
    r = np.random.Generator(np.random.PCG64(530))
    src, roi, _, _ = normalize_nd_case(r, (3, 5, 6, 7, 40), 8, 3, np.float32)
    size = 3 * 5 * 6 * 7
    mean = r.uniform(-1, 1, size).astype(np.float32)
    std = r.uniform(0, 1, size).astype(np.float32)
    got, exp, m, m_ref, s, s_ref = run_both(gpu, oracle, src, src.shape, 8, mean, std, 3, 1.0, 0.0, roi)
    check(got, exp, 3, np.float32)
    check_stats(m, m_ref, s, s_ref, 3)


def test_normalize_nd_status_codes(gpu):
    x = torch.zeros(4096, device="cuda")
    m, s = torch.zeros(64, device="cuda"), torch.zeros(64, device="cuda")
    roi = np.array([0, 0, 0, 4, 4, 4], np.uint32)
    d3 = generic_desc((1, 4, 4, 4))
    # type mismatch, unknown type
    other = generic_desc((1, 4, 4, 4), RpptDataType.U8)
    assert audio.normalize(x, d3, x, other, 1, m, s, 3, 1.0, 0.0, roi, gpu) == RppStatus.RPP_ERROR_NOT_IMPLEMENTED
    i16 = generic_desc((1, 4, 4, 4), RpptDataType.I16)
    assert audio.normalize(x, i16, x, i16, 1, m, s, 3, 1.0, 0.0, roi, gpu) == RppStatus.RPP_ERROR_NOT_IMPLEMENTED
    # axis mask beyond the rank, or empty
    assert audio.normalize(x, d3, x, d3, 8, m, s, 3, 1.0, 0.0, roi, gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
    assert audio.normalize(x, d3, x, d3, 0, m, s, 3, 1.0, 0.0, roi, gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
    # a roi whose dense region runs past the sample
    big = np.array([0, 0, 1, 4, 4, 4], np.uint32)
    u8 = generic_desc((1, 4, 4, 4), RpptDataType.U8)
    assert audio.normalize(x, u8, x, u8, 1, m, s, 3, 1.0, 0.0, big, gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
