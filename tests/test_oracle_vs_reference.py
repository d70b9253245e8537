"""Cross-checks the C restatement against the reference's own host library on seeded synthetic
batches, op by op, across the parameter space the reference supports (border types, channel
counts, rate pairs, mel formulas, ROI shapes, reset intervals).  The float restatements must
agree bit for bit; this is what lets the GPU tests use the restatement as the oracle on a box
where the reference sources are absent.
"""
import numpy as np
import pytest

from rpp_b200 import synth
from rpp_b200.types import audio_desc, spectra_desc, RpptImagePatch, RpptLayout


def rng(k):
    return np.random.Generator(np.random.PCG64(1000 + k))


def small_batch(n=6, lo=1, hi=9000, seed=0):
    r = rng(seed)
    lens = r.integers(lo, hi, n).astype(np.int32)
    lens[0] = hi   # one full-stride sample
    x, lens = synth.mono_batch(n, lens, r, gaps=True)
    return x, lens


@pytest.mark.parametrize("border", [0, 1, 2])
def test_pre_emphasis(oracle, reference, border):
    x, lens = small_batch(seed=border)
    d = audio_desc(len(lens), x.shape[1])
    coeff = rng(7).uniform(0.5, 0.99, len(lens)).astype(np.float32)
    a = np.zeros_like(x)
    b = np.zeros_like(x)
    oracle.pre_emphasis(x, a, lens, coeff, border)
    assert reference.pre_emphasis_filter(x, d, b, d, lens, coeff, border) == 0
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("channels", [1, 2, 3, 5, 8, 11])
@pytest.mark.parametrize("normalize", [False, True])
def test_down_mixing(oracle, reference, channels, normalize):
    r = rng(channels)
    n, L = 4, 3001
    lens = r.integers(1, L + 1, n).astype(np.int32)
    x = r.normal(0, 0.3, (n, L * channels)).astype(np.float32)
    dims = np.stack([lens, np.full(n, channels, np.int32)], 1).ravel().astype(np.int32)
    sd = audio_desc(n, L, channels=channels, num_dims=3)
    dd = audio_desc(n, L)
    a = np.zeros((n, L), np.float32)
    b = np.zeros((n, L), np.float32)
    oracle.down_mixing(x, a, dims, normalize)
    assert reference.down_mixing(x, sd, b, dd, dims, normalize) == 0
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("rates,channels", [((16000, 18400), 1), ((48000, 16000), 1), ((44100, 16000), 1),
                                            ((22050, 16000), 2), ((16000, 16000), 1), ((8000, 44100), 1)])
def test_resample(oracle, reference, rates, channels):
    r = rng(3)
    n, L = 3, 4000
    lens = np.array([L, 1777, 1], np.int32)
    x = r.normal(0, 0.3, (n, L * channels)).astype(np.float32)
    lut, scale, center, lobes = oracle.windowed_sinc(16 * 64 + 1, 16)
    ir = np.full(n, rates[0], np.float32)
    orr = np.full(n, rates[1], np.float32)
    out_len = int(np.ceil(L * rates[1] / rates[0])) + 8
    dims = np.stack([lens, np.full(n, channels, np.int32)], 1).ravel().astype(np.int32)
    sd = audio_desc(n, L, channels=channels)
    dd = audio_desc(n, out_len, channels=channels)
    a = np.zeros((n, out_len * channels), np.float32)
    b = np.zeros((n, out_len * channels), np.float32)
    oracle.resample(x, a, ir, orr, dims, lut, scale, center, lobes)
    assert reference.resample(x, sd, b, dd, ir, orr, dims, lut, scale, center, lobes, 16 * 64 + 1) == 0
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("htk,normalize,nfft,nmel,fmin,fmax", [
    (0, 1, 512, 128, 0.0, 8000.0), (1, 1, 512, 80, 0.0, 0.0), (0, 0, 1024, 64, 60.0, 7600.0),
    (1, 0, 256, 40, 20.0, 4000.0)])
def test_mel_filter_bank(oracle, reference, htk, normalize, nfft, nmel, fmin, fmax):
    r = rng(nfft + nmel)
    n, bins, T = 3, nfft // 2 + 1, 97
    frames = np.array([T, 50, 1], np.int32)
    spec = (r.random((n, bins, T)) ** 4).astype(np.float32)
    dims = np.stack([np.full(n, bins, np.int32), frames], 1).ravel().astype(np.int32)
    sd = spectra_desc(n, bins, T)
    dd = spectra_desc(n, nmel, T)
    a = np.full((n, nmel, T), -7.0, np.float32)
    b = np.full((n, nmel, T), -7.0, np.float32)
    oracle.mel_filter_bank(spec, a, dims, fmax, fmin, htk, nmel, 16000, normalize)
    assert reference.mel_filter_bank(spec, sd, b, dd, dims, fmax, fmin, htk, nmel, 16000, normalize) == 0
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("two_d,ref", [(False, 0.0), (True, 0.0), (True, 2.5), (False, 1.0)])
def test_to_decibels(oracle, reference, two_d, ref):
    r = rng(11)
    n, H, Wd = 3, 40, 77
    if two_d:
        x = (r.random((n, H, Wd)) ** 3).astype(np.float32)
        wh = [(Wd, H), (30, 12), (1, 1)]
        sd = spectra_desc(n, H, Wd)
    else:
        x = r.normal(0, 1, (n, H * Wd)).astype(np.float32) ** 2
        wh = [(1, H * Wd), (1, 100), (1, 1)]
        sd = audio_desc(n, H * Wd)
    dims = np.array(wh, np.uint32)
    patches = (RpptImagePatch * n)()
    for i, (w, h) in enumerate(wh):
        patches[i].width, patches[i].height = w, h
    a = np.zeros_like(x)
    b = np.zeros_like(x)
    oracle.to_decibels(x, a, dims, -80.0, 10.0, ref)
    assert reference.to_decibels(x, sd, b, sd, patches, -80.0, 10.0, ref) == 0
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("reset,window,ref,cut", [(8192, 2048, 0.0, -60.0), (-1, 2048, 0.0, -60.0),
                                                  (1000, 333, 0.0, -40.0), (8192, 2048, 0.05, -20.0)])
def test_nsr(oracle, reference, reset, window, ref, cut):
    x, lens = small_batch(n=5, lo=1, hi=20000, seed=5)
    d = audio_desc(len(lens), x.shape[1])
    b1, l1 = oracle.nsr(x, lens, cut, window, ref, reset)
    b2 = np.zeros(len(lens), np.int32)
    l2 = np.zeros(len(lens), np.int32)
    assert reference.nsr(x, d, lens, b2, l2, cut, window, ref, reset) == 0
    np.testing.assert_array_equal(b1, b2)
    np.testing.assert_array_equal(l1, l2)


@pytest.mark.parametrize("nfft,W,hop,center,reflect,layout", [
    (512, 400, 160, True, True, RpptLayout.NFT), (512, 320, 160, True, False, RpptLayout.NTF),
    (256, 256, 100, False, True, RpptLayout.NFT), (400, 400, 160, True, True, RpptLayout.NFT)])
def test_spectrogram_f64_vs_reference(oracle, reference, nfft, W, hop, center, reflect, layout):
    x, lens = small_batch(n=4, lo=1, hi=6000, seed=9)
    n = len(lens)
    F = [oracle.num_windows(l, W, hop, center) for l in lens]
    mf = max(F)
    bins = nfft // 2 + 1
    nft = layout == RpptLayout.NFT
    dd = spectra_desc(n, bins, mf, layout) if nft else spectra_desc(n, mf, bins, layout)
    out = np.zeros((n, bins, mf) if nft else (n, mf, bins), np.float32)
    assert reference.spectrogram(x, audio_desc(n, x.shape[1]), out, dd, lens, center, reflect, None, nfft, 2, W,
                                 hop) == 0
    o = oracle.spectrogram_f64(x, lens, center, reflect, None, nfft, 2, W, hop, nft, max_frames=mf)
    for i in range(n):
        if F[i] <= 0 or lens[i] < 2:
            continue
        g = out[i, :, :F[i]] if nft else out[i, :F[i], :].T
        e = o[i, :, :F[i]] if nft else o[i, :F[i], :].T
        scale = np.maximum(g.max(axis=0, keepdims=True), 1e-30)
        assert (np.abs(e - g) / scale).max() < 2e-6


@pytest.mark.parametrize("num_dims", [1, 2])
@pytest.mark.parametrize("dtype", [np.float32, np.uint8])
@pytest.mark.parametrize("pad", [False, True])
def test_slice(oracle, reference, num_dims, dtype, pad):
    """Boxes inside and overlapping the roi lengths (padding needed), both element types."""
    r = rng(50 + num_dims)
    n = 7
    shape_t = (n, 3000) if num_dims == 1 else (n, 40, 64)
    if dtype == np.uint8:
        src = r.integers(0, 255, shape_t).astype(np.uint8)
    else:
        src = r.standard_normal(shape_t).astype(np.float32)
    ext = np.array(shape_t[1:])
    length = np.stack([r.integers(e // 2, e + 1, n) for e in ext], 1).astype(np.int32)
    # anchors stay below the roi lengths: beyond them the reference copies a negative length
    # converted to unsigned (slice.cpp:203-204), i.e. crashes
    anchor = np.stack([r.integers(0, e // 2, n) for e in ext], 1).astype(np.int32)
    shape = np.stack([r.integers(1, e, n) for e in ext], 1).astype(np.int32)
    anchor[0] = 0
    shape[1] = ext - anchor[1]        # reaches past a short roi: padding
    roi = np.concatenate([np.zeros_like(length), length], 1).astype(np.uint32)
    fill = 7 if dtype == np.uint8 else -3.5
    a = np.full_like(src, 9 if dtype == np.uint8 else 9.25)
    b = a.copy()
    oracle.slice(src, a, anchor.ravel(), shape.ravel(), roi.ravel(), fill, pad, num_dims)
    reference.slice(src, b, anchor.ravel(), shape.ravel(), roi.ravel(), fill, pad, num_dims)
    np.testing.assert_array_equal(a, b)


SLICE_ND = [(RpptLayout.NCHW, (5, 3, 37, 53)), (RpptLayout.NCHW, (5, 1, 29, 64)), (RpptLayout.NHWC, (5, 31, 47, 3)),
            (RpptLayout.NHWC, (5, 17, 40, 4)), (RpptLayout.NCDHW, (4, 3, 9, 21, 33)),
            (RpptLayout.NCDHW, (4, 1, 7, 16, 24)), (RpptLayout.NDHWC, (4, 8, 19, 27, 3)),
            (RpptLayout.NDHWC, (4, 6, 11, 13, 2))]


def slice_nd_case(r, shp, layout):
    """Random per-sample roi lengths, anchors below them (the reference turns a negative extent
    into a huge unsigned size) and shapes, one sample reaching past its lengths (padding)."""
    n, ext = shp[0], np.array(shp[1:])
    length = np.stack([r.integers(max(e // 2, 1), e + 1, n) for e in ext], 1).astype(np.int32)
    anchor = np.stack([r.integers(0, max(e // 2, 1), n) for e in ext], 1).astype(np.int32)
    shape = np.stack([r.integers(1, e + 1, n) for e in ext], 1).astype(np.int32)
    shape[1] = ext - anchor[1]
    roi = np.concatenate([np.zeros_like(length), length], 1).astype(np.uint32)
    return anchor.ravel(), shape.ravel(), roi.ravel()


@pytest.mark.parametrize("case", range(len(SLICE_ND)))
@pytest.mark.parametrize("dtype", [np.float32, np.uint8])
@pytest.mark.parametrize("pad", [False, True])
def test_slice_nd(oracle, reference, case, dtype, pad):
    """3-D and 4-D boxes in the four layouts the reference slices (NCHW / NHWC, NCDHW / NDHWC)."""
    layout, shp = SLICE_ND[case]
    r = rng(70 + case)
    src = (r.integers(0, 255, shp).astype(np.uint8) if dtype == np.uint8
           else r.standard_normal(shp).astype(np.float32))
    anchor, shape, roi = slice_nd_case(r, shp, layout)
    fill = 7 if dtype == np.uint8 else -3.5
    a = np.full_like(src, 9 if dtype == np.uint8 else 9.25)
    b = a.copy()
    oracle.slice_nd(src, a, anchor, shape, roi, fill, pad, int(layout))
    reference.slice_nd(src, b, anchor, shape, roi, fill, pad, int(layout))
    np.testing.assert_array_equal(a, b)
    assert (a != (9 if dtype == np.uint8 else 9.25)).any()


@pytest.mark.parametrize("axis_mask", [1, 2, 3])
@pytest.mark.parametrize("compute", [0, 1, 2, 3])
def test_normalize_2d(oracle, reference, axis_mask, compute):
    """2-D F32 normalize (the audio branch of normalize.cpp): rois smaller than the tensor, long
    reductions (the recursive halving sums), internal and external mean / std dev, bit for bit
    including the in-out mean and std-dev arrays (same CPU, same rsqrt instruction)."""
    r = rng(60 + axis_mask * 4 + compute)
    n, R, C = 5, 40, 700
    src = (r.standard_normal((n, R, C)) * 3 + 1).astype(np.float32)
    src[2, 3, :] = 0.5      # a constant row: zero variance
    roi = np.zeros((n, 4), np.uint32)
    roi[:, 2] = r.integers(20, R + 1, n)
    roi[:, 3] = r.integers(300, C + 1, n)
    roi[0, 2:] = (R, C)
    size = max(int(np.prod([1 if axis_mask & (1 << i) else roi[b, 2 + i] for i in range(2)])) for b in range(n))
    per = n * size
    mean = (r.standard_normal(per) * 0.1).astype(np.float32)
    std = r.uniform(0.5, 2.0, per).astype(np.float32)
    std[1] = 0.0
    outs = []
    for impl in (oracle, reference):
        m, s_ = mean.copy(), std.copy()
        dst = np.full((n, R, C), 7.0, np.float32)
        impl.normalize_2d(src, dst, axis_mask, m, s_, compute, 1.5, 0.25, roi.ravel())
        outs.append((dst, m, s_))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    np.testing.assert_array_equal(outs[0][2], outs[1][2])


def normalize_nd_case(r, shp, axis_mask, compute, dtype, begin_fits=False):
    """Source, roi and in-out statistics for a normalize case; integer sources keep their results
    inside the type's range (where the host path's float-to-integer conversion is defined)."""
    n, ext = shp[0], np.array(shp[1:])
    T = len(ext)
    if dtype == np.float32:
        src = (r.standard_normal(shp) * 3 + 1).astype(np.float32)
    elif dtype == np.uint8:
        src = r.integers(0, 256, shp).astype(np.uint8)
    else:
        src = r.integers(0, 128, shp).astype(np.int8)   # non-negative: the host path reads int8 as unsigned
    roi = np.zeros((n, 2 * T), np.uint32)
    roi[:, T:] = ext
    if begin_fits:
        # a dense region of the roi lengths from the begin offset, inside the sample
        roi[1:, T:] = np.maximum(ext // 2, 1)
        roi[1:, 0] = 1
    size = max(int(np.prod([1 if axis_mask & (1 << i) else roi[b, T + i] for i in range(T)])) for b in range(n))
    per = n * size
    if compute == 0:
        centre = {np.float32: 0.0, np.uint8: 128.0, np.int8: 64.0}[dtype]
        mean = (r.uniform(-0.5, 0.5, per) + centre).astype(np.float32)
        std = r.uniform(20.0, 40.0, per).astype(np.float32)
    else:
        mean = np.zeros(per, np.float32)
        std = np.zeros(per, np.float32) if compute & 2 else np.full(per, 0.25, np.float32)
        if compute == 2:
            mean[:] = 60.0 if dtype != np.float32 else 0.5
    return src, roi.ravel(), mean, std


def run_normalize_nd(impls, src, dst_shape, dst_dtype, axis_mask, mean, std, compute, scale, shift, roi, sl, dl):
    outs = []
    for impl in impls:
        m, s_ = mean.copy(), std.copy()
        dst = np.full(dst_shape, 7, dst_dtype)
        impl.normalize_nd(src, dst, axis_mask, m, s_, compute, scale, shift, roi, sl, dl)
        outs.append((dst, m, s_))
    return outs


NORM3D = [(1, 1, m) for m in range(1, 8)] + [(1, 0, 3), (0, 0, 3)]


@pytest.mark.parametrize("case", range(len(NORM3D)))
@pytest.mark.parametrize("compute", [0, 1, 2, 3])
def test_normalize_f32_3d(oracle, reference, case, compute):
    """The F32 3-D branch: NHWC -> NHWC for every axis mask, NHWC -> NCHW (mask 3) and NCHW ->
    NCHW (statistics only: the reference writes zeros), bit for bit with the in-out arrays."""
    sl, dl, mask = NORM3D[case]
    r = rng(200 + case * 4 + compute)
    shp = (3, 19, 23, 3) if sl == 1 else (3, 3, 19, 23)
    src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, np.float32, begin_fits=mask in (1, 2, 4, 5))
    dshape = shp if dl == sl else (3, 3, 19, 23)
    a, b = run_normalize_nd((oracle, reference), src, dshape, np.float32, mask, mean, std, compute, 1.5, 0.25, roi,
                            sl, dl)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_normalize_f32_3d_16_channels(oracle, reference):
    """NHWC with 16 channels and mask 3 (the reference's vectorized row path)."""
    r = rng(240)
    src, roi, mean, std = normalize_nd_case(r, (2, 9, 11, 16), 3, 3, np.float32)
    a, b = run_normalize_nd((oracle, reference), src, (2, 9, 11, 16), np.float32, 3, mean, std, 3, 2.0, -1.0, roi,
                            1, 1)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


NORMND = [((4, 700), 1), ((3, 5, 6, 7, 40), 1), ((3, 5, 6, 7, 40), 8), ((3, 5, 6, 7, 40), 6),
          ((3, 5, 6, 7, 40), 9), ((3, 5, 6, 7, 40), 15), ((3, 5, 6, 7, 40), 11), ((3, 5, 6, 7, 40), 13)]


@pytest.mark.parametrize("case", range(len(NORMND)))
@pytest.mark.parametrize("compute", [0, 1, 2, 3])
def test_normalize_f32_nd(oracle, reference, case, compute):
    """F32 at ranks 1, 4 and 5 (the N-D branch: collapsed axes, dense addressing from the roi begin)."""
    shp, mask = NORMND[case]
    r = rng(260 + case * 4 + compute)
    src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, np.float32, begin_fits=case == 2)
    a, b = run_normalize_nd((oracle, reference), src, shp, np.float32, mask, mean, std, compute, 1.5, 0.25, roi, 0, 0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


NORMINT = [((4, 37, 61), 1), ((4, 37, 61), 2), ((4, 37, 61), 3), ((3, 9, 11, 3), 4), ((3, 9, 11, 3), 3),
           ((3, 9, 11, 3), 5), ((2, 4, 5, 6, 3), 8), ((2, 4, 5, 6, 3), 7)]


@pytest.mark.parametrize("case", range(len(NORMINT)))
@pytest.mark.parametrize("compute", [0, 3])
@pytest.mark.parametrize("dtype", [np.uint8, np.int8])
def test_normalize_integer(oracle, reference, case, compute, dtype):
    """U8 and I8 (non-negative values, results in range) through the generic N-D path at ranks 2-4,
    including the statistics accumulated onto the caller's arrays."""
    shp, mask = NORMINT[case]
    r = rng(300 + case * 4 + compute + (100 if dtype == np.int8 else 0))
    src, roi, mean, std = normalize_nd_case(r, shp, mask, compute, dtype)
    scale, shift = (15.0, 64.0) if dtype == np.int8 else (20.0, 128.0)
    if compute == 0:
        scale = 15.0   # scale / std dev <= 0.75: results stay in range
    a, b = run_normalize_nd((oracle, reference), src, shp, dtype, mask, mean, std, compute, scale, shift, roi, 0, 0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.view(np.uint8) if x.dtype == np.int8 else x,
                                      y.view(np.uint8) if y.dtype == np.int8 else y)
    assert (a[0][0] != 7).any()


def test_normalize_nd_accumulates_onto_caller_statistics(oracle, reference):
    """The N-D branch adds its sums to the values already in the caller's mean / std-dev arrays
    (normalize.cpp:200-242 never clears them); the restatement does the same."""
    r = rng(330)
    src, roi, _, _ = normalize_nd_case(r, (3, 5, 6, 7, 40), 8, 3, np.float32)
    size = 3 * 5 * 6 * 7
    mean = r.uniform(-1, 1, size).astype(np.float32)
    std = r.uniform(0, 1, size).astype(np.float32)
    a, b = run_normalize_nd((oracle, reference), src, src.shape, np.float32, 8, mean, std, 3, 1.0, 0.0, roi, 0, 0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
