"""GPU parity of the seven rppt_*_gpu entry points, called through the C ABI (librppb.so),
against the oracle (C restatement, itself pinned bit-exact to the reference's host library and
goldens) on seeded inputs, plus the shipped golden outputs, edge cases and status codes.

Bars: bit-exact for pre-emphasis, down-mixing, resampling and NSR begin/length (NSR may differ
only where a moving mean square is within 1 ulp of the cutoff); mel bit-exact in > 99.9% of
values and within 1e-5 of each frame's maximum everywhere; spectrogram within 1e-5 of each
frame's maximum bin (SPEC_FRAME_REL); decibels within 1e-3 dB (DB_ABS).
"""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, synth
from rpp_b200.types import RppStatus, RpptLayout, audio_desc, spectra_desc, RpptDataType
from gpu_util import dev, pinned, host, canvas, frame_rel_err, SPEC_FRAME_REL, DB_ABS

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS


def rng(k):
    return np.random.Generator(np.random.PCG64(5000 + k))


def batch(n=7, hi=20000, seed=0, lens=None):
    r = rng(seed)
    if lens is None:
        lens = r.integers(1, hi, n)
        lens[0] = hi
    return synth.mono_batch(len(lens), np.asarray(lens, np.int32), r, gaps=True)


# ---------------------------------------------------------------- pre-emphasis

@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("stride_pad", [0, 3])
def test_pre_emphasis(gpu, oracle, border, stride_pad):
    x, lens = batch(seed=border)
    lens[1] = 0
    lens[2] = 1
    n, L = x.shape
    xs = np.zeros((n, L + stride_pad), np.float32)
    xs[:, :L] = x
    d = audio_desc(n, L + stride_pad)
    coeff = rng(3).uniform(0.5, 0.99, n).astype(np.float32)
    ref = np.full_like(xs, -12345.0)
    oracle.pre_emphasis(xs, ref, lens, coeff, border)
    out = canvas(xs.shape)
    st = audio.pre_emphasis_filter(dev(xs), d, out, d, dev(lens), dev(coeff), border, gpu)
    assert st == OK
    np.testing.assert_array_equal(host(out), ref)


def test_pre_emphasis_golden(gpu, golden):
    lens = golden["lengths"].astype(np.int32)
    d = audio_desc(3, int(lens.max()), pad_to_8=True)
    x = np.zeros((3, d.w), np.float32)
    for i in range(3):
        x[i, :lens[i]] = golden[f"pcm{i}"].astype(np.float32) / 32768.0
    out = canvas(x.shape, 0.0)
    coeff = pinned(np.full(3, 0.97, np.float32))
    assert audio.pre_emphasis_filter(dev(x), d, out, d, pinned(lens), coeff, 1, gpu) == OK
    g = golden["pre_emphasis_filter"].reshape(3, d.w)
    o = host(out)
    for i in range(3):
        np.testing.assert_array_equal(o[i, :lens[i]], g[i, :lens[i]])


def test_pre_emphasis_pageable_tensors(gpu, oracle):
    """Per-sample tensors in pageable host memory are staged by the library."""
    x, lens = batch(n=3, seed=11)
    d = audio_desc(3, x.shape[1])
    coeff = np.full(3, 0.9, np.float32)
    ref = np.full_like(x, -12345.0)
    oracle.pre_emphasis(x, ref, lens, coeff, 0)
    out = canvas(x.shape)
    assert audio.pre_emphasis_filter(dev(x), d, out, d, lens, coeff, 0, gpu) == OK
    np.testing.assert_array_equal(host(out), ref)


# ---------------------------------------------------------------- down-mixing

@pytest.mark.parametrize("channels", [1, 2, 3, 4, 6, 8, 13])
@pytest.mark.parametrize("normalize", [False, True])
def test_down_mixing(gpu, oracle, channels, normalize):
    r = rng(channels)
    n, L = 5, 7001
    lens = r.integers(0, L + 1, n).astype(np.int32)
    lens[0] = L
    x = r.normal(0, 0.3, (n, L * channels)).astype(np.float32)
    dims = np.stack([lens, np.full(n, channels, np.int32)], 1).astype(np.int32)
    ref = np.full((n, L), -12345.0, np.float32)
    oracle.down_mixing(x, ref, dims.ravel(), normalize)
    out = canvas((n, L))
    st = audio.down_mixing(dev(x), audio_desc(n, L, channels=channels, num_dims=3), out, audio_desc(n, L),
                           dev(dims), normalize, gpu)
    assert st == OK
    np.testing.assert_array_equal(host(out), ref)


# ---------------------------------------------------------------- resample

@pytest.mark.parametrize("rates,channels", [((16000, 18400), 1), ((48000, 16000), 1), ((44100, 16000), 1),
                                            ((22050, 16000), 1), ((16000, 16000), 1), ((8000, 44100), 1),
                                            ((48000, 16000), 2), ((22050, 16000), 3)])
def test_resample(gpu, oracle, rates, channels):
    r = rng(17)
    n, L = 4, 9000
    lens = np.array([L, 3001, 1, 0], np.int32)
    x = r.normal(0, 0.3, (n, L * channels)).astype(np.float32)
    lut, scale, center, lobes = oracle.windowed_sinc(16 * 64 + 1, 16)
    ir = np.full(n, rates[0], np.float32)
    orr = np.full(n, rates[1], np.float32)
    out_len = int(np.ceil(L * rates[1] / rates[0])) + 8
    dims = np.stack([lens, np.full(n, channels, np.int32)], 1).astype(np.int32)
    ref = np.full((n, out_len * channels), -12345.0, np.float32)
    oracle.resample(x, ref, ir, orr, dims.ravel(), lut, scale, center, lobes)
    out = canvas(ref.shape)
    lut_d = dev(lut)
    win = audio.resampling_window(lut_d, scale, center, lobes)
    st = audio.resample(dev(x), audio_desc(n, L, channels=channels), out, audio_desc(n, out_len, channels=channels),
                        dev(ir), dev(orr), dev(dims), win, gpu)
    assert st == OK
    np.testing.assert_array_equal(host(out), ref)


@pytest.mark.parametrize("coeffs,lobes", [(8 * 64 + 1, 8), (24 * 64 + 1, 24), (16 * 48 + 1, 16), (16 * 128 + 1, 16)])
@pytest.mark.parametrize("rates", [(48000, 16000), (22050, 16000), (16000, 44100)])
def test_resample_windows(gpu, oracle, coeffs, lobes, rates):
    """Tables of scale 32 with 8 and 24 lobes take the exact walk from phase 16 and 32 on; scale 24 (not a
    power of two) and scale 64 (a power of two other than 32) never do.  Bit-exact either way, on mono and
    down-mixed stereo input."""
    r = rng(23 + lobes)
    n, L = 3, 12000
    lens = np.array([L, 5003, 700], np.int32)
    lut, scale, center, lobes = oracle.windowed_sinc(coeffs, lobes)
    ir = np.full(n, rates[0], np.float32)
    orr = np.full(n, rates[1], np.float32)
    out_len = int(np.ceil(L * rates[1] / rates[0])) + 8
    lut_d = dev(lut)
    win = audio.resampling_window(lut_d, scale, center, lobes)
    x = r.normal(0, 0.3, (n, L)).astype(np.float32)
    dims = np.stack([lens, np.ones(n, np.int32)], 1).astype(np.int32)
    ref = np.full((n, out_len), -12345.0, np.float32)
    oracle.resample(x, ref, ir, orr, dims.ravel(), lut, scale, center, lobes)
    out = canvas(ref.shape)
    assert audio.resample(dev(x), audio_desc(n, L), out, audio_desc(n, out_len), dev(ir), dev(orr), dev(dims), win,
                          gpu) == OK
    np.testing.assert_array_equal(host(out), ref)
    # the same mono signal as two equal channels, down-mixed on the fly: the channel mean is the signal
    x2 = np.repeat(x, 2, axis=1)
    dims2 = np.stack([lens, np.full(n, 2, np.int32)], 1).astype(np.int32)
    mono = np.full((n, L), 0.0, np.float32)
    oracle.down_mixing(x2, mono, dims2.ravel(), False)
    ref2 = np.full((n, out_len), -12345.0, np.float32)
    oracle.resample(mono, ref2, ir, orr, dims.ravel(), lut, scale, center, lobes)
    out2 = canvas(ref2.shape)
    assert audio.downmix_resample(dev(x2), audio_desc(n, L, channels=2, num_dims=3), out2, audio_desc(n, out_len),
                                  dev(ir), dev(orr), dev(dims2), False, lut_d, scale, center, lobes, gpu) == OK
    np.testing.assert_array_equal(host(out2), ref2)


def test_resample_golden(gpu, oracle, golden):
    lens = golden["lengths"].astype(np.int32)
    d = audio_desc(3, int(lens.max()), pad_to_8=True)
    x = np.zeros((3, d.w), np.float32)
    for i in range(3):
        x[i, :lens[i]] = golden[f"pcm{i}"].astype(np.float32) / 32768.0
    lut, scale, center, lobes = oracle.windowed_sinc(16 * 64 + 1, 16)
    out_rate = np.float32(16000 * np.float32(1.15))
    g = golden["resample"].reshape(3, -1)
    out = canvas(g.shape, 0.0)
    dims = np.stack([lens, np.ones(3, np.int32)], 1).astype(np.int32)
    lut_p = pinned(lut)
    win = audio.resampling_window(lut_p, scale, center, lobes)
    st = audio.resample(dev(x), d, out, audio_desc(3, g.shape[1]), pinned(np.full(3, 16000, np.float32)),
                        pinned(np.full(3, out_rate, np.float32)), pinned(dims), win, gpu)
    assert st == OK
    o = host(out)
    for i in range(3):
        ol = int(np.ceil(np.float32(np.float32(lens[i]) * out_rate) / np.float32(16000)))
        np.testing.assert_array_equal(o[i, :ol], g[i, :ol])


# ---------------------------------------------------------------- spectrogram

SPEC_CASES = [
    (512, 400, 160, True, True, RpptLayout.NFT, 2),
    (512, 320, 160, True, True, RpptLayout.NTF, 2),
    (512, 512, 128, False, True, RpptLayout.NFT, 1),
    (256, 200, 80, True, False, RpptLayout.NFT, 2),
    (128, 128, 64, True, True, RpptLayout.NTF, 2),
    (1024, 1024, 256, True, True, RpptLayout.NFT, 2),
    (2048, 1600, 512, True, True, RpptLayout.NTF, 2),
    (400, 400, 160, True, True, RpptLayout.NFT, 2),     # non-power-of-two: direct DFT
]


@pytest.mark.parametrize("nfft,W,hop,center,reflect,layout,power", SPEC_CASES)
def test_spectrogram(gpu, oracle, nfft, W, hop, center, reflect, layout, power):
    x, lens = batch(n=6, hi=24000, seed=nfft + W)
    lens[1], lens[2], lens[3] = 1, 2, W - 1
    n = len(lens)
    nft = layout == RpptLayout.NFT
    F = [oracle.num_windows(l, W, hop, center) for l in lens]
    mf = max(F)
    bins = nfft // 2 + 1
    shape = (n, bins, mf) if nft else (n, mf, bins)
    dd = spectra_desc(n, bins, mf, layout) if nft else spectra_desc(n, mf, bins, layout)
    out = canvas(shape)
    st = audio.spectrogram(dev(x), audio_desc(n, x.shape[1]), out, dd, pinned(lens), center, reflect, None, nfft,
                           power, W, hop, gpu)
    assert st == OK
    o = host(out)
    ref = oracle.spectrogram_f64(x, lens, center, reflect, None, nfft, power, W, hop, nft, max_frames=mf)
    for i in range(n):
        if F[i] <= 0:
            assert (o[i] == -12345.0).all()
            continue
        got = o[i, :, :F[i]] if nft else o[i, :F[i], :].T
        exp = ref[i, :, :F[i]] if nft else ref[i, :F[i], :].T
        assert frame_rel_err(got, exp) < SPEC_FRAME_REL, (i, frame_rel_err(got, exp))
        tail = o[i, :, F[i]:] if nft else o[i, F[i]:, :]
        assert (tail == -12345.0).all()


def test_spectrogram_vs_reference_library(gpu, reference):
    """Against the reference's own FP32 host spectrogram (ffts), per-frame relative 1e-5."""
    x, lens = batch(n=5, hi=30000, seed=77)
    n = len(lens)
    F = [l // 160 + 1 for l in lens]
    mf = max(F)
    dd = spectra_desc(n, 257, mf)
    ref = np.zeros((n, 257, mf), np.float32)
    sd = audio_desc(n, x.shape[1])
    assert reference.spectrogram(x, sd, ref, dd, lens, True, True, None, 512, 2, 400, 160) == 0
    out = canvas((n, 257, mf))
    assert audio.spectrogram(dev(x), sd, out, dd, dev(lens), True, True, None, 512, 2, 400, 160, gpu) == OK
    o = host(out)
    for i in range(n):
        assert frame_rel_err(o[i, :, :F[i]], ref[i, :, :F[i]]) < SPEC_FRAME_REL


def test_spectrogram_golden(gpu, golden):
    lens = golden["lengths"].astype(np.int32)
    d = audio_desc(3, int(lens.max()), pad_to_8=True)
    x = np.zeros((3, d.w), np.float32)
    for i in range(3):
        x[i, :lens[i]] = golden[f"pcm{i}"].astype(np.float32) / 32768.0
    F = [225, 211, 214]
    dd = spectra_desc(3, 257, 225)
    out = canvas((3, 257, 225), 0.0)
    assert audio.spectrogram(dev(x), d, out, dd, pinned(lens), True, True, None, 512, 2, 320, 160, gpu) == OK
    o = host(out)
    g = golden["spectrogram"].reshape(3, 257, 225)
    for i in range(3):
        assert frame_rel_err(o[i, :, :F[i]], g[i, :, :F[i]]) < SPEC_FRAME_REL


def test_spectrogram_custom_window(gpu, oracle):
    x, lens = batch(n=3, hi=8000, seed=5)
    W = 300
    win = np.hamming(W).astype(np.float32)
    F = [oracle.num_windows(l, W, 100, True) for l in lens]
    mf = max(F)
    out = canvas((3, 257, mf))
    st = audio.spectrogram(dev(x), audio_desc(3, x.shape[1]), out, spectra_desc(3, 257, mf), dev(lens), True, True,
                           win, 512, 2, W, 100, gpu)
    assert st == OK
    ref = oracle.spectrogram_f64(x, lens, 1, 1, win, 512, 2, W, 100, 1, max_frames=mf)
    o = host(out)
    for i in range(3):
        assert frame_rel_err(o[i, :, :F[i]], ref[i, :, :F[i]]) < SPEC_FRAME_REL


# ---------------------------------------------------------------- mel filter bank

@pytest.mark.parametrize("htk,normalize,nfft,nmel,fmin,fmax", [
    (0, 1, 512, 128, 0.0, 8000.0), (1, 1, 512, 80, 0.0, 0.0), (0, 0, 1024, 64, 60.0, 7600.0),
    (1, 0, 256, 40, 20.0, 4000.0), (0, 1, 2048, 256, 0.0, 8000.0)])
def test_mel_filter_bank(gpu, oracle, htk, normalize, nfft, nmel, fmin, fmax):
    r = rng(nfft + nmel)
    n, bins, T = 4, nfft // 2 + 1, 150
    frames = np.array([T, 70, 1, 0], np.int32)
    spec = (r.random((n, bins, T)) ** 4).astype(np.float32)
    dims = np.stack([np.full(n, bins, np.int32), frames], 1).astype(np.int32)
    ref = np.full((n, nmel, T), -12345.0, np.float32)
    oracle.mel_filter_bank(spec, ref, dims.ravel(), fmax, fmin, htk, nmel, 16000, normalize)
    out = canvas((n, nmel, T))
    st = audio.mel_filter_bank(dev(spec), spectra_desc(n, bins, T), out, spectra_desc(n, nmel, T), pinned(dims),
                               fmax, fmin, htk, nmel, 16000, normalize, gpu)
    assert st == OK
    o = host(out)
    exact = (o == ref).mean()
    assert exact > 0.999, exact
    for i in range(n):
        zc = min(frames[i] + 8, T)
        assert (o[i, :, zc:] == -12345.0).all()
        if frames[i]:
            assert frame_rel_err(o[i, :, :frames[i]], ref[i, :, :frames[i]]) < 1e-6


def test_mel_filter_bank_golden(gpu, golden):
    dims = np.array([[257, 225], [257, 211], [257, 214]], np.int32)
    spec = golden["spectrogram"].reshape(3, 257, 225).copy()
    out = canvas((3, 80, 225), 0.0)
    st = audio.mel_filter_bank(dev(spec), spectra_desc(3, 257, 225), out, spectra_desc(3, 80, 225), dev(dims), 8000,
                               0, 0, 80, 16000, True, gpu)
    assert st == OK
    o = host(out)
    g = golden["mel_filter_bank"].reshape(3, 80, 225)
    for i in range(3):
        np.testing.assert_array_equal(o[i, :, :dims[i, 1]], g[i, :, :dims[i, 1]])


# ---------------------------------------------------------------- to_decibels

@pytest.mark.parametrize("two_d,ref_mag", [(False, 0.0), (True, 0.0), (True, 2.5), (False, 1.0)])
def test_to_decibels(gpu, oracle, two_d, ref_mag):
    r = rng(21)
    n, H, Wd = 4, 128, 1601
    if two_d:
        x = (r.random((n, H, Wd)) ** 3).astype(np.float32)
        wh = [(Wd, H), (700, 100), (1, 1), (0, 0)]
        desc = spectra_desc(n, H, Wd)
    else:
        x = (r.normal(0, 1, (n, H * Wd)) ** 2).astype(np.float32)
        wh = [(1, H * Wd), (1, 10001), (1, 1), (1, 0)]
        desc = audio_desc(n, H * Wd)
    dims = np.array(wh, np.uint32)
    ref = np.full_like(x, -12345.0)
    oracle.to_decibels(x, ref, dims, -80.0, 10.0, ref_mag)
    out = canvas(x.shape)
    st = audio.to_decibels(dev(x), desc, out, desc, audio.image_patches(*zip(*wh)), -80.0, 10.0, ref_mag, gpu)
    assert st == OK
    o = host(out)
    untouched = ref == -12345.0
    assert (o[untouched] == -12345.0).all()
    assert np.abs(o[~untouched] - ref[~untouched]).max() <= DB_ABS / 10


def test_to_decibels_golden(gpu, golden):
    lens = golden["lengths"].astype(np.int32)
    d = audio_desc(3, int(lens.max()), pad_to_8=True)
    x = np.zeros((3, d.w), np.float32)
    for i in range(3):
        x[i, :lens[i]] = golden[f"pcm{i}"].astype(np.float32) / 32768.0
    dims = np.stack([np.ones(3, np.uint32), lens.astype(np.uint32)], 1)
    out = canvas(x.shape, 0.0)
    st = audio.to_decibels(dev(x), d, out, d, pinned(dims), np.float32(np.log(1e-20)), np.float32(np.log(10)), 1.0,
                           gpu)
    assert st == OK
    o = host(out)
    g = golden["to_decibels"].reshape(3, d.w)
    for i in range(3):
        assert np.abs(o[i, :lens[i]] - g[i, :lens[i]]).max() <= DB_ABS / 10


# ---------------------------------------------------------------- non-silent region

@pytest.mark.parametrize("reset,window,ref,cut", [(8192, 2048, 0.0, -60.0), (-1, 2048, 0.0, -60.0),
                                                  (1000, 333, 0.0, -40.0), (8192, 2048, 0.05, -20.0),
                                                  (4096, 1, 0.0, -3.0)])
def test_nsr(gpu, oracle, reset, window, ref, cut):
    x, lens = batch(n=9, hi=70000, seed=31)
    lens[1], lens[2] = 0, 1
    x[3] = 0.0          # a silent sample
    b_ref, l_ref, mms, cutoff = oracle.nsr(x, lens, cut, window, ref, reset, want_mms=True)
    begin = torch.full((len(lens),), -7, dtype=torch.int32, device="cuda")
    length = torch.full((len(lens),), -7, dtype=torch.int32, device="cuda")
    st = audio.non_silent_region_detection(dev(x), audio_desc(len(lens), x.shape[1]), dev(lens), begin, length, cut,
                                           window, ref, reset, gpu)
    assert st == OK
    np.testing.assert_array_equal(host(begin), b_ref)
    np.testing.assert_array_equal(host(length), l_ref)


def test_nsr_golden_pinned_outputs(gpu, golden):
    lens = golden["lengths"].astype(np.int32)
    d = audio_desc(3, int(lens.max()), pad_to_8=True)
    x = np.zeros((3, d.w), np.float32)
    for i in range(3):
        x[i, :lens[i]] = golden[f"pcm{i}"].astype(np.float32) / 32768.0
    begin = pinned(np.full(3, -1, np.int32))
    length = pinned(np.full(3, -1, np.int32))
    assert audio.non_silent_region_detection(dev(x), d, pinned(lens), begin, length, -60.0, 2048, 0.0, 8192,
                                             gpu) == OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(begin.numpy(), golden["nsr_begin"])
    np.testing.assert_array_equal(length.numpy(), golden["nsr_length"])


def test_nsr_pageable_outputs(gpu, oracle):
    x, lens = batch(n=4, hi=30000, seed=41)
    b_ref, l_ref = oracle.nsr(x, lens, -50, 1024, 0.0, 4096)
    begin = np.full(4, -1, np.int32)
    length = np.full(4, -1, np.int32)
    assert audio.non_silent_region_detection(dev(x), audio_desc(4, x.shape[1]), lens, begin, length, -50, 1024, 0.0,
                                             4096, gpu) == OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(begin, b_ref)
    np.testing.assert_array_equal(length, l_ref)


# ---------------------------------------------------------------- status codes (reference GPU dispatch)

def test_status_codes(gpu):
    x = dev(np.zeros((2, 64), np.float32))
    y = canvas((2, 64))
    lens = dev(np.array([64, 64], np.int32))
    coeff = dev(np.array([0.9, 0.9], np.float32))
    d1 = audio_desc(2, 64)
    d3 = audio_desc(2, 64, num_dims=3)
    assert audio.pre_emphasis_filter(x, d3, y, d1, lens, coeff, 0, gpu) == RppStatus.RPP_ERROR_INVALID_SRC_DIMS
    du8 = audio_desc(2, 64)
    du8.dataType = RpptDataType.U8
    assert audio.pre_emphasis_filter(x, du8, y, d1, lens, coeff, 0, gpu) == RppStatus.RPP_ERROR_NOT_IMPLEMENTED
    patches = audio.image_patches([1, 1], [64, 64])
    assert audio.to_decibels(x, d1, y, d1, patches, -80, 0.0, 0, gpu) == RppStatus.RPP_ERROR_ZERO_DIVISION
    sd = spectra_desc(2, 257, 8)
    sd.layout = RpptLayout.NCHW
    assert audio.spectrogram(x, d1, y, sd, lens, True, True, None, 512, 2, 400, 160,
                             gpu) == RppStatus.RPP_ERROR_INVALID_DST_LAYOUT
    assert audio.spectrogram(x, d3, y, spectra_desc(2, 257, 8), lens, True, True, None, 512, 2, 400, 160,
                             gpu) == RppStatus.RPP_ERROR_INVALID_SRC_DIMS
    assert audio.spectrogram(x, d1, y, spectra_desc(2, 257, 8), lens, True, True, None, 256, 2, 400, 160,
                             gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
    ms = spectra_desc(2, 257, 8)
    assert audio.mel_filter_bank(x, ms, y, ms, lens, 9000, 0, 0, 16, 16000, True,
                                 gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
    ms_t = spectra_desc(2, 257, 8, RpptLayout.NTF)
    assert audio.mel_filter_bank(x, ms_t, y, ms, lens, 8000, 0, 0, 16, 16000, True,
                                 gpu) == RppStatus.RPP_ERROR_INVALID_SRC_LAYOUT
    b = torch.zeros(2, dtype=torch.int32, device="cuda")
    assert audio.non_silent_region_detection(x, d1, lens, b, b, -60, 2048, 0.0, 0,
                                             gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
    assert audio.non_silent_region_detection(x, d3, lens, b, b, -60, 2048, 0.0, 8192,
                                             gpu) == RppStatus.RPP_ERROR_INVALID_SRC_DIMS
    torch.cuda.synchronize()


# ---------------------------------------------------------------- fused down-mix + resample

@pytest.mark.parametrize("channels,normalize", [(2, False), (2, True), (1, False), (5, False)])
def test_downmix_resample_equals_two_calls(gpu, channels, normalize):
    from rpp_b200.windows import kaiser_sinc
    r = rng(71 + channels)
    n, L = 6, 20000
    lens = r.integers(1, L + 1, n).astype(np.int32)
    lens[0] = L
    rates = np.array([16000, 22050, 44100, 48000, 48000, 16000], np.float32)
    x = r.normal(0, 0.3, (n, L * channels)).astype(np.float32)
    lut, scale, center, lobes = kaiser_sinc(16)
    out_len = int(np.ceil(L * 16000 / 16000)) + 8
    dims = dev(np.stack([lens, np.full(n, channels, np.int32)], 1).astype(np.int32))
    mono_dims = dev(np.stack([lens, np.ones(n, np.int32)], 1).astype(np.int32))
    xd = dev(x)
    mono = canvas((n, L))
    assert audio.down_mixing(xd, audio_desc(n, L, channels=channels, num_dims=3), mono, audio_desc(n, L), dims,
                             normalize, gpu) == OK
    ref = canvas((n, out_len))
    lut_d = dev(lut)
    win = audio.resampling_window(lut_d, scale, center, lobes)
    ir, orr = dev(rates), dev(np.full(n, 16000, np.float32))
    assert audio.resample(mono, audio_desc(n, L), ref, audio_desc(n, out_len), ir, orr, mono_dims, win, gpu) == OK
    out = canvas((n, out_len))
    assert audio.downmix_resample(xd, audio_desc(n, L, channels=channels, num_dims=3), out, audio_desc(n, out_len),
                                  ir, orr, dims, normalize, lut_d, scale, center, lobes, gpu) == OK
    np.testing.assert_array_equal(host(out), host(ref))


# ---------------------------------------------------------------- slice (api/rppt_tensor_geometric_augmentations.h:486)

def test_slice_golden_case(gpu, oracle, golden):
    """The audio QA slice (1-D, anchor 10, shape length/2, roi {10, length}, padding with fill 0)
    through the C ABI equals the oracle on every element the call writes."""
    from rpp_b200.types import generic_desc
    lens = golden["lengths"].astype(np.int32)
    n = len(lens)
    w = (int(lens.max()) // 8) * 8 + 8
    x = np.zeros((n, w), np.float32)
    for i in range(n):
        x[i, :lens[i]] = golden[f"pcm{i}"].astype(np.float32) / 32768.0
    anchor = np.full(n, 10, np.int32)
    shape = (lens // 2).astype(np.int32)
    roi = np.stack([np.full(n, 10), lens], 1).astype(np.uint32).ravel()
    d = generic_desc((n, w))
    out = torch.full((n, w), -7.0, device="cuda")
    fill = np.zeros(1, np.float32)
    assert audio.slice(dev(x), d, out, d, anchor, shape, fill, True, roi, gpu) == RppStatus.RPP_SUCCESS
    exp = np.full((n, w), -7.0, np.float32)
    oracle.slice(x, exp, anchor, shape, roi, 0.0, True, 1)
    np.testing.assert_array_equal(host(out), exp)


@pytest.mark.parametrize("num_dims", [1, 2])
@pytest.mark.parametrize("dtype", [np.float32, np.uint8])
@pytest.mark.parametrize("pad", [False, True])
def test_slice_vs_oracle(gpu, oracle, num_dims, dtype, pad):
    """Random boxes, some past the roi lengths (padding), some with anchors beyond the length
    (nothing copied), per-sample tensors in pageable, pinned and device memory."""
    from rpp_b200.types import generic_desc, RpptDataType
    r = np.random.Generator(np.random.PCG64(77 + num_dims))
    n = 9
    shp = (n, 20000) if num_dims == 1 else (n, 33, 70)
    src = (r.integers(0, 255, shp).astype(np.uint8) if dtype == np.uint8
           else r.standard_normal(shp).astype(np.float32))
    ext = np.array(shp[1:])
    length = np.stack([r.integers(1, e + 1, n) for e in ext], 1).astype(np.int32)
    anchor = np.stack([r.integers(0, e, n) for e in ext], 1).astype(np.int32)
    shape = np.stack([r.integers(1, e + 1, n) for e in ext], 1).astype(np.int32)
    roi = np.concatenate([np.zeros_like(length), length], 1).astype(np.uint32).ravel()
    fill = np.array([5 if dtype == np.uint8 else -2.5], dtype)
    dt = RpptDataType.U8 if dtype == np.uint8 else RpptDataType.F32
    d = generic_desc(shp, dt)
    canvas_v = 9 if dtype == np.uint8 else 9.75
    out = torch.from_numpy(np.full(shp, canvas_v, dtype)).cuda()
    a_t, s_t = anchor.ravel(), shape.ravel()
    args = [(a_t, s_t, roi), (pinned(a_t), pinned(s_t), pinned(roi)), (dev(a_t), dev(s_t), dev(roi))]
    for k, (aa, ss, rr) in enumerate(args):
        out.fill_(canvas_v)
        st = audio.slice(dev(src), d, out, d, aa, ss, fill, pad, rr, gpu)
        assert st == RppStatus.RPP_SUCCESS
        exp = np.full(shp, canvas_v, dtype)
        oracle.slice(src, exp, a_t, s_t, roi, fill[0], pad, num_dims)
        np.testing.assert_array_equal(host(out), exp)


SLICE_ND = [(0, (5, 3, 37, 53)), (0, (5, 1, 29, 64)), (1, (5, 31, 47, 3)), (1, (5, 17, 40, 4)),
            (2, (4, 3, 9, 21, 33)), (2, (4, 1, 7, 16, 24)), (3, (4, 8, 19, 27, 3)), (3, (4, 6, 11, 13, 2))]


@pytest.mark.parametrize("case", range(len(SLICE_ND)))
@pytest.mark.parametrize("dtype", [np.float32, np.uint8])
@pytest.mark.parametrize("pad", [False, True])
def test_slice_nd_vs_oracle(gpu, oracle, case, dtype, pad):
    """3-D (NCHW, NHWC) and 4-D (NCDHW, NDHWC) boxes: random anchors (some beyond the roi length:
    nothing copied), shapes and roi lengths, bit for bit against the restatement of the
    reference's host slice, the rest of the destination untouched."""
    from rpp_b200.types import generic_desc, RpptDataType
    layout, shp = SLICE_ND[case]
    r = np.random.Generator(np.random.PCG64(177 + case))
    n, ext = shp[0], np.array(shp[1:])
    src = (r.integers(0, 255, shp).astype(np.uint8) if dtype == np.uint8
           else r.standard_normal(shp).astype(np.float32))
    length = np.stack([r.integers(1, e + 1, n) for e in ext], 1).astype(np.int32)
    anchor = np.stack([r.integers(0, e, n) for e in ext], 1).astype(np.int32)
    shape = np.stack([r.integers(1, e + 1, n) for e in ext], 1).astype(np.int32)
    anchor[0] = 0
    length[0] = ext
    shape[0] = ext                                     # the whole first sample
    roi = np.concatenate([np.zeros_like(length), length], 1).astype(np.uint32).ravel()
    fill = np.array([5 if dtype == np.uint8 else -2.5], dtype)
    dt = RpptDataType.U8 if dtype == np.uint8 else RpptDataType.F32
    d = generic_desc(shp, dt, layout)
    canvas_v = 9 if dtype == np.uint8 else 9.75
    out = torch.from_numpy(np.full(shp, canvas_v, dtype)).cuda()
    st = audio.slice(dev(src), d, out, d, anchor.ravel(), shape.ravel(), fill, pad, roi, gpu)
    assert st == RppStatus.RPP_SUCCESS
    exp = np.full(shp, canvas_v, dtype)
    oracle.slice_nd(src, exp, anchor.ravel(), shape.ravel(), roi, fill[0], pad, layout)
    got = host(out)
    np.testing.assert_array_equal(got, exp)
    np.testing.assert_array_equal(got[0], src[0])


def test_slice_status_codes(gpu):
    from rpp_b200.types import generic_desc, RpptDataType, RpptLayout
    x = torch.zeros((2, 100), device="cuda")
    a = np.zeros(2, np.int32)
    s = np.full(2, 10, np.int32)
    roi = np.array([0, 100, 0, 100], np.uint32)
    f = np.zeros(1, np.float32)
    d = generic_desc((2, 100))
    bad = generic_desc((2, 100), RpptDataType.F16)
    assert audio.slice(x, bad, x, d, a, s, f, True, roi, gpu) == RppStatus.RPP_ERROR_INVALID_SRC_DATATYPE
    assert audio.slice(x, d, x, bad, a, s, f, True, roi, gpu) == RppStatus.RPP_ERROR_INVALID_DST_DATATYPE
    other = generic_desc((2, 100), layout=RpptLayout.NHWC)
    assert audio.slice(x, d, x, other, a, s, f, True, roi, gpu) == RppStatus.RPP_ERROR_LAYOUT_MISMATCH
    # 3-D / 4-D tensors in layouts the reference does not slice
    d4 = generic_desc((2, 1, 10, 10), layout=RpptLayout.NFT)
    assert audio.slice(x, d4, x, d4, a, s, f, True, roi, gpu) == RppStatus.RPP_ERROR_NOT_IMPLEMENTED
    d5 = generic_desc((2, 1, 2, 5, 10), layout=RpptLayout.NCHW)
    assert audio.slice(x, d5, x, d5, a, s, f, True, roi, gpu) == RppStatus.RPP_ERROR_NOT_IMPLEMENTED
    # channel counts must match; destination strides must nest
    a3, s3 = np.zeros(6, np.int32), np.full(6, 2, np.int32)
    roi3 = np.tile(np.array([0, 0, 0, 1, 10, 10], np.uint32), 2)
    src3 = generic_desc((2, 1, 10, 10))
    dst3 = generic_desc((2, 2, 10, 5))
    assert audio.slice(x, src3, x, dst3, a3, s3, f, True, roi3, gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS
    squeezed = generic_desc((2, 1, 10, 10))
    squeezed.strides[2] = 5   # rows of 10 elements 5 apart
    assert audio.slice(x, src3, x, squeezed, a3, s3, f, True, roi3, gpu) == RppStatus.RPP_ERROR_INVALID_ARGUMENTS


# ---------------------------------------------------------------- normalize (api/rppt_tensor_statistical_operations.h:193)

@pytest.mark.parametrize("cols", [300, 700, 3000])
@pytest.mark.parametrize("axis_mask", [1, 2, 3])
@pytest.mark.parametrize("compute", [0, 1, 2, 3])
def test_normalize_vs_oracle(gpu, oracle, cols, axis_mask, compute):
    """2-D F32 normalize against the oracle (itself bit-exact to the reference host library): the
    computed means bit for bit (the same halving-tree sums), the inverse std devs and the outputs
    within 1e-5 (the reference refines an SSE rsqrt estimate, CUDA rounds rsqrt correctly); the
    destination outside the roi is zeroed."""
    from rpp_b200.types import generic_desc
    r = np.random.Generator(np.random.PCG64(300 + cols + 10 * axis_mask + compute))
    n, R = 5, 40
    src = (r.standard_normal((n, R, cols)) * 3 + 1).astype(np.float32)
    src[2, 3, :] = 0.5
    roi = np.zeros((n, 4), np.uint32)
    roi[:, 2] = r.integers(20, R + 1, n)
    roi[:, 3] = r.integers(cols // 2, cols + 1, n)
    roi[0, 2:] = (R, cols)
    size = max(int(np.prod([1 if axis_mask & (1 << i) else roi[b, 2 + i] for i in range(2)])) for b in range(n))
    per = n * size
    mean = (r.standard_normal(per) * 0.1).astype(np.float32)
    std = r.uniform(0.5, 2.0, per).astype(np.float32)
    std[1] = 0.0
    m_ref, s_ref = mean.copy(), std.copy()
    exp = np.full((n, R, cols), 7.0, np.float32)
    oracle.normalize_2d(src, exp, axis_mask, m_ref, s_ref, compute, 1.5, 0.25, roi.ravel())
    d = generic_desc((n, R, cols))
    out = torch.full((n, R, cols), 7.0, device="cuda")
    m_gpu, s_gpu = dev(mean.copy()), dev(std.copy())
    st = audio.normalize(dev(src), d, out, d, axis_mask, m_gpu, s_gpu, compute, 1.5, 0.25, roi.ravel(), gpu)
    assert st == RppStatus.RPP_SUCCESS
    got = host(out)
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-5)
    if compute & 1:
        np.testing.assert_array_equal(host(m_gpu)[:per], m_ref[:per])
    if compute & 2:
        np.testing.assert_allclose(host(s_gpu)[:per], s_ref[:per], rtol=1e-6, atol=0)


def test_normalize_frontend_output(gpu, oracle):
    """The RNN-T-style step: per-filter normalisation over time of the fused front end's decibels."""
    from rpp_b200.types import generic_desc, frontend_params
    x, lens = synth.gapped_clips(n=6, max_len=48000)
    n, L = x.shape
    mf = 48000 // 160 + 1
    db = torch.zeros((n, 128, mf), device="cuda")
    assert audio.frontend(dev(x), audio_desc(n, L), db, spectra_desc(n, 128, mf), dev(lens),
                          dev(np.full(n, 0.97, np.float32)), frontend_params(), gpu) == RppStatus.RPP_SUCCESS
    F = lens // 160 + 1
    roi = np.stack([np.zeros(n), np.zeros(n), np.full(n, 128), F], 1).astype(np.uint32).ravel()
    d = generic_desc((n, 128, mf))
    out = torch.zeros_like(db)
    mean, std = torch.zeros(n * 128, device="cuda"), torch.zeros(n * 128, device="cuda")
    assert audio.normalize(db, d, out, d, 2, mean, std, 3, 1.0, 0.0, roi, gpu) == RppStatus.RPP_SUCCESS
    src = host(db)
    exp = np.zeros_like(src)
    m, s = np.zeros(n * 128, np.float32), np.zeros(n * 128, np.float32)
    oracle.normalize_2d(src, exp, 2, m, s, 3, 1.0, 0.0, roi)
    np.testing.assert_allclose(host(out), exp, rtol=1e-5, atol=1e-5)
    np.testing.assert_array_equal(host(mean), m)


# ---------------------------------------------------------------- 16-bit PCM ingest (extension)

@pytest.mark.parametrize("channels", [1, 2, 6])
def test_pcm16_to_f32(gpu, golden, channels):
    """int16 -> float / 32768 on the device equals the test suite's host conversion (exact), only
    over each clip's frames x channels; the QA WAVs convert to the goldens' inputs."""
    r = np.random.Generator(np.random.PCG64(90 + channels))
    n = 7
    frames = r.integers(0, 5000, n).astype(np.int32)
    frames[0] = 5000
    L = 5000 * channels + 3
    pcm = r.integers(-32768, 32768, (n, L)).astype(np.int16)
    sd = audio_desc(n, L // channels if channels > 1 else L, channels=channels)
    sd.strides.nStride = L
    sd.dataType = RpptDataType.I16
    dd = audio_desc(n, L // channels if channels > 1 else L, channels=channels)
    dd.strides.nStride = L
    out = torch.full((n, L), -9.0, device="cuda")
    assert audio.pcm16_to_f32(dev(pcm), sd, out, dd, frames, gpu) == RppStatus.RPP_SUCCESS
    got = host(out)
    for b in range(n):
        k = int(frames[b]) * channels
        np.testing.assert_array_equal(got[b, :k], pcm[b, :k].astype(np.float32) / np.float32(32768.0))
        assert (got[b, k:] == -9.0).all()
    # the QA WAVs
    lens = golden["lengths"].astype(np.int32)
    w = int(lens.max())
    q = np.zeros((3, w), np.int16)
    for i in range(3):
        q[i, :lens[i]] = golden[f"pcm{i}"]
    qs = audio_desc(3, w)
    qs.dataType = RpptDataType.I16
    qo = torch.zeros((3, w), device="cuda")
    assert audio.pcm16_to_f32(dev(q), qs, qo, audio_desc(3, w), lens, gpu) == RppStatus.RPP_SUCCESS
    np.testing.assert_array_equal(host(qo), q.astype(np.float32) / 32768.0)


def test_mel_filter_bank_256_filters(gpu, oracle):
    """256 filters: the mel tile's dynamic shared memory plus its static part passes 48 KB, which
    needs the kernel's opt-in attribute."""
    r = np.random.Generator(np.random.PCG64(123))
    n, mf = 3, 200
    spec = r.uniform(0, 4, (n, 257, mf)).astype(np.float32)
    F = np.array([200, 150, 1], np.int32)
    dims = np.stack([np.full(n, 257, np.int32), F], 1).astype(np.int32)
    out = torch.zeros((n, 256, mf), device="cuda")
    assert audio.mel_filter_bank(dev(spec), spectra_desc(n, 257, mf), out, spectra_desc(n, 256, mf), dev(dims), 8000.0,
                                 0.0, 0, 256, 16000.0, True, gpu) == RppStatus.RPP_SUCCESS
    exp = np.zeros((n, 256, mf), np.float32)
    oracle.mel_filter_bank(spec, exp, dims.ravel(), 8000.0, 0.0, 0, 256, 16000.0, 1)
    got = host(out)
    for i in range(n):
        np.testing.assert_array_equal(got[i, :, :F[i]], exp[i, :, :F[i]])
