"""Seeded random cases of the bit-exact entry points against the oracle (the C restatement of the
reference's host path, itself pinned bit-exact to the reference's library), and of the fused front end
against the plain four calls.

The parity suites pin fixed parameter sets; these draw batch sizes, lengths (0, 1, 2, full rows and
window-length edges mixed in), row padding, borders, channel counts, rate pairs (down, up and equal),
window lobes, FFT sizes, windows, steps, filter counts, frequency ranges, mel formulas, reset intervals
and cutoffs at random, and require the same bits everywhere the oracle writes, and the canvas
everywhere it does not.
"""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, synth
from rpp_b200.types import RppStatus, audio_desc, frontend_params, spectra_desc
from gpu_util import dev, host
from test_gpu_frontend import plain_chain

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS
SEEDS = range(12)
CANVAS = -12345.0


def lengths(r, n, L, extra=()):
    special = [0, 1, 2, 3, L - 1, L] + list(extra)
    v = r.integers(0, L + 1, n)
    for i in range(1, n):
        if r.random() < 0.4:
            v[i] = special[int(r.integers(0, len(special)))]
    v[0] = L
    return np.clip(v, 0, L).astype(np.int32)


def canvas_like(shape):
    return torch.full(shape, CANVAS, device="cuda"), np.full(shape, CANVAS, np.float32)


@pytest.mark.parametrize("seed", SEEDS)
def test_pre_emphasis_and_down_mixing_random(gpu, oracle, seed):
    r = np.random.Generator(np.random.PCG64(7000 + seed))
    n, L, pad = int(r.integers(1, 9)), int(r.integers(1, 20000)), int(r.choice([0, 1, 3, 8]))
    lens = lengths(r, n, L)
    x = r.normal(0, 0.3, (n, L + pad)).astype(np.float32)
    coeff = r.uniform(0.0, 1.0, n).astype(np.float32)
    border = int(r.integers(0, 3))
    out, ref = canvas_like(x.shape)
    oracle.pre_emphasis(x, ref, lens, coeff, border)
    assert audio.pre_emphasis_filter(dev(x), audio_desc(n, L + pad), out, audio_desc(n, L + pad), dev(lens),
                                     dev(coeff), border, gpu) == OK
    np.testing.assert_array_equal(host(out), ref)

    C = int(r.integers(1, 13))
    normalize = bool(r.integers(0, 2))
    xc = r.normal(0, 0.3, (n, (L + pad) * C)).astype(np.float32)
    dims = np.stack([lens, np.full(n, C, np.int32)], 1).astype(np.int32)
    out, ref = canvas_like((n, L + pad))
    oracle.down_mixing(xc, ref, dims.ravel(), normalize)
    assert audio.down_mixing(dev(xc), audio_desc(n, L + pad, channels=C, num_dims=3), out, audio_desc(n, L + pad),
                             dev(dims), normalize, gpu) == OK
    np.testing.assert_array_equal(host(out), ref)


@pytest.mark.parametrize("seed", SEEDS)
def test_resample_random(gpu, oracle, seed):
    r = np.random.Generator(np.random.PCG64(7100 + seed))
    n, L = int(r.integers(1, 7)), int(r.integers(1, 30000))
    lens = lengths(r, n, L)
    rates = np.array([8000, 11025, 16000, 22050, 32000, 44100, 48000], np.float32)
    ir = r.choice(rates, n).astype(np.float32)
    orr = np.full(n, r.choice(rates), np.float32)
    lobes = int(r.choice([4, 8, 16, 24]))
    coeffs = lobes * int(r.choice([64, 48])) + 1        # table scale 32 (exact walk) or 24 (general path)
    lut, scale, center, lobes = oracle.windowed_sinc(coeffs, lobes)
    C = int(r.integers(1, 4))
    out_len = int(max(np.ceil(np.float32(np.float32(L) * o) / i) for i, o in zip(ir, orr))) + int(r.integers(0, 9))
    x = r.normal(0, 0.3, (n, L * C)).astype(np.float32)
    dims = np.stack([lens, np.full(n, C, np.int32)], 1).astype(np.int32)
    out, ref = canvas_like((n, out_len * C))
    oracle.resample(x, ref, ir, orr, dims.ravel(), lut, scale, center, lobes)
    lut_d = dev(lut)
    win = audio.resampling_window(lut_d, scale, center, lobes)
    assert audio.resample(dev(x), audio_desc(n, L, channels=C), out, audio_desc(n, out_len, channels=C), dev(ir),
                          dev(orr), dev(dims), win, gpu) == OK
    np.testing.assert_array_equal(host(out), ref)


@pytest.mark.parametrize("seed", SEEDS)
def test_mel_filter_bank_random(gpu, oracle, seed):
    r = np.random.Generator(np.random.PCG64(7200 + seed))
    nfft = int(r.choice([256, 512, 1024]))
    bins = nfft // 2 + 1
    n, T = int(r.integers(1, 7)), int(r.integers(1, 400))
    frames = r.integers(0, T + 1, n).astype(np.int32)
    frames[0] = T
    nmel = int(min(r.choice([20, 40, 64, 80, 128]), bins - 1))
    fmax = float(r.choice([0.0, 6000.0, 8000.0]))
    fmin = float(r.choice([0.0, 30.0, 300.0]))
    htk, normalize = int(r.integers(0, 2)), bool(r.integers(0, 2))
    spec = (r.random((n, bins, T)) ** 2).astype(np.float32)
    dims = np.stack([np.full(n, bins, np.int32), frames], 1).astype(np.int32)
    out, ref = canvas_like((n, nmel, T))
    oracle.mel_filter_bank(spec, ref, dims.ravel(), fmax, fmin, htk, nmel, 16000.0, normalize)
    assert audio.mel_filter_bank(dev(spec), spectra_desc(n, bins, T), out, spectra_desc(n, nmel, T), dev(dims), fmax,
                                 fmin, htk, nmel, 16000.0, normalize, gpu) == OK
    np.testing.assert_array_equal(host(out), ref)


@pytest.mark.parametrize("seed", SEEDS)
def test_nsr_random(gpu, oracle, seed):
    r = np.random.Generator(np.random.PCG64(7300 + seed))
    n, L = int(r.integers(1, 9)), int(r.integers(1, 60000))
    window = int(r.choice([16, 100, 512, 2048]))
    lens = lengths(r, n, L, extra=[window - 1, window, window + 1])
    x = r.normal(0, 0.3, (n, L)).astype(np.float32)
    for b in range(n):   # silent stretches
        for _ in range(int(r.integers(0, 4))):
            a = int(r.integers(0, L))
            x[b, a:a + int(r.integers(1, L // 3 + 2))] = 0.0
    reset = int(r.choice([-1, 1000, 8192]))
    cut, ref_power = float(r.choice([-60.0, -30.0, -10.0])), float(r.choice([0.0, 0.05]))
    b_ref, l_ref = oracle.nsr(x, lens, cut, window, ref_power, reset)
    begin = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    length = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    assert audio.non_silent_region_detection(dev(x), audio_desc(n, L), dev(lens), begin, length, cut, window,
                                             ref_power, reset, gpu) == OK
    np.testing.assert_array_equal(host(begin), b_ref)
    np.testing.assert_array_equal(host(length), l_ref)


@pytest.mark.parametrize("seed", SEEDS)
def test_frontend_equals_plain_chain_random(gpu, seed):
    r = np.random.Generator(np.random.PCG64(7400 + seed))
    nfft = int(r.choice([128, 256, 512, 1024, 2048]))
    W = int(r.integers(max(8, nfft // 4), nfft + 1))
    hop = int(r.integers(max(1, W // 4), min(W, 1000) + 1))
    kw = dict(nfft=nfft, window_length=W, window_step=hop, num_filter=int(min(r.choice([20, 40, 80, 128]), nfft // 2)),
              center=bool(r.integers(0, 2)), reflect=bool(r.integers(0, 2)), border=int(r.integers(0, 3)),
              mel_formula=int(r.integers(0, 2)), normalize=bool(r.integers(0, 2)),
              reference_magnitude=float(r.choice([0.0, 1.0])), lookahead=int(r.choice([0, 1, 8, 64])),
              db_frames=int(r.choice([0, 16, 64, 256])), power=int(r.integers(1, 3)))
    p = frontend_params(**kw)
    L = int(r.integers(W, 40000))
    lens = lengths(r, 9, L, extra=[W - 1, W, W + 1])
    x, lens = synth.mono_batch(len(lens), lens, r, gaps=True)
    n = x.shape[0]
    coeff = r.uniform(0.5, 0.99, n).astype(np.float32)
    maxf = L // hop + 1
    ref, F = plain_chain(gpu, x, lens, coeff, p, maxf)
    out = torch.full((n, p.numFilter, maxf), CANVAS, device="cuda")
    st = audio.frontend(dev(x), audio_desc(n, x.shape[1]), out, spectra_desc(n, p.numFilter, maxf), dev(lens),
                        dev(coeff), p, gpu)
    if st == RppStatus.RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE:
        pytest.skip("frame tile larger than a CTA's shared memory (documented limit)")
    assert st == OK
    o = host(out)
    for i in range(n):
        if F[i] <= 1:
            continue   # one-frame clips: the plain chain's to_decibels reads them as a 1-D run (see test_gpu_frontend)
        np.testing.assert_array_equal(o[i, :, :F[i]], ref[i, :, :F[i]])
    assert audio.device_error(gpu) == 0
