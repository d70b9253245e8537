"""Random valid calls of every entry point against the bounds-checked library (librppb_checked.so).

Seeded random batch sizes, lengths (0, 1, 2, lengths equal to the row and just below it included),
row strides (tight or padded), layouts and parameters, all inside what the headers allow.  Each call must
succeed: any load or store outside the caller's tensors as their descriptors describe them, the per-sample
tensors, the workspace or the handle's tables would make the checked library return an error status with
the offending site.  Runs only against that library (RPPB_LIBRARY=checked, started by
tests/test_gpu_checked.py); the parity suites check the values.
"""
import os

import numpy as np
import pytest
import torch

from rpp_b200 import audio, lib
from rpp_b200.types import (RppStatus, RpptDataType, RpptLayout, audio_desc, frontend_params, generic_desc,
                            spectra_desc)
from rpp_b200.windows import kaiser_sinc
from gpu_util import dev

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("RPPB_LIBRARY") != "checked",
                                 reason="runs against librppb_checked.so (tests/test_gpu_checked.py)")]

SEEDS = range(40)
OK = RppStatus.RPP_SUCCESS


def lengths(r, n, L):
    """n lengths in [0, L] with the edge values mixed in; the first fills the row."""
    special = [0, 1, 2, 3, L - 1, L]
    v = r.integers(0, L + 1, n)
    for i in range(1, n):
        if r.random() < 0.4:
            v[i] = special[int(r.integers(0, len(special)))]
    v[0] = L
    return np.clip(v, 0, L).astype(np.int32)


def signal(r, n, width):
    return dev(r.uniform(-0.5, 0.5, (n, width)).astype(np.float32))


def case(r):
    n = int(r.integers(1, 7))
    L = int(r.integers(1, 6000))
    pad = int(r.choice([0, 0, 1, 3, 8]))
    return n, L, pad


def run(st, tile_limit=False):
    """tile_limit: a call whose frame tile does not fit a CTA's shared memory may return the documented
    RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE (large nfft with a long window and step, many filters)."""
    if tile_limit and st == RppStatus.RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE:
        return False
    assert st == OK, (st, lib.last_error())
    return True


@pytest.mark.parametrize("seed", SEEDS)
def test_pre_emphasis_down_mixing_pcm(gpu, seed):
    r = np.random.Generator(np.random.PCG64(1000 + seed))
    n, L, pad = case(r)
    lens = lengths(r, n, L)
    x = signal(r, n, L + pad)
    run(audio.pre_emphasis_filter(x, audio_desc(n, L + pad), torch.zeros((n, L + pad), device="cuda"),
                                  audio_desc(n, L + pad), dev(lens), dev(r.uniform(0, 1, n).astype(np.float32)),
                                  int(r.integers(0, 3)), gpu))
    C = int(r.integers(1, 6))
    xc = signal(r, n, (L + pad) * C)
    dims = np.stack([lens, np.full(n, C, np.int32)], 1).astype(np.int32)
    run(audio.down_mixing(xc, audio_desc(n, L + pad, channels=C, num_dims=3), torch.zeros((n, L + pad), device="cuda"),
                          audio_desc(n, L + pad), dev(dims), bool(r.integers(0, 2)), gpu))
    pcm = dev(r.integers(-32768, 32768, (n, (L + pad) * C)).astype(np.int16))
    sd = audio_desc(n, L + pad, channels=C)
    sd.dataType = RpptDataType.I16
    run(audio.pcm16_to_f32(pcm, sd, torch.zeros((n, (L + pad) * C), device="cuda"), audio_desc(n, L + pad, channels=C),
                           dev(lens), gpu))


@pytest.mark.parametrize("seed", SEEDS)
def test_resample(gpu, seed):
    r = np.random.Generator(np.random.PCG64(2000 + seed))
    n, L, pad = case(r)
    lens = lengths(r, n, L)
    rates_in = r.choice(np.array([8000, 16000, 22050, 44100, 48000], np.float32), n)
    rate_out = np.float32(r.choice([8000.0, 16000.0, 44100.0]))
    out = int(max(int(np.ceil(np.float32(np.float32(L) * rate_out) / ri)) for ri in rates_in)) + int(r.integers(0, 3))
    lut, scale, center, lobes = kaiser_sinc(int(r.choice([4, 8, 16])))
    lut_d = dev(lut)
    win = audio.resampling_window(lut_d, scale, center, lobes)
    C = int(r.integers(1, 3))
    x = signal(r, n, (L + pad) * C)
    dims = np.stack([lens, np.full(n, C, np.int32)], 1).astype(np.int32)
    run(audio.resample(x, audio_desc(n, L + pad, channels=C), torch.zeros((n, out * C), device="cuda"),
                       audio_desc(n, out, channels=C), dev(rates_in), dev(np.full(n, rate_out, np.float32)), dev(dims),
                       win, gpu))
    run(audio.downmix_resample(x, audio_desc(n, L + pad, channels=C, num_dims=3), torch.zeros((n, out), device="cuda"),
                               audio_desc(n, out), dev(rates_in), dev(np.full(n, rate_out, np.float32)), dev(dims),
                               bool(r.integers(0, 2)), lut_d, scale, center, lobes, gpu))


def frames(L, W, hop, center):
    """Frames of a clip as the library counts them (C integer division, truncating toward zero)."""
    Lw = L if center else L - W
    q = Lw // hop if Lw >= 0 else -((-Lw) // hop)
    return max(0, q + 1)


@pytest.mark.parametrize("seed", SEEDS)
def test_spectrogram_mel_decibels(gpu, seed):
    r = np.random.Generator(np.random.PCG64(3000 + seed))
    n, L, pad = case(r)
    nfft = int(r.choice([128, 256, 512, 1024, 2048]))
    W = int(r.integers(max(8, nfft // 4), nfft + 1))
    hop = int(r.integers(max(1, W // 4), W + 1))
    center, reflect = bool(r.integers(0, 2)), bool(r.integers(0, 2))
    L = max(L, W)
    lens = lengths(r, n, L)
    F = [frames(int(l), W, hop, center) for l in lens]
    mf = max(max(F), 1)
    bins = nfft // 2 + 1
    nft = bool(r.integers(0, 2))
    layout = RpptLayout.NFT if nft else RpptLayout.NTF
    spec = torch.zeros((n, bins, mf) if nft else (n, mf, bins), device="cuda")
    dd = spectra_desc(n, bins, mf, layout) if nft else spectra_desc(n, mf, bins, layout)
    if not run(audio.spectrogram(signal(r, n, L + pad), audio_desc(n, L + pad), spec, dd, dev(lens), center, reflect,
                                 None, nfft, int(r.integers(1, 3)), W, hop, gpu), tile_limit=True):
        return
    if not nft:
        return
    nmel = int(min(r.choice([16, 40, 80, 128]), bins - 1))
    fmax = float(r.choice([0.0, 4000.0, 8000.0]))
    dims = np.stack([np.full(n, bins, np.int32), np.array(F, np.int32)], 1).astype(np.int32)
    mel = torch.zeros((n, nmel, mf), device="cuda")
    run(audio.mel_filter_bank(spec.abs() + 1e-6, spectra_desc(n, bins, mf), mel, spectra_desc(n, nmel, mf), dev(dims),
                              fmax if fmax else 8000.0, float(r.choice([0.0, 20.0])), int(r.integers(0, 2)), nmel,
                              16000.0, bool(r.integers(0, 2)), gpu), tile_limit=True)
    patches = audio.image_patches(F, [nmel] * n)
    run(audio.to_decibels(mel.abs() + 1e-6, spectra_desc(n, nmel, mf), torch.zeros((n, nmel, mf), device="cuda"),
                          spectra_desc(n, nmel, mf), patches, -80.0, 10.0, float(r.choice([0.0, 1.0])), gpu))


@pytest.mark.parametrize("seed", SEEDS)
def test_frontend(gpu, seed):
    r = np.random.Generator(np.random.PCG64(4000 + seed))
    n, L, pad = case(r)
    engine = int(r.integers(0, 2))
    nfft = 512 if engine else int(r.choice([128, 256, 512, 1024, 2048]))
    W = int(r.integers(max(8, nfft // 4), nfft + 1))
    hop = int(r.integers(max(1, W // 4), W + 1))
    center = bool(r.integers(0, 2))
    L = max(L, W)
    lens = lengths(r, n, L)
    mf = max(1, max(frames(int(l), W, hop, center) for l in lens))
    nmel = int(min(r.choice([16, 40, 80, 128]), nfft // 2))
    p = frontend_params(nfft=nfft, window_length=W, window_step=hop, num_filter=nmel, center=center,
                        reflect=bool(r.integers(0, 2)), border=int(r.integers(0, 3)), engine=engine,
                        lookahead=int(r.choice([0, 1, 8])), db_frames=int(r.choice([0, 16, 64])))
    x = signal(r, n, L + pad)
    coeff = dev(r.uniform(0.5, 0.99, n).astype(np.float32))
    fits = run(audio.frontend(x, audio_desc(n, L + pad), torch.zeros((n, nmel, mf), device="cuda"),
                              spectra_desc(n, nmel, mf), dev(lens), coeff, p, gpu), tile_limit=True)
    if fits and engine == 0 and seed % 4 == 0:
        xh = torch.from_numpy(r.uniform(-0.5, 0.5, (n, L + pad)).astype(np.float32)).pin_memory()
        out = torch.zeros((n, nmel, mf)).pin_memory()
        run(audio.frontend_host(xh, audio_desc(n, L + pad), out, spectra_desc(n, nmel, mf), lens,
                                r.uniform(0.5, 0.99, n).astype(np.float32), p, int(r.choice([0, 1, 3])), gpu))


@pytest.mark.parametrize("seed", SEEDS)
def test_nsr(gpu, seed):
    r = np.random.Generator(np.random.PCG64(5000 + seed))
    n, L, pad = case(r)
    L = L * 4
    lens = lengths(r, n, L)
    x = signal(r, n, L + pad)
    begin = torch.zeros(n, dtype=torch.int32, device="cuda")
    length = torch.zeros(n, dtype=torch.int32, device="cuda")
    run(audio.non_silent_region_detection(x, audio_desc(n, L + pad), dev(lens), begin, length,
                                          float(r.choice([-60.0, -20.0])), int(r.choice([16, 512, 2048])),
                                          float(r.choice([0.0, 0.5])), int(r.choice([-1, 1000, 8192])), gpu))


@pytest.mark.parametrize("seed", SEEDS)
def test_slice_normalize(gpu, seed):
    r = np.random.Generator(np.random.PCG64(6000 + seed))
    n = int(r.integers(1, 7))
    num_dims = int(r.integers(1, 3))
    shp = (n, int(r.integers(1, 4000))) if num_dims == 1 else (n, int(r.integers(1, 40)), int(r.integers(1, 90)))
    ext = np.array(shp[1:])
    length = np.stack([r.integers(0, e + 1, n) for e in ext], 1).astype(np.int32)
    anchor = np.stack([r.integers(0, e + 1, n) for e in ext], 1).astype(np.int32)
    shape = np.stack([r.integers(1, e + 1, n) for e in ext], 1).astype(np.int32)
    roi = np.concatenate([np.zeros_like(length), length], 1).astype(np.uint32).ravel()
    d = generic_desc(shp)
    x = dev(r.standard_normal(shp).astype(np.float32))
    run(audio.slice(x, d, torch.zeros(shp, device="cuda"), d, anchor.ravel(), shape.ravel(),
                    np.array([1.5], np.float32), bool(r.integers(0, 2)), roi, gpu))
    if num_dims == 2:
        R, Cc = shp[1], shp[2]
        mask = int(r.integers(1, 4))
        rl = np.stack([np.zeros(n), np.zeros(n), r.integers(1, R + 1, n), r.integers(1, Cc + 1, n)], 1)
        roi2 = rl.astype(np.uint32).ravel()
        size = max(int(np.prod([1 if mask & (1 << i) else rl[b, 2 + i] for i in range(2)])) for b in range(n))
        mean = torch.zeros(n * size, device="cuda")
        std = torch.ones(n * size, device="cuda")
        run(audio.normalize(x, d, torch.zeros(shp, device="cuda"), d, mask, mean, std, int(r.integers(0, 4)), 1.0, 0.0,
                            roi2, gpu))
