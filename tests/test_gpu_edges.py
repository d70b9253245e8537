"""Edge cases across the entry points: empty batches, and the full 256-clip batch checked through
properties that hold at any size (fused == plain chain bit for bit; decibels within [cutoff, 0]
with ~0 dB reached at each clip's maximum)."""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, synth
from rpp_b200.types import RppStatus, audio_desc, spectra_desc, frontend_params, generic_desc
from rpp_b200.windows import kaiser_sinc
from gpu_util import dev, canvas

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS


def test_empty_batch_every_entry_point(gpu):
    """n = 0: every call succeeds and writes nothing."""
    one_i = dev(np.zeros(2, np.int32))
    one_f = dev(np.ones(2, np.float32))
    buf = canvas((1, 64))
    d0 = audio_desc(0, 64)
    s0 = spectra_desc(0, 4, 16)
    sp = canvas((1, 4, 16))
    assert audio.pre_emphasis_filter(buf, d0, buf, d0, one_i, one_f, 0, gpu) == OK
    assert audio.down_mixing(buf, audio_desc(0, 32, channels=2, num_dims=3), buf, audio_desc(0, 32), one_i, False,
                             gpu) == OK
    lut, scale, center, lobes = kaiser_sinc(16, beta=8.0)
    win = audio.resampling_window(dev(lut), scale, center, lobes)
    assert audio.resample(buf, d0, buf, d0, one_f, one_f, one_i, win, gpu) == OK
    assert audio.spectrogram(buf, d0, sp, s0, one_i, True, True, None, 8, 2, 8, 4, gpu) == OK
    assert audio.mel_filter_bank(sp, s0, sp, s0, one_i, 8000.0, 0.0, 0, 4, 16000.0, True, gpu) == OK
    assert audio.to_decibels(sp, s0, sp, s0, one_i, -80.0, 10.0, 0.0, gpu) == OK
    assert audio.non_silent_region_detection(buf, d0, one_i, one_i, one_i, -60.0, 8, 0.0, 16, gpu) == OK
    assert audio.frontend(buf, d0, sp, s0, one_i, one_f, frontend_params(nfft=8, window_length=8, window_step=4,
                                                                          num_filter=4), gpu) == OK
    g0 = generic_desc((0, 64))
    roi = dev(np.zeros(4, np.int32))
    assert audio.slice(buf, g0, buf, g0, one_i, one_i, one_f, True, roi, gpu) == OK
    torch.cuda.synchronize()
    assert (buf == -12345.0).all() and (sp == -12345.0).all()
    assert audio.device_error(gpu) == 0


@pytest.fixture(scope="module")
def full_batch():
    x, lens = synth.gapped_clips(n=256)
    return x, lens


def test_full_size_fused_equals_plain(gpu, full_batch):
    """The 256-clip batch at full size (1-16 s): the fused call and the four plain calls give the same
    bits over every valid decibel, compared on the device."""
    x, lens = full_batch
    n, L = x.shape
    p = frontend_params()
    F = (lens // p.windowStep + 1).astype(np.int32)
    mf = int(F.max())
    xd, ld, cd = dev(x), dev(lens), dev(np.full(n, 0.97, np.float32))
    d = audio_desc(n, L)
    fused = torch.full((n, 128, mf), -12345.0, device="cuda")
    assert audio.frontend(xd, d, fused, spectra_desc(n, 128, mf), ld, cd, p, gpu) == OK
    pre = torch.zeros_like(xd)
    assert audio.pre_emphasis_filter(xd, d, pre, d, ld, cd, 0, gpu) == OK
    spec = torch.zeros((n, 257, mf), device="cuda")
    assert audio.spectrogram(pre, d, spec, spectra_desc(n, 257, mf), ld, True, True, None, 512, 2, 400, 160,
                             gpu) == OK
    dims = dev(np.stack([np.full(n, 257, np.int32), F], 1).astype(np.int32))
    mel = torch.zeros((n, 128, mf), device="cuda")
    assert audio.mel_filter_bank(spec, spectra_desc(n, 257, mf), mel, spectra_desc(n, 128, mf), dims, 8000.0, 0.0, 0,
                                 128, 16000.0, True, gpu) == OK
    del spec
    db = torch.full((n, 128, mf), -12345.0, device="cuda")
    patches = dev(np.stack([F, np.full(n, 128, np.int32)], 1).astype(np.int32))
    assert audio.to_decibels(mel, spectra_desc(n, 128, mf), db, spectra_desc(n, 128, mf), patches, -80.0, 10.0, 0.0,
                             gpu) == OK
    torch.cuda.synchronize()
    frames = torch.arange(mf, device="cuda")[None, None, :]
    valid = frames < torch.from_numpy(F).cuda()[:, None, None]
    assert torch.equal(fused[valid.expand_as(fused)], db[valid.expand_as(db)])
    assert (fused[~valid.expand_as(fused)] == -12345.0).all()
    assert audio.device_error(gpu) == 0


def test_full_size_decibel_range(gpu, full_batch):
    """Per clip the decibels lie in [cutoff, 0] up to rounding and reach 0 dB at the clip maximum: x * (1/ref)
    with a rounded reciprocal is within an ulp of 1 there, so within 1e-5 dB."""
    x, lens = full_batch
    n, L = x.shape
    p = frontend_params()
    F = (lens // p.windowStep + 1).astype(np.int32)
    mf = int(F.max())
    out = torch.full((n, 128, mf), -12345.0, device="cuda")
    assert audio.frontend(dev(x), audio_desc(n, L), out, spectra_desc(n, 128, mf), dev(lens),
                          dev(np.full(n, 0.97, np.float32)), p, gpu) == OK
    torch.cuda.synchronize()
    for b in range(0, n, 17):
        v = out[b, :, :F[b]]
        assert abs(float(v.max())) <= 1e-5
        assert float(v.min()) >= -80.0 - 1e-3


def test_frame_tile_too_large_for_shared_memory(gpu):
    """nfft 2048 with a 1512-sample window every 1031 samples: the frame tile and its span do not fit a CTA's
    shared memory, and the call says so with the documented status instead of failing to launch."""
    n, L = 2, 6000
    x = torch.zeros((n, L), device="cuda")
    lens = torch.full((n,), L, dtype=torch.int32, device="cuda")
    F = L // 1031 + 1
    out = torch.zeros((n, 1025, F), device="cuda")
    st = audio.spectrogram(x, audio_desc(n, L), out, spectra_desc(n, 1025, F), lens, True, True, None, 2048, 2, 1512,
                           1031, gpu)
    assert st == RppStatus.RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, st
