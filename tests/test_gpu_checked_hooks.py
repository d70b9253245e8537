"""The bounds-checked library (librppb_checked.so) catching accesses outside a call's regions.

These run only against that library (RPPB_LIBRARY=checked); tests/test_gpu_checked.py starts them in a
child process together with the parity suites.  Every entry point runs on inputs whose last sample fills
its row, so the call reads the last element of its source and writes the last element of its
destination.  rppb_check_shrink_next_tensors then registers the source (or the destination) a few bytes
short of what its descriptor says: the library must report that call's last loads (or stores) as out of
bounds, name the kernel file that made them, and skip them.  Nothing here touches memory out of bounds:
the flagged accesses lie inside the caller's buffers, and the library redirects them to its dummy.
"""
import os

import numpy as np
import pytest
import torch

from rpp_b200 import audio, lib
from rpp_b200.types import (RppStatus, RpptDataType, audio_desc, frontend_params, generic_desc, spectra_desc)
from rpp_b200.windows import kaiser_sinc
from gpu_util import dev

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("RPPB_LIBRARY") != "checked",
                                 reason="runs against librppb_checked.so (tests/test_gpu_checked.py)")]

N = 3


def rnd(shape, seed=5, lo=-0.5, hi=0.5):
    return np.random.Generator(np.random.PCG64(seed)).uniform(lo, hi, shape).astype(np.float32)


def canvas(shape):
    return torch.full(shape, -7.0, device="cuda")


def lens_full(L):
    return np.array([L // 2, 7, L], np.int32)   # the last clip fills its row


# Each case: (name, function(handle) -> status, source files that read, destination files that write,
# source shrink in bytes)
def c_preemph(h):
    L = 1000
    x = rnd((N, L))
    return audio.pre_emphasis_filter(dev(x), audio_desc(N, L), canvas((N, L)), audio_desc(N, L), dev(lens_full(L)),
                                     dev(np.full(N, 0.97, np.float32)), 0, h)


def c_downmix(h):
    L = 1000
    x = rnd((N, 2 * L))
    dims = np.stack([lens_full(L), np.full(N, 2, np.int32)], 1).astype(np.int32)
    return audio.down_mixing(dev(x), audio_desc(N, L, channels=2, num_dims=3), canvas((N, L)), audio_desc(N, L),
                             dev(dims), False, h)


def window():
    lut, scale, center, lobes = kaiser_sinc(16)
    return dev(lut), scale, center, lobes


def c_resample(h):
    L, out = 3000, 1000
    x = rnd((N, L))
    lut, scale, center, lobes = window()
    dims = np.stack([lens_full(L), np.ones(N, np.int32)], 1).astype(np.int32)
    c_resample.keep = lut
    win = audio.resampling_window(lut, scale, center, lobes)
    return audio.resample(dev(x), audio_desc(N, L), canvas((N, out)), audio_desc(N, out),
                          dev(np.full(N, 48000, np.float32)), dev(np.full(N, 16000, np.float32)), dev(dims), win, h)


def c_downmix_resample(h):
    L, out = 3000, 1000
    x = rnd((N, 2 * L))
    lut, scale, center, lobes = window()
    dims = np.stack([lens_full(L), np.full(N, 2, np.int32)], 1).astype(np.int32)
    return audio.downmix_resample(dev(x), audio_desc(N, L, channels=2, num_dims=3), canvas((N, out)),
                                  audio_desc(N, out), dev(np.full(N, 48000, np.float32)),
                                  dev(np.full(N, 16000, np.float32)), dev(dims), False, lut, scale, center, lobes, h)


L_SPEC = 4000
F_SPEC = L_SPEC // 160 + 1


def c_spectrogram(h):
    x = rnd((N, L_SPEC))
    return audio.spectrogram(dev(x), audio_desc(N, L_SPEC), canvas((N, 257, F_SPEC)), spectra_desc(N, 257, F_SPEC),
                             dev(lens_full(L_SPEC)), True, True, None, 512, 2, 400, 160, h)


def c_spectrogram_tc(h):
    x = rnd((N, L_SPEC))
    return audio.spectrogram_tc(dev(x), audio_desc(N, L_SPEC), canvas((N, 257, F_SPEC)), spectra_desc(N, 257, F_SPEC),
                                dev(lens_full(L_SPEC)), None, 0, True, True, 512, 2, 400, 160,
                                audio.TC_BF16_HILO3, h)


def c_mel(h):
    F = 30
    x = rnd((N, 257, F), lo=0.0, hi=1.0)
    dims = np.array([[257, 10], [257, 3], [257, F]], np.int32)
    return audio.mel_filter_bank(dev(x), spectra_desc(N, 257, F), canvas((N, 128, F)), spectra_desc(N, 128, F),
                                 dev(dims), 8000.0, 0.0, 0, 128, 16000.0, True, h)


def c_decibels(h):
    F = 50
    x = rnd((N, 128, F), lo=0.01, hi=1.0)
    patches = audio.image_patches([20, 3, F], [128, 128, 128])
    return audio.to_decibels(dev(x), spectra_desc(N, 128, F), canvas((N, 128, F)), spectra_desc(N, 128, F), patches,
                             -80.0, 10.0, 0.0, h)


def c_nsr(h):
    L = 20000
    x = rnd((N, L))
    begin = torch.zeros(N, dtype=torch.int32, device="cuda")
    length = torch.zeros(N, dtype=torch.int32, device="cuda")
    return audio.non_silent_region_detection(dev(x), audio_desc(N, L), dev(lens_full(L)), begin, length, -60.0, 2048,
                                             0.0, 8192, h)


def c_slice(h):
    L = 1000
    x = rnd((N, L))
    anchor = np.zeros(N, np.int32)
    shape = np.full(N, L, np.int32)
    roi = np.stack([np.zeros(N), np.full(N, L)], 1).astype(np.uint32).ravel()
    return audio.slice(dev(x), generic_desc((N, L)), canvas((N, L)), generic_desc((N, L)), anchor, shape,
                       np.zeros(1, np.float32), False, roi, h)


def c_normalize(h):
    R, C = 8, 100
    x = rnd((N, R, C))
    roi = np.tile(np.array([0, 0, R, C], np.uint32), N)
    mean = torch.zeros(N * R, device="cuda")
    std = torch.zeros(N * R, device="cuda")
    return audio.normalize(dev(x), generic_desc((N, R, C)), canvas((N, R, C)), generic_desc((N, R, C)), 2, mean, std,
                           3, 1.0, 0.0, roi, h)


def c_pcm(h):
    L = 1000
    pcm = np.random.Generator(np.random.PCG64(3)).integers(-32768, 32768, (N, L)).astype(np.int16)
    sd = audio_desc(N, L)
    sd.dataType = RpptDataType.I16
    return audio.pcm16_to_f32(dev(pcm), sd, canvas((N, L)), audio_desc(N, L), dev(lens_full(L)), h)


L_FE = 16000
F_FE = L_FE // 160 + 1


def c_frontend(h, engine=0):
    x = rnd((N, L_FE))
    return audio.frontend(dev(x), audio_desc(N, L_FE), canvas((N, 128, F_FE)), spectra_desc(N, 128, F_FE),
                          dev(lens_full(L_FE)), dev(np.full(N, 0.97, np.float32)), frontend_params(engine=engine), h)


def c_frontend_tc(h):
    return c_frontend(h, engine=1)


def c_frontend_host(h):
    x = torch.from_numpy(rnd((N, L_FE))).pin_memory()
    out = torch.full((N, 128, F_FE), -7.0).pin_memory()
    c_frontend_host.keep = (x, out)
    return audio.frontend_host(x, audio_desc(N, L_FE), out, spectra_desc(N, 128, F_FE), lens_full(L_FE),
                               np.full(N, 0.97, np.float32), frontend_params(), 0, h)


# where the loads of each entry point's source can first be flagged (common.cuh: the L2 prefetch of a span)
STFT_READ = {"stft.cuh", "common.cuh", "fused_queue.cuh", "fused.cu", "fused_tc.cu"}
CASES = [
    ("pre_emphasis", c_preemph, {"preemph.cu"}, {"preemph.cu"}, 4),
    ("down_mixing", c_downmix, {"downmix.cuh", "downmix.cu"}, {"downmix.cu"}, 4),
    ("resample", c_resample, {"resample.cu", "common.cuh"}, {"resample.cu"}, 4),
    ("downmix_resample", c_downmix_resample, {"downmix.cuh", "resample.cu", "common.cuh"}, {"resample.cu"}, 4),
    ("spectrogram", c_spectrogram, {"stft.cuh", "common.cuh"}, {"spectrogram.cu"}, 4),
    ("spectrogram_tc", c_spectrogram_tc, {"tc_dft.cu"}, {"tc_dft.cu"}, 4),
    # mel reads bins below maxFreq only: the last (Nyquist) row is not read, so cut it and one more value
    ("mel_filter_bank", c_mel, {"mel.cu"}, {"mel.cu"}, 4 * (30 + 1)),
    ("to_decibels", c_decibels, {"to_decibels.cu"}, {"to_decibels.cu"}, 4),
    ("non_silent_region_detection", c_nsr, {"nsr.cu", "common.cuh"}, {"nsr.cu"}, 4),
    ("slice", c_slice, {"slice.cu"}, {"slice.cu"}, 4),
    ("normalize", c_normalize, {"normalize.cu"}, {"normalize.cu"}, 4),
    ("pcm16_to_f32", c_pcm, {"pcm.cu"}, {"pcm.cu"}, 4),
    ("frontend", c_frontend, STFT_READ, {"fused.cu"}, 4),
    ("frontend_tensor_core", c_frontend_tc, STFT_READ, {"fused_tc.cu"}, 4),
    ("frontend_host", c_frontend_host, {"host_io.cu"}, {"host_io.cu"}, 4),
]


def site_file(msg):
    # "... outside the call's regions at <file>:<line> (<n> accesses)"
    return msg.split(" at ")[-1].split(":")[0]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_every_entry_point_reports_stray_reads_and_writes(gpu, case):
    name, call, read_files, write_files, src_shrink = case
    L = lib.load()
    assert call(gpu) == RppStatus.RPP_SUCCESS, lib.last_error()   # as described: clean
    assert L.rppb_check_shrink_next_tensors(src_shrink, 0) == 0
    st = call(gpu)
    msg = lib.last_error()
    assert st == RppStatus.RPP_ERROR_OUT_OF_BOUND_SRC_ROI, (st, msg)
    assert "read of" in msg and site_file(msg) in read_files, msg
    assert L.rppb_check_shrink_next_tensors(0, 4) == 0
    st = call(gpu)
    msg = lib.last_error()
    assert st == RppStatus.RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH, (st, msg)
    assert "write of" in msg and site_file(msg) in write_files, msg
    assert call(gpu) == RppStatus.RPP_SUCCESS, lib.last_error()   # the record was read and cleared


def test_skipped_store_leaves_the_destination(gpu, oracle):
    """The flagged stores are skipped: pre-emphasis with its destination registered a float short
    writes everything but the last vector of the last row."""
    L = 1000
    x = rnd((N, L))
    lens = lens_full(L)
    coeff = np.full(N, 0.97, np.float32)
    ref = np.full_like(x, -7.0)
    oracle.pre_emphasis(x, ref, lens, coeff, 0)
    out = canvas((N, L))
    assert lib.load().rppb_check_shrink_next_tensors(0, 4) == 0
    st = audio.pre_emphasis_filter(dev(x), audio_desc(N, L), out, audio_desc(N, L), dev(lens), dev(coeff), 0, gpu)
    assert st == RppStatus.RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH
    torch.cuda.synchronize()
    got = out.cpu().numpy().ravel()
    np.testing.assert_array_equal(got[:-4], ref.ravel()[:-4])
    assert (got[-4:] == -7.0).all()


def test_read_past_the_described_source(gpu):
    """A source described shorter than its lengths (the last clip 64 samples past its row) over a buffer
    256 floats longer: the loads past the described tensor are reported and read the dummy instead."""
    L = 1000
    x = rnd((N, L))
    lens = lens_full(L)
    lens[-1] = L + 64
    buf = torch.zeros(N * L + 256, device="cuda")
    buf[: N * L] = torch.from_numpy(x.ravel()).cuda()
    dst = torch.full((N, L + 128), -7.0, device="cuda")
    st = audio.pre_emphasis_filter(buf, audio_desc(N, L), dst, audio_desc(N, L + 128), dev(lens),
                                   dev(np.full(N, 0.97, np.float32)), 0, gpu)
    assert st == RppStatus.RPP_ERROR_OUT_OF_BOUND_SRC_ROI, st
    msg = lib.last_error()
    assert "read of" in msg and site_file(msg) == "preemph.cu", msg
