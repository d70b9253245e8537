"""The tensor-core spectrogram (rppb_spectrogram_tc_gpu, tcgen05 DFT-GEMM) against the FP64 oracle.
Bounds are per-frame relative (error / the frame's largest bin) and follow the operand precision:
BF16 keeps 8 significant bits, the hi/lo split (hi*hi + hi*lo + lo*hi) about 16, TF32 11, E4M3 4."""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, synth
from rpp_b200.types import RppStatus, RpptLayout, audio_desc, spectra_desc
from gpu_util import dev, host, canvas, frame_rel_err

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS
BOUND = {audio.TC_BF16: 2e-2, audio.TC_BF16_HILO3: 5e-5, audio.TC_TF32: 5e-3, audio.TC_FP8_E4M3: 0.25}
PRECISIONS = [audio.TC_BF16, audio.TC_BF16_HILO3, audio.TC_TF32, audio.TC_FP8_E4M3]

CASES = [
    dict(nfft=512, W=400, hop=160, center=True, reflect=True, power=2, nft=True, preemph=True),
    dict(nfft=1024, W=1024, hop=256, center=True, reflect=True, power=2, nft=False, preemph=False),
    dict(nfft=256, W=200, hop=64, center=False, reflect=False, power=1, nft=True, preemph=True, border=1),
    dict(nfft=512, W=512, hop=128, center=True, reflect=False, power=2, nft=True, preemph=False),
]


def run_tc(h, x, lens, coeff, c, precision, maxf):
    n, L = x.shape
    bins = c["nfft"] // 2 + 1
    shape = (n, bins, maxf) if c["nft"] else (n, maxf, bins)
    out = canvas(shape)
    dd = spectra_desc(n, bins, maxf) if c["nft"] else spectra_desc(n, maxf, bins, layout=RpptLayout.NTF)
    st = audio.spectrogram_tc(dev(x), audio_desc(n, L), out, dd, dev(lens), dev(coeff) if c["preemph"] else None,
                              c.get("border", 0), c["center"], c["reflect"], c["nfft"], c["power"], c["W"], c["hop"],
                              precision, h)
    assert st == OK
    return host(out)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_tc_spectrogram_vs_fp64(gpu, oracle, ci, precision):
    c = CASES[ci]
    r = np.random.Generator(np.random.PCG64(7 + ci))
    lens = r.integers(1, 40000, 9).astype(np.int32)
    lens[0], lens[1], lens[2] = 40000, 1, c["W"] + 3
    x, lens = synth.mono_batch(len(lens), lens, r, gaps=True)
    n = x.shape[0]
    coeff = r.uniform(0.9, 0.99, n).astype(np.float32)
    F = np.array([max(0, oracle.num_windows(l, c["W"], c["hop"], c["center"])) for l in lens])
    maxf = int(F.max())
    got = run_tc(gpu, x, lens, coeff, c, precision, maxf)
    exp = oracle.spectrogram_f64(x, lens, c["center"], c["reflect"], None, c["nfft"], c["power"], c["W"], c["hop"],
                                 c["nft"], max_frames=maxf, preemph_coeff=coeff if c["preemph"] else None,
                                 border=c.get("border", 0))
    for i in range(n):
        f = F[i]
        if c["nft"]:
            g, e = got[i, :, :f], exp[i, :, :f]
            assert (got[i, :, f:] == -12345.0).all()
            err = frame_rel_err(g, e, axis=0)
        else:
            g, e = got[i, :f, :], exp[i, :f, :]
            assert (got[i, f:, :] == -12345.0).all()
            err = frame_rel_err(g, e, axis=1)
        assert err < BOUND[precision], (i, f, err)
    assert audio.device_error(gpu) == 0


def test_tc_spectrogram_many_tiles(gpu, oracle):
    """Clips long enough for several 128-frame tiles per clip and more work items than SMs."""
    x, lens = synth.gapped_clips(n=24, max_len=160000)
    n, L = x.shape
    coeff = np.full(n, 0.97, np.float32)
    c = dict(CASES[0])
    F = lens // 160 + 1
    maxf = int(F.max())
    got = run_tc(gpu, x, lens, coeff, c, audio.TC_BF16_HILO3, maxf)
    exp = oracle.spectrogram_f64(x, lens, 1, 1, None, 512, 2, 400, 160, 1, max_frames=maxf, preemph_coeff=coeff)
    for i in range(n):
        assert frame_rel_err(got[i, :, :F[i]], exp[i, :, :F[i]]) < BOUND[audio.TC_BF16_HILO3]


@pytest.mark.parametrize("precision", [audio.TC_BF16, audio.TC_BF16_HILO3, audio.TC_TF32])
@pytest.mark.parametrize("ci", [0, 3])
def test_tc_spectrogram_materialized_frames_same_bits(gpu, ci, precision):
    """Frames written out as [frame][kPad] rows (the form taken when the driver refuses an
    overlapping-row tensor map) give the same bits as frames read in place: the padding columns
    meet zero basis entries either way, and the MMAs run in the same order."""
    c = CASES[ci]
    r = np.random.Generator(np.random.PCG64(101 + ci))
    lens = r.integers(1, 60000, 7).astype(np.int32)
    lens[0], lens[1] = 60000, c["W"] + 1
    x, lens = synth.mono_batch(len(lens), lens, r, gaps=True)
    coeff = r.uniform(0.9, 0.99, len(lens)).astype(np.float32)
    maxf = int(60000 // c["hop"]) + 1
    inplace = run_tc(gpu, x, lens, coeff, c, precision, maxf)
    assert audio.set_tc_materialized_frames(gpu, True) == OK
    try:
        rows = run_tc(gpu, x, lens, coeff, c, precision, maxf)
    finally:
        assert audio.set_tc_materialized_frames(gpu, False) == OK
    np.testing.assert_array_equal(rows, inplace)
    assert audio.device_error(gpu) == 0


def test_tc_spectrogram_rejects(gpu):
    x = np.zeros((2, 4000), np.float32)
    lens = np.array([4000, 4000], np.int32)
    out = canvas((2, 257, 30))
    args = lambda nfft, hop, prec: (dev(x), audio_desc(2, 4000), out, spectra_desc(2, 257, 30), dev(lens), None, 0,
                                    True, True, nfft, 2, 400, hop, prec, gpu)
    NI = RppStatus.RPP_ERROR_NOT_IMPLEMENTED
    assert audio.spectrogram_tc(*args(512, 150, audio.TC_BF16_HILO3)) == NI   # hop % 8 (BF16 rows in place)
    assert audio.spectrogram_tc(*args(512, 150, audio.TC_TF32)) == NI         # hop % 4
    assert audio.spectrogram_tc(*args(400, 160, audio.TC_BF16)) == NI         # nfft % 256
    assert audio.spectrogram_tc(*args(512, 160, 4)) == NI                     # unknown precision
    assert audio.spectrogram_tc(*args(1024, 160, audio.TC_TF32)) == RppStatus.RPP_ERROR_INVALID_DST_DIMS  # 513 bins
    assert audio.spectrogram_tc(*args(512, 150, audio.TC_FP8_E4M3)) == OK     # FP8 frames are materialized


MEL_BOUND = {audio.TC_BF16: 1e-2, audio.TC_BF16_HILO3: 5e-5, audio.TC_TF32: 3e-3, audio.TC_FP8_E4M3: 0.25}


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("nmel,htk,normalize", [(128, 0, True), (80, 1, False), (256, 0, True)])
def test_tc_mel_vs_fp32(gpu, precision, nmel, htk, normalize):
    """rppb_mel_filter_bank_tc_gpu against the FP32 mel_filter_bank (bit-exact to the reference) on
    the same spectrum: per-frame relative error within the operand precision's bound; only the
    valid frames are written."""
    x, lens = synth.gapped_clips(n=10, max_len=80000)
    n, L = x.shape
    F = (lens // 160 + 1).astype(np.int32)
    mf = int(F.max())
    xd, ld = dev(x), dev(lens)
    spec = torch.zeros((n, 257, mf), device="cuda")
    sd, spd = audio_desc(n, L), spectra_desc(n, 257, mf)
    assert audio.spectrogram(xd, sd, spec, spd, ld, True, True, None, 512, 2, 400, 160, gpu) == OK
    dims = dev(np.stack([np.full(n, 257, np.int32), F], 1).astype(np.int32))
    md = spectra_desc(n, nmel, mf)
    ref = torch.zeros((n, nmel, mf), device="cuda")
    assert audio.mel_filter_bank(spec, spd, ref, md, dims, 8000.0, 0.0, htk, nmel, 16000.0, normalize, gpu) == OK
    out = canvas((n, nmel, mf))
    assert audio.mel_filter_bank_tc(spec, spd, out, md, dims, 8000.0, 0.0, htk, nmel, 16000.0, normalize, precision,
                                    gpu) == OK
    r, o = host(ref), host(out)
    for i in range(n):
        assert (o[i, :, F[i]:] == -12345.0).all()
        assert frame_rel_err(o[i, :, :F[i]], r[i, :, :F[i]]) < MEL_BOUND[precision]
    assert audio.device_error(gpu) == 0
