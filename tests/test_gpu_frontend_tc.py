"""The fused front end with the tensor-core spectrum engine (RPPB_ENGINE_TENSOR_CORE_F16X3): the
512-point DFT factored into two F16 hi/lo x3 GEMM stages on tcgen05 (each frame scaled by a power of
two), inside the same persistent launch as the mel and decibel steps.

Its mel power is checked against the FP64 oracle chain (pre-emphasis -> spectrogram -> mel in double
precision): at most 1e-4 of each frame's largest mel value, the bound of the precision target.  The
decibel output is read back as mel power by running with referenceMagnitude 1 and a cutoff of -200 dB,
so y = 10 log10(mel) is inverted exactly enough (~1e-6 relative) for the check.  The engine's results
do not depend on the schedule (tile frames, decibel frames, lookahead, CTAs per SM), bit for bit."""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, synth
from rpp_b200.types import (ENGINE_TENSOR_CORE_F16X3, RppStatus, audio_desc, frontend_params, spectra_desc)
from gpu_util import canvas, dev, host

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS
MEL_BAR = 1e-4   # mel power error / frame maximum, against FP64


def run_tc(h, x, lens, coeff, p, maxf):
    n, L = x.shape
    out = canvas((n, p.numFilter, maxf))
    st = audio.frontend(dev(x), audio_desc(n, L), out, spectra_desc(n, p.numFilter, maxf), dev(lens), dev(coeff), p, h)
    assert st == OK, st
    assert audio.device_error(h) == 0
    return host(out)


def frames(lens, p):
    """Frames per clip as the reference counts them (C integer division, truncating toward zero)."""
    out = []
    for l in lens:
        v = int(l) - (0 if p.centerWindows else p.windowLength)
        q = abs(v) // p.windowStep
        out.append(max(0, (q if v >= 0 else -q) + 1))
    return out


def mel64(oracle, x, lens, coeff, p, maxf, window=None):
    spec = oracle.spectrogram_f64(x, lens, int(p.centerWindows), int(p.reflectPadding), window, p.nfft, p.power,
                                  p.windowLength, p.windowStep, 1, max_frames=maxf, preemph_coeff=coeff,
                                  border=p.borderType)
    F = frames(lens, p)
    dims = np.stack([np.full(len(lens), p.nfft // 2 + 1, np.int32), np.minimum(F, maxf)], 1).astype(np.int32).ravel()
    return oracle.mel_filter_bank_f64(spec, dims, p.maxFreq, p.minFreq, p.melFormula, p.numFilter, p.sampleRate,
                                      int(p.normalize))


def mel_error(db, m64, lens, p, maxf):
    """max |mel - mel64| / the frame's largest mel64.  Values at the -200 dB floor read as 0, and frames
    more than 120 dB below their clip's loudest (silent gaps, empty clips) are scaled by that level
    instead of their own maximum."""
    worst = 0.0
    for i, f in enumerate(frames(lens, p)):
        f = min(f, maxf)
        if f == 0:
            continue
        got = 10.0 ** (db[i, :, :f].astype(np.float64) / 10.0)
        got[got <= 1.0001e-20] = 0.0
        exp = m64[i, :, :f]
        scale = np.maximum(exp.max(axis=0, keepdims=True), max(1e-12 * exp.max(), 1e-30))
        worst = max(worst, float((np.abs(got - exp) / scale).max()))
    return worst


CASES = [
    dict(),
    dict(window_length=320, num_filter=80, border=1),
    dict(window_length=512, window_step=128, num_filter=64, mel_formula=1, normalize=False, border=2),
    dict(window_step=100, center=False, reflect=False),
    dict(power=1, num_filter=40, max_freq=6000.0, min_freq=100.0),
    dict(window_length=256, window_step=51),
]


@pytest.mark.parametrize("kw", CASES)
def test_tc_engine_mel_power_vs_fp64(gpu, oracle, kw):
    r = np.random.Generator(np.random.PCG64(17))
    lens = r.integers(1, 48000, 10)
    lens[0], lens[1], lens[2], lens[3], lens[4] = 48000, 1, 2, 399, 0
    x, lens = synth.mono_batch(len(lens), lens.astype(np.int32), r, gaps=True)
    coeff = r.uniform(0.9, 0.99, len(lens)).astype(np.float32)
    p = frontend_params(engine=ENGINE_TENSOR_CORE_F16X3, cut_off_db=-200.0, reference_magnitude=1.0, **kw)
    maxf = 48000 // p.windowStep + 1
    db = run_tc(gpu, x, lens, coeff, p, maxf)
    err = mel_error(db, mel64(oracle, x, lens, coeff, p, maxf), lens, p, maxf)
    assert err <= MEL_BAR, err
    # nothing outside each clip's valid frames and filters is written
    for i, f in enumerate(frames(lens, p)):
        assert (db[i, :, min(f, maxf):] == -12345.0).all()


def test_tc_engine_benchmark_clips_vs_fp64(gpu, oracle):
    """The benchmark's signal model at full length (clips up to 16 s, silent gaps), default parameters."""
    x, lens = synth.gapped_clips(n=256)
    idx = np.argsort(lens)[[0, 100, 200, 253, 254, 255]]
    x = np.ascontiguousarray(x[idx, :int(lens[idx].max())])
    lens = np.ascontiguousarray(lens[idx])
    coeff = np.full(len(lens), 0.97, np.float32)
    p = frontend_params(engine=ENGINE_TENSOR_CORE_F16X3, cut_off_db=-200.0, reference_magnitude=1.0)
    maxf = int(lens.max()) // 160 + 1
    db = run_tc(gpu, x, lens, coeff, p, maxf)
    err = mel_error(db, mel64(oracle, x, lens, coeff, p, maxf), lens, p, maxf)
    assert err <= MEL_BAR, err


def test_tc_engine_decibels_close_to_fp32_engine(gpu):
    """With the benchmark's decibel parameters (-80 dB, per-clip maximum) the two engines agree to the
    spectrum's precision where the mel power is within 60 dB of its frame maximum."""
    x, lens = synth.gapped_clips(n=12, max_len=64000)
    n = len(lens)
    coeff = np.full(n, 0.97, np.float32)
    maxf = 64000 // 160 + 1
    a = run_tc(gpu, x, lens, coeff, frontend_params(), maxf)
    b = run_tc(gpu, x, lens, coeff, frontend_params(engine=ENGINE_TENSOR_CORE_F16X3), maxf)
    for i in range(n):
        f = int(lens[i]) // 160 + 1
        ai, bi = a[i, :, :f], b[i, :, :f]
        near = ai >= ai.max(axis=0, keepdims=True) - 60.0
        assert np.abs(ai - bi)[near].max() < 2e-3
        assert (b[i, :, f:] == -12345.0).all()


@pytest.mark.parametrize("sched", [dict(tile_frames=16), dict(tile_frames=64, db_frames=32), dict(lookahead=1),
                                   dict(ctas_per_sm=1, lookahead=96, db_frames=64)])
def test_tc_engine_schedule_independent(gpu, sched):
    x, lens = synth.gapped_clips(n=20, max_len=80000)
    n = len(lens)
    coeff = np.full(n, 0.97, np.float32)
    maxf = 80000 // 160 + 1
    base = run_tc(gpu, x, lens, coeff, frontend_params(engine=ENGINE_TENSOR_CORE_F16X3), maxf)
    other = run_tc(gpu, x, lens, coeff, frontend_params(engine=ENGINE_TENSOR_CORE_F16X3, **sched), maxf)
    np.testing.assert_array_equal(other, base)


def test_tc_engine_graph_capture(gpu):
    x, lens = synth.gapped_clips(n=16, max_len=48000)
    n, L = x.shape
    p = frontend_params(engine=ENGINE_TENSOR_CORE_F16X3)
    mf = 48000 // 160 + 1
    xd, ld, cd = dev(x), dev(lens), dev(np.full(n, 0.97, np.float32))
    out = canvas((n, 128, mf))
    sd, dd = audio_desc(n, L), spectra_desc(n, 128, mf)
    assert audio.frontend(xd, sd, out, dd, ld, cd, p, gpu) == OK
    first = host(out).copy()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    gpu.set_stream(s.cuda_stream)
    try:
        with torch.cuda.stream(s):
            out.fill_(-12345.0)
            torch.cuda.synchronize()
            with torch.cuda.graph(g, stream=s):
                assert audio.frontend(xd, sd, out, dd, ld, cd, p, gpu) == OK
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(host(out), first)
    finally:
        gpu.set_stream(torch.cuda.current_stream().cuda_stream)
        del g
    assert audio.device_error(gpu) == 0


def test_tc_engine_rejects_unsupported_shapes(gpu):
    x = dev(np.zeros((2, 4000), np.float32))
    lens = dev(np.array([4000, 100], np.int32))
    coeff = dev(np.full(2, 0.97, np.float32))
    for kw in (dict(nfft=1024, window_length=1024), dict(nfft=256, window_length=256), dict(tile_frames=48),
               dict(engine=2)):
        kw.setdefault("engine", ENGINE_TENSOR_CORE_F16X3)
        p = frontend_params(**kw)
        out = canvas((2, 128, 64))
        st = audio.frontend(x, audio_desc(2, 4000), out, spectra_desc(2, 128, 64), lens, coeff, p, gpu)
        assert st in (RppStatus.RPP_ERROR_NOT_IMPLEMENTED, RppStatus.RPP_ERROR_INVALID_ARGUMENTS), (kw, st)
