"""The fused front end (rppb_frontend_gpu) against the plain four-call chain through the same
C ABI — bit-identical by construction — and against the FP64 oracle chain."""
import numpy as np
import pytest
import torch

from rpp_b200 import audio, synth
from rpp_b200.types import RppStatus, audio_desc, spectra_desc, frontend_params
from gpu_util import dev, host, canvas, frame_rel_err

pytestmark = pytest.mark.gpu
OK = RppStatus.RPP_SUCCESS


def plain_chain(h, x, lens, coeff, p, maxf):
    n, L = x.shape
    bins = p.nfft // 2 + 1
    d = audio_desc(n, L)
    xd, ld, cd = dev(x), dev(lens), dev(coeff)
    pre = torch.zeros_like(xd)
    assert audio.pre_emphasis_filter(xd, d, pre, d, ld, cd, p.borderType, h) == OK
    spec = torch.zeros((n, bins, maxf), device="cuda")
    sdsc = spectra_desc(n, bins, maxf)
    assert audio.spectrogram(pre, d, spec, sdsc, ld, p.centerWindows, p.reflectPadding, None, p.nfft, p.power,
                             p.windowLength, p.windowStep, h) == OK
    F = [max(0, min(maxf, (int(l) - (0 if p.centerWindows else p.windowLength)) // p.windowStep + 1)) for l in lens]
    dims = dev(np.array([[bins, f] for f in F], np.int32))
    mel = torch.zeros((n, p.numFilter, maxf), device="cuda")
    mdsc = spectra_desc(n, p.numFilter, maxf)
    assert audio.mel_filter_bank(spec, sdsc, mel, mdsc, dims, p.maxFreq, p.minFreq, p.melFormula, p.numFilter,
                                 p.sampleRate, p.normalize, h) == OK
    db = canvas((n, p.numFilter, maxf))
    patches = dev(np.array([[f, p.numFilter] for f in F], np.int32))
    assert audio.to_decibels(mel, mdsc, db, mdsc, patches, p.cutOffDB, p.multiplier, p.referenceMagnitude, h) == OK
    return host(db), F


CASES = [
    dict(nfft=512, window_length=400, window_step=160, num_filter=128),
    dict(nfft=512, window_length=320, window_step=160, num_filter=80, border=1, lookahead=1),
    dict(nfft=256, window_length=256, window_step=100, num_filter=40, mel_formula=1, normalize=False, border=2),
    dict(nfft=1024, window_length=1024, window_step=256, num_filter=64, reference_magnitude=1.0, lookahead=64),
    dict(nfft=512, window_length=400, window_step=160, num_filter=128, center=False, reflect=False,
         cut_off_db=-60.0),
    dict(nfft=2048, window_length=1600, window_step=400, num_filter=128),
    dict(nfft=128, window_length=100, window_step=51, num_filter=20),    # odd hop: unpaired window gather
    dict(nfft=512, window_length=400, window_step=160, num_filter=128, power=1),
]


@pytest.mark.parametrize("kw", CASES)
def test_frontend_equals_plain_chain(gpu, kw):
    r = np.random.Generator(np.random.PCG64(99))
    lens = r.integers(1, 48000, 11)
    lens[0], lens[1], lens[2] = 48000, 1, 2
    x, lens = synth.mono_batch(len(lens), lens.astype(np.int32), r, gaps=True)
    n, L = x.shape
    coeff = r.uniform(0.9, 0.99, n).astype(np.float32)
    p = frontend_params(**kw)
    maxf = 48000 // p.windowStep + 1
    ref, F = plain_chain(gpu, x, lens, coeff, p, maxf)
    out = canvas((n, p.numFilter, maxf))
    st = audio.frontend(dev(x), audio_desc(n, L), out, spectra_desc(n, p.numFilter, maxf), dev(lens), dev(coeff), p,
                        gpu)
    assert st == OK
    o = host(out)
    for i in range(n):
        assert (o[i, :, F[i]:] == -12345.0).all()
        if F[i] == 1:
            # one-frame clips: the four-call chain hands to_decibels srcDims {width 1, height numFilter},
            # which the reference treats as a 1-D run of numFilter contiguous values
            # (cpu/kernel/to_decibels.cpp:58-83); the fused call converts the clip's column instead
            assert np.isfinite(o[i, :, 0]).all() and (o[i, :, 0] <= 0).all()
            continue
        np.testing.assert_array_equal(o[i, :, :F[i]], ref[i, :, :F[i]])
    assert audio.device_error(gpu) == 0


def test_frontend_vs_fp64_oracle(gpu, oracle):
    """Error of the fused chain against the FP64 chain.  Any FP32 FFT chain, the reference's own
    host path included (up to 1.9e-3 dB on this input), loses accuracy in bins far below the frame's
    largest, so the bound is 1e-3 dB where the mel power is within 60 dB of its frame's maximum and
    1e-2 dB everywhere else above the cutoff."""
    x, lens = synth.gapped_clips(n=12, max_len=64000)
    n, L = x.shape
    coeff = np.full(n, 0.97, np.float32)
    p = frontend_params()
    F = (lens // 160 + 1).astype(np.int32)
    mf = int(F.max())
    out = canvas((n, 128, mf))
    assert audio.frontend(dev(x), audio_desc(n, L), out, spectra_desc(n, 128, mf), dev(lens), dev(coeff), p,
                          gpu) == OK
    o = host(out)
    spec64 = oracle.spectrogram_f64(x, lens, 1, 1, None, 512, 2, 400, 160, 1, max_frames=mf, preemph_coeff=coeff)
    dims = np.stack([np.full(n, 257, np.int32), F], 1).ravel()
    mel64 = oracle.mel_filter_bank_f64(spec64, dims, 8000.0, 0.0, 0, 128, 16000.0, 1)
    db64 = oracle.to_decibels_f64(mel64, np.full(n, 128, np.int32), F, -80.0, 10.0, 0.0)
    for i in range(n):
        got, exp = o[i, :, :F[i]], db64[i, :, :F[i]]
        err = np.abs(got - exp)
        near = exp >= exp.max(axis=0, keepdims=True) - 60.0
        assert err[near].max() < 1e-3
        assert err.max() < 1e-2


def test_frontend_graph_capture(gpu):
    """After one uncaptured call sized the workspace, the fused call captures into a CUDA graph
    and replays to the same result."""
    x, lens = synth.gapped_clips(n=16, max_len=48000)
    n, L = x.shape
    p = frontend_params()
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
            out.fill_(-12345.0)   # the canvas value: replay must rewrite exactly the first call's values
            torch.cuda.synchronize()
            with torch.cuda.graph(g, stream=s):
                assert audio.frontend(xd, sd, out, dd, ld, cd, p, gpu) == OK
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(host(out), first)
    finally:
        gpu.set_stream(torch.cuda.current_stream().cuda_stream)


def test_frontend_capture_builds_uncached_tables():
    """The fused kernel's mel tables are cached per handle and mel parameters by the first uncaptured
    call.  A call captured with parameters not cached yet (here 80 filters, after a 128-filter call
    sized the workspace of a fresh handle) builds them in every CTA instead; both ways give the same
    bits."""
    from rpp_b200 import lib
    h = lib.Handle(batch_size=1, stream=torch.cuda.current_stream().cuda_stream)
    g = None
    try:
        x, lens = synth.gapped_clips(n=12, max_len=48000)
        n, L = x.shape
        mf = 48000 // 160 + 1
        xd, ld, cd = dev(x), dev(lens), dev(np.full(n, 0.97, np.float32))
        sd = audio_desc(n, L)
        out128 = canvas((n, 128, mf))
        assert audio.frontend(xd, sd, out128, spectra_desc(n, 128, mf), ld, cd, frontend_params(), h) == OK
        p80 = frontend_params(num_filter=80)
        d80 = spectra_desc(n, 80, mf)
        out80 = canvas((n, 80, mf))
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        h.set_stream(s.cuda_stream)
        with torch.cuda.stream(s):
            torch.cuda.synchronize()
            with torch.cuda.graph(g, stream=s):
                assert audio.frontend(xd, sd, out80, d80, ld, cd, p80, h) == OK
        g.replay()
        torch.cuda.synchronize()
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        captured = host(out80).copy()
        # the same call uncaptured now builds and caches the 80-filter tables
        out80.fill_(-12345.0)
        assert audio.frontend(xd, sd, out80, d80, ld, cd, p80, h) == OK
        np.testing.assert_array_equal(captured, host(out80))
        assert audio.device_error(h) == 0
    finally:
        torch.cuda.synchronize()
        del g
        h.close()


@pytest.mark.parametrize("chunks,pinned_io", [(0, True), (1, True), (3, True), (50, True), (4, False)])
def test_frontend_host_equals_device(gpu, chunks, pinned_io):
    """rppb_frontend_host_gpu (host tensors, chunked copy/compute overlap) writes exactly what
    rppb_frontend_gpu writes on the same data, and nothing outside the valid region."""
    r = np.random.Generator(np.random.PCG64(5))
    lens = r.integers(0, 40000, 13).astype(np.int32)
    lens[0], lens[1], lens[2], lens[3] = 40000, 0, 1, 2
    x, lens = synth.mono_batch(len(lens), lens, r, gaps=True)
    n, L = x.shape
    coeff = r.uniform(0.9, 0.99, n).astype(np.float32)
    p = frontend_params(border=2)
    mf = 40000 // p.windowStep + 1
    sd, dd = audio_desc(n, L), spectra_desc(n, p.numFilter, mf)
    ref = canvas((n, p.numFilter, mf))
    assert audio.frontend(dev(x), sd, ref, dd, dev(lens), dev(coeff), p, gpu) == OK
    exp = host(ref)
    if pinned_io:
        xs, out = torch.from_numpy(x).pin_memory(), torch.full((n, p.numFilter, mf), -12345.0).pin_memory()
        ls, cs = torch.from_numpy(lens).pin_memory(), torch.from_numpy(coeff).pin_memory()
    else:
        xs, out, ls, cs = x, np.full((n, p.numFilter, mf), -12345.0, np.float32), lens, coeff
    assert audio.frontend_host(xs, sd, out, dd, ls, cs, p, chunks, gpu) == OK
    torch.cuda.synchronize()
    got = out.numpy() if hasattr(out, "numpy") else out
    np.testing.assert_array_equal(got, exp)
    assert audio.device_error(gpu) == 0


SCHEDULES = [dict(tile_frames=32), dict(tile_frames=64, db_frames=16), dict(db_frames=32, lookahead=8),
             dict(db_frames=128, ctas_per_sm=1),
             dict(tile_frames=32, db_frames=256, lookahead=96, ctas_per_sm=2)]


@pytest.mark.parametrize("sched", SCHEDULES)
def test_frontend_schedule_knobs_are_bit_identical(gpu, sched):
    """Tile frames, decibel item frames, lookahead and CTAs per SM move work between CTAs and in
    time only: every schedule writes exactly the default schedule's bits."""
    x, lens = synth.gapped_clips(n=20, max_len=64000)
    n, L = x.shape
    mf = 64000 // 160 + 1
    xd, ld, cd = dev(x), dev(lens), dev(np.full(n, 0.97, np.float32))
    sd, dd = audio_desc(n, L), spectra_desc(n, 128, mf)
    ref = canvas((n, 128, mf))
    assert audio.frontend(xd, sd, ref, dd, ld, cd, frontend_params(), gpu) == OK
    out = canvas((n, 128, mf))
    assert audio.frontend(xd, sd, out, dd, ld, cd, frontend_params(**sched), gpu) == OK
    np.testing.assert_array_equal(host(out), host(ref))
    assert audio.device_error(gpu) == 0


def test_frontend_tune(gpu):
    """The autotuner picks a valid schedule, leaves the result unchanged, and answers a repeated
    shape from its cache."""
    x, lens = synth.gapped_clips(n=32, max_len=96000)
    n, L = x.shape
    mf = 96000 // 160 + 1
    xd, ld, cd = dev(x), dev(lens), dev(np.full(n, 0.97, np.float32))
    sd, dd = audio_desc(n, L), spectra_desc(n, 128, mf)
    ref = canvas((n, 128, mf))
    assert audio.frontend(xd, sd, ref, dd, ld, cd, frontend_params(), gpu) == OK
    p = frontend_params()
    out = canvas((n, 128, mf))
    st, ms = audio.frontend_tune(xd, sd, out, dd, ld, cd, p, gpu, reps=2)
    assert st == OK and ms > 0
    assert p.tileFrames in (16, 32, 64) and p.dbFrames in (32, 64, 128) and p.lookahead in (8, 32, 96)
    assert p.ctasPerSm in (0, 2)
    np.testing.assert_array_equal(host(out), host(ref))
    q = frontend_params()
    st2, ms2 = audio.frontend_tune(xd, sd, out, dd, ld, cd, q, gpu)
    assert st2 == OK and ms2 == ms
    assert (q.tileFrames, q.dbFrames, q.lookahead, q.ctasPerSm) == (p.tileFrames, p.dbFrames, p.lookahead,
                                                                     p.ctasPerSm)
    out2 = canvas((n, 128, mf))
    assert audio.frontend(xd, sd, out2, dd, ld, cd, q, gpu) == OK
    np.testing.assert_array_equal(host(out2), host(ref))


def test_frontend_wait_timeout_reports_device_error():
    """Failure detection without a fault or a hang.  With the wait fault injection on, every decibel
    item of the fused kernel waits for a spectrum tile that is never counted; its bounded wait gives
    up (~1024 polls), sets the device error word, leaves the item's mel power unconverted, and the
    launch ends.  The host reads the error, and the same handle, injection off, then computes the
    batch exactly as before."""
    from rpp_b200 import lib
    h = lib.Handle(batch_size=1, stream=torch.cuda.current_stream().cuda_stream)
    try:
        x, lens = synth.gapped_clips(n=6, max_len=32000)
        n, L = x.shape
        coeff = np.full(n, 0.97, np.float32)
        p = frontend_params()
        F = (lens // 160 + 1).astype(np.int32)
        mf = int(F.max())
        args = (dev(x), audio_desc(n, L))
        rest = (spectra_desc(n, 128, mf), dev(lens), dev(coeff), p, h)
        ref = canvas((n, 128, mf))
        assert audio.frontend(*args, ref, *rest) == OK
        assert audio.device_error(h) == 0
        r = host(ref)

        assert audio.set_wait_fault_injection(h, True) == OK
        try:
            out = canvas((n, 128, mf))
            assert audio.frontend(*args, out, *rest) == OK
            assert audio.device_error(h) == 1
        finally:
            assert audio.set_wait_fault_injection(h, False) == OK
        o = host(out)
        for i in range(n):
            # decibels are <= 0 (reference = the clip's maximum); the skipped items hold mel power >= 0
            assert (r[i, :, :F[i]] <= 0).all()
            assert (o[i, :, :F[i]] >= 0).all()
            assert (o[i, :, F[i]:] == -12345.0).all()

        again = canvas((n, 128, mf))
        assert audio.frontend(*args, again, *rest) == OK
        assert audio.device_error(h) == 0
        np.testing.assert_array_equal(host(again), r)
    finally:
        torch.cuda.synchronize()
        h.close()
