"""A C++ caller through the C ABI: tests/caller/rnnt_pipeline.cpp includes only include/*.h, links
librppb.so and runs the RNN-T speech front end the way an augmentation pipeline binds RPP (int16 PCM
-> float, non-silent region detection, slice to the region, pre-emphasis, spectrogram, mel filter
bank, decibels, per-filter normalisation; one handle on its own stream, per-sample tensors in
pinned memory).  Each stage's output is checked against the oracle on the previous stage's output:
bit for bit for the integer and replayed-order float stages, within the parity bounds of the other
GPU tests for the spectrogram (FFT order), decibels (log) and normalisation (rsqrt)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from rpp_b200 import synth
from gpu_util import DB_ABS, SPEC_FRAME_REL, frame_rel_err

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "caller", "rnnt_pipeline.cpp")
BUILD = os.path.join(ROOT, "tests", "caller", "_build")
NFFT, WIN, HOP, BINS, NMEL = 512, 400, 160, 257, 128


def build_caller():
    """g++ against include/ and rpp_b200/librppb.so, as a C++ project would link the library."""
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.fail("g++ is needed to build the C++ caller")
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "rnnt_pipeline")
    lib_dir = os.path.join(ROOT, "rpp_b200")
    cuda = "/usr/local/cuda"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"), SRC, "-o", exe, "-L", lib_dir, "-lrppb",
           "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + lib_dir,
           "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def make_input(path, n=8, seed=20261230):
    """Seeded clips with silence before and after the signal (so the detection trims something),
    quantised to int16 PCM as a WAV file holds it."""
    r = np.random.Generator(np.random.PCG64(seed))
    body, body_lens = synth.gapped_clips(n=n, max_len=48000)
    lead = r.integers(0, 8000, n)
    tail = r.integers(0, 8000, n)
    lens = (lead + body_lens + tail).astype(np.int32)
    w = int(lens.max())
    pcm = np.zeros((n, w), np.int16)
    for b in range(n):
        s = np.clip(np.round(body[b, :body_lens[b]] * 16384.0), -32768, 32767).astype(np.int16)
        pcm[b, lead[b]:lead[b] + body_lens[b]] = s
    with open(path, "wb") as f:
        np.array([n, w], np.int32).tofile(f)
        lens.tofile(f)
        pcm.tofile(f)
    return pcm, lens


def load(out_dir, name, dtype, shape):
    return np.fromfile(os.path.join(out_dir, name + ".bin"), dtype=dtype).reshape(shape)


def test_cpp_caller_rnnt_pipeline(tmp_path, oracle):
    exe = build_caller()
    inp = str(tmp_path / "input.bin")
    pcm, lens = make_input(inp)
    out_dir = str(tmp_path / "out")
    os.makedirs(out_dir)
    r = subprocess.run([exe, inp, out_dir], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    n, w, mf = (int(v) for v in np.fromfile(os.path.join(out_dir, "meta.bin"), np.int32))
    assert (n, w) == pcm.shape

    # int16 -> float: exact / 32768 over each clip, the untouched tail stays as the caller zeroed it
    sig = load(out_dir, "signal", np.float32, (n, w))
    exp_sig = np.zeros((n, w), np.float32)
    for b in range(n):
        exp_sig[b, :lens[b]] = pcm[b, :lens[b]].astype(np.float32) / np.float32(32768.0)
    np.testing.assert_array_equal(sig, exp_sig)

    # detection: integers, bit for bit; the leading silence is found on every clip
    begin = load(out_dir, "nsr_begin", np.int32, (n,))
    length = load(out_dir, "nsr_length", np.int32, (n,))
    eb, el = oracle.nsr(sig, lens, -60.0, 2048, 0.0, 8192)
    np.testing.assert_array_equal(begin, eb)
    np.testing.assert_array_equal(length, el)
    assert (length > 0).all() and (length < lens).any()

    # slice to the detected region (no padding): bit for bit, zeros elsewhere
    trimmed = load(out_dir, "trimmed", np.float32, (n, w))
    roi = np.stack([np.zeros(n), lens], 1).astype(np.uint32).ravel()
    exp_trim = oracle.slice(sig, np.zeros((n, w), np.float32), begin, length, roi, 0.0, False, 1)
    np.testing.assert_array_equal(trimmed, exp_trim)

    # pre-emphasis (0.97, ZERO border) over the detected lengths: the reference's order, bit for bit
    pre = load(out_dir, "preemph", np.float32, (n, w))
    exp_pre = oracle.pre_emphasis(trimmed, np.zeros((n, w), np.float32), length, np.full(n, 0.97, np.float32), 0)
    np.testing.assert_array_equal(pre, exp_pre)

    # spectrogram against FP64, per frame relative to the frame's largest bin
    F = (length // HOP + 1).astype(np.int32)
    assert int(F.max()) == mf
    spec = load(out_dir, "spectrogram", np.float32, (n, BINS, mf))
    spec64 = oracle.spectrogram_f64(pre, length, 1, 1, None, NFFT, 2, WIN, HOP, 1, max_frames=mf)
    for b in range(n):
        assert frame_rel_err(spec[b, :, :F[b]], spec64[b, :, :F[b]]) <= SPEC_FRAME_REL

    # mel filter bank on the GPU's spectrum: bit for bit
    mel = load(out_dir, "mel", np.float32, (n, NMEL, mf))
    dims = np.stack([np.full(n, BINS), F], 1).astype(np.int32).ravel()
    exp_mel = oracle.mel_filter_bank(spec, np.zeros((n, NMEL, mf), np.float32), dims, 8000.0, 0.0, 0, NMEL,
                                     16000.0, 1)
    for b in range(n):
        np.testing.assert_array_equal(mel[b, :, :F[b]], exp_mel[b, :, :F[b]])

    # decibels on the GPU's mel power
    db = load(out_dir, "decibels", np.float32, (n, NMEL, mf))
    exp_db = oracle.to_decibels(mel, np.zeros((n, NMEL, mf), np.float32), np.stack([F, np.full(n, NMEL)], 1),
                                -80.0, 10.0, 0.0)
    for b in range(n):
        assert np.abs(db[b, :, :F[b]] - exp_db[b, :, :F[b]]).max() <= DB_ABS

    # per-filter normalisation over time of the GPU's decibels
    norm = load(out_dir, "normalized", np.float32, (n, NMEL, mf))
    mean = load(out_dir, "mean", np.float32, (n * NMEL,))
    inv_std = load(out_dir, "inv_std", np.float32, (n * NMEL,))
    nroi = np.stack([np.zeros(n), np.zeros(n), np.full(n, NMEL), F], 1).astype(np.uint32).ravel()
    m_ref, s_ref = np.zeros(n * NMEL, np.float32), np.zeros(n * NMEL, np.float32)
    exp_norm = oracle.normalize_2d(db, np.zeros((n, NMEL, mf), np.float32), 2, m_ref, s_ref, 3, 1.0, 0.0, nroi)
    np.testing.assert_array_equal(mean, m_ref)
    np.testing.assert_allclose(inv_std, s_ref, rtol=1e-6, atol=0)
    np.testing.assert_allclose(norm, exp_norm, rtol=1e-5, atol=1e-5)
