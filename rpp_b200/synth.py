"""Seeded synthetic audio batches with the shapes and value distributions of the benchmark
workloads (no datasets are available offline).  NumPy PCG64; each batch kind has its own seed.

  short_clips            8 mono clips, 16 kHz, lengths U[16000, 60000] (seed 20261203)
  gapped_clips           256 mono clips, 16 kHz, lengths U[16000, 256000] (1-16 s), plus 0-3 silent
                         spans of 0.1-1 s per clip (seed 20261204)
  dynamic_range_clips    1024 mono clips of 160000 samples; the white noise sits 40/60/80/100/120 dB
                         below the tones' peak (clip i: 40 + 20 * (i % 5) dB) instead of at sigma 0.1,
                         sweeping the dynamic range (seed 20261205)
  stereo_multirate_clips 2048 stereo clips, durations log-normal (median 4 s, sigma 0.25) clipped to
                         0.5-30 s, input rate uniform over {16000, 22050, 44100, 48000}; both channels
                         share the sines and have independent noise (seed 20261206)

Signal model (all but dynamic_range_clips): Gaussian noise sigma 0.1 plus 3 sinusoids with
frequency U[100, 6000] Hz and amplitude U[0.05, 0.5].
"""
import numpy as np

SEED = 20261203


def _tones(rng, length, rate, n_tones=3):
    t = np.arange(length, dtype=np.float64) / rate
    x = np.zeros(length, np.float64)
    for _ in range(n_tones):
        f = rng.uniform(100.0, 6000.0)
        a = rng.uniform(0.05, 0.5)
        ph = rng.uniform(0.0, 2 * np.pi)
        x += a * np.sin(2 * np.pi * f * t + ph)
    return x


def mono_batch(n, lengths, rng, rate=16000, gaps=False, floor_db=None):
    """Returns (float32 [n][maxLen] zero-padded, int32 lengths)."""
    lengths = np.asarray(lengths, np.int32)
    L = int(lengths.max()) if n else 0
    out = np.zeros((n, L), np.float32)
    for i in range(n):
        li = int(lengths[i])
        x = _tones(rng, li, rate)
        if floor_db is None:
            x += rng.normal(0.0, 0.1, li)
        else:
            # the white noise sits floor_db below the tones' peak (a fixed sigma of 0.1 would pin the
            # dynamic range near 20 dB and leave nothing to sweep)
            peak = np.abs(x).max() if li else 1.0
            x += rng.normal(0.0, peak * 10.0 ** (-floor_db[i] / 20.0), li)
        if gaps:
            for _ in range(rng.integers(0, 4)):
                g = int(rng.uniform(0.1, 1.0) * rate)
                s = int(rng.integers(0, max(1, li - g)))
                x[s:s + g] = 0.0
        out[i, :li] = x.astype(np.float32)
    return out, lengths


def short_clips(n=8):
    rng = np.random.Generator(np.random.PCG64(SEED + 0))
    lengths = rng.integers(16000, 60001, n)
    return mono_batch(n, lengths, rng)


def gapped_clips(n=256, max_len=256000):
    rng = np.random.Generator(np.random.PCG64(SEED + 1))
    lengths = rng.integers(16000, max_len + 1, n)
    return mono_batch(n, lengths, rng, gaps=True)


def dynamic_range_clips(n=1024, length=160000):
    rng = np.random.Generator(np.random.PCG64(SEED + 2))
    floors = np.array([40, 60, 80, 100, 120], np.float64)[np.arange(n) % 5]
    return mono_batch(n, np.full(n, length), rng, floor_db=floors) + (floors,)


def stereo_multirate_clips(n=2048):
    """Returns (float32 [n][maxLen*2] interleaved stereo, int32 lengths, float32 in rates)."""
    rng = np.random.Generator(np.random.PCG64(SEED + 3))
    dur = np.clip(rng.lognormal(np.log(4.0), 0.25, n), 0.5, 30.0)
    rates = rng.choice(np.array([16000, 22050, 44100, 48000], np.float32), n)
    lengths = np.maximum(1, (dur * rates).astype(np.int64)).astype(np.int32)
    L = int(lengths.max())
    out = np.zeros((n, 2 * L), np.float32)
    for i in range(n):
        li = int(lengths[i])
        s = _tones(rng, li, float(rates[i]))
        left = s + rng.normal(0.0, 0.1, li)
        right = s + rng.normal(0.0, 0.1, li)
        out[i, 0:2 * li:2] = left.astype(np.float32)
        out[i, 1:2 * li:2] = right.astype(np.float32)
    return out, lengths, rates
