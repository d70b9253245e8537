"""ORACLE — test infrastructure only: the reference host library's own output for the front-end
chain and the non-silent-region detector, and the parity metrics of a GPU result against it.

Used by tests/test_gpu_parity_reference.py and by bench.py's parity leg; never by the product.

The chain is the benchmark's: pre_emphasis_filter (coeff per clip, border ZERO) -> spectrogram
(nfft 512, window 400, hop 160, Hann, centred, reflect, power 2, NFT) -> mel_filter_bank (128
Slaney filters, 0-8 kHz, normalized) -> to_decibels (x10, -80 dB cutoff, reference = per-clip
maximum), each step run by the reference's rppt_*_host entry point
(src/modules/tensor/cpu/kernel/{pre_emphasis_filter,spectrogram,mel_filter_bank,to_decibels}.cpp).

Metrics (the parity bars):
  pre-emphasis        bit-exact (max |diff| = 0)
  spectrogram, mel    |got - ref| / max over the frame's bins of ref   <= 1e-5
  decibels            |got - ref| in dB, reported overall and where the reference's mel power lies
                      within 60 dB of its frame maximum; the count and share of values above 1e-3 dB
                      and the distribution (percentiles) are reported beside the maximum
  NSR begin/length    bit-exact (src/modules/tensor/cpu/kernel/non_silent_region_detection.cpp:93-191)
"""
import numpy as np

from rpp_b200.types import RpptImagePatch, audio_desc, spectra_desc

NFFT, WIN, HOP, NMEL, RATE = 512, 400, 160, 128, 16000.0
DB_BAR = 1e-3
POWER_BAR = 1e-5


def frames_of(lens, hop=HOP):
    return (np.asarray(lens, np.int64) // hop + 1).astype(np.int32)


def reference_front_end(ref, x, lens, coeff=0.97, nfft=NFFT, W=WIN, hop=HOP, nmel=NMEL, cutoff=-80.0, mult=10.0):
    """The reference's four host calls on (x, lens); returns float32 pre [n][L], spec [n][bins][mf],
    mel and db [n][nmel][mf] (valid frames only are meaningful)."""
    x = np.ascontiguousarray(x, np.float32)
    lens = np.ascontiguousarray(lens, np.int32)
    n, L = x.shape
    F = frames_of(lens, hop)
    mf = int(F.max())
    bins = nfft // 2 + 1
    sd = audio_desc(n, L)
    pre = np.zeros_like(x)
    spec = np.zeros((n, bins, mf), np.float32)
    mel = np.zeros((n, nmel, mf), np.float32)
    db = np.zeros_like(mel)
    co = np.full(n, coeff, np.float32)
    dims = np.stack([np.full(n, bins, np.int32), F], 1).astype(np.int32).ravel()
    patches = (RpptImagePatch * n)()
    for i in range(n):
        patches[i].width, patches[i].height = int(F[i]), nmel
    spd, md = spectra_desc(n, bins, mf), spectra_desc(n, nmel, mf)
    assert ref.pre_emphasis_filter(x, sd, pre, sd, lens, co, 0) == 0
    assert ref.spectrogram(pre, sd, spec, spd, lens, True, True, None, nfft, 2, W, hop) == 0
    assert ref.mel_filter_bank(spec, spd, mel, md, dims, 8000.0, 0.0, 0, nmel, RATE, True) == 0
    assert ref.to_decibels(mel, md, db, md, patches, cutoff, mult, 0.0) == 0
    return {"pre": pre, "spec": spec, "mel": mel, "db": db, "frames": F}


def reference_nsr(ref, x, lens, cutoff=-60.0, window=2048, ref_power=0.0, reset=8192):
    """rppt_non_silent_region_detection_host on the raw clips: int32 (begin, length) per clip."""
    x = np.ascontiguousarray(x, np.float32)
    lens = np.ascontiguousarray(lens, np.int32)
    n, L = x.shape
    begin = np.zeros(n, np.int32)
    length = np.zeros(n, np.int32)
    assert ref.nsr(x, audio_desc(n, L), lens, begin, length, cutoff, window, ref_power, reset) == 0
    return begin, length


def _frame_rel(got, exp):
    """max over the clip of |got - exp| / (the frame's largest exp); frames along the last axis."""
    exp = exp.astype(np.float64)
    scale = np.maximum(exp.max(axis=0, keepdims=True), 1e-30)
    return float((np.abs(got.astype(np.float64) - exp) / scale).max()) if exp.size else 0.0


def chain_parity(refo, pre=None, spec=None, mel=None, db=None, lens=None):
    """Parity metrics of GPU outputs (any subset of pre/spec/mel/db, same shapes as the reference's)
    against the reference output `refo` of reference_front_end."""
    F = refo["frames"]
    n = len(F)
    out = {"clips": n, "frames": int(F.sum())}
    if pre is not None:
        d = 0.0
        for i in range(n):
            li = int(lens[i])
            d = max(d, float(np.abs(pre[i, :li] - refo["pre"][i, :li]).max()) if li else 0.0)
        out["pre_emphasis_max_abs_diff"] = d
        out["pre_emphasis_bit_exact"] = d == 0.0
    if spec is not None:
        out["spectrogram_power_rel_err_per_frame_max"] = max(
            _frame_rel(spec[i, :, :F[i]], refo["spec"][i, :, :F[i]]) for i in range(n))
    if mel is not None:
        out["mel_power_rel_err_per_frame_max"] = max(
            _frame_rel(mel[i, :, :F[i]], refo["mel"][i, :, :F[i]]) for i in range(n))
    if db is not None:
        errs, near_errs = [], []
        for i in range(n):
            r = refo["db"][i, :, :F[i]].astype(np.float64)
            e = np.abs(db[i, :, :F[i]].astype(np.float64) - r)
            # within 60 dB of the frame maximum of the reference's decibels (= of its mel power)
            near = r >= r.max(axis=0, keepdims=True) - 60.0
            errs.append(e.ravel())
            near_errs.append(e[near])
        e = np.concatenate(errs)
        en = np.concatenate(near_errs)
        above = int((e > DB_BAR).sum())
        out.update({
            "db_max_abs_err": float(e.max()) if e.size else 0.0,
            "db_max_abs_err_within_60db_of_frame_max": float(en.max()) if en.size else 0.0,
            "db_values": int(e.size),
            "db_values_above_1e-3": above,
            "db_share_above_1e-3": above / max(1, e.size),
            "db_values_above_1e-3_within_60db": int((en > DB_BAR).sum()),
            "db_abs_err_percentiles": {p: float(np.percentile(e, float(p))) for p in ("50", "99", "99.9", "99.99")}
            if e.size else {},
        })
    return out
