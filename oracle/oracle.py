"""ORACLE — test infrastructure only: ctypes fronts of the two CPU checkers (see __init__)."""
import ctypes
import glob
import os
import subprocess

import numpy as np

from rpp_b200.types import RpptDesc, RpptImagePatch

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
_REF_SO = os.path.join(HERE, "_ref", "librpp_audio_ref.so")


def oracle_lib_path():
    return _ORACLE_SO


def reference_lib_path():
    return _REF_SO


def _gcc_spec_dir(cc):
    """A gcc library directory holding libgomp.spec (some gcc installs on PATH lack it)."""
    cands = []
    try:
        lib = subprocess.run([cc, "-print-libgcc-file-name"], capture_output=True, text=True).stdout.strip()
        cands.append(os.path.dirname(lib))
    except OSError:
        pass
    cands += sorted(glob.glob("/usr/lib/gcc/x86_64-linux-gnu/*"))
    for d in cands:
        if os.path.isfile(os.path.join(d, "libgomp.spec")):
            return d
    return None


def build_oracle(force=False):
    """Compiles oracle/rppb_oracle.c into oracle/_build/liboracle.so (float ops uncontracted)."""
    src = os.path.join(HERE, "rppb_oracle.c")
    if not force and os.path.isfile(_ORACLE_SO) and os.path.getmtime(_ORACLE_SO) >= os.path.getmtime(src):
        return _ORACLE_SO
    os.makedirs(os.path.dirname(_ORACLE_SO), exist_ok=True)
    cc = os.environ.get("CC", "gcc")
    cmd = [cc, "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-fopenmp"]
    spec = _gcc_spec_dir(cc)
    if spec:
        cmd.append("-B" + spec + "/")
    cmd += ["-o", _ORACLE_SO + ".tmp", src, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(_ORACLE_SO + ".tmp", _ORACLE_SO)
    return _ORACLE_SO


def build_reference(ref_root=None):
    """Compiles the reference host audio path (oracle/build_ref.sh) when its sources exist.

    Returns the library path, or None when the reference sources are absent (the GPU box uses
    the prebuilt oracle/_ref/librpp_audio_ref.so)."""
    # default: the reference checkout beside this repository (../reference), or $RPP_REF
    root = ref_root or os.environ.get("RPP_REF", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
    if not os.path.isdir(os.path.join(root, "src", "modules", "tensor", "cpu", "kernel")):
        return _REF_SO if os.path.isfile(_REF_SO) else None
    env = dict(os.environ, RPP_REF=root)
    subprocess.run(["bash", os.path.join(HERE, "build_ref.sh")], check=True, env=env,
                   stdout=subprocess.DEVNULL)
    return _REF_SO


_F32P = ctypes.POINTER(ctypes.c_float)
_F64P = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int32)
_U32P = ctypes.POINTER(ctypes.c_uint32)
_L = ctypes.c_long
_I = ctypes.c_int
_F = ctypes.c_float


def _p(a, ct):
    return a.ctypes.data_as(ct)


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


class Oracle:
    """The C restatement (oracle/rppb_oracle.c)."""

    def __init__(self, path=None):
        path = path or _ORACLE_SO
        if not os.path.isfile(path):
            build_oracle()
        L = self.lib = ctypes.CDLL(path)
        L.oracle_pre_emphasis.argtypes = [_F32P, _L, _F32P, _L, _I, _I32P, _F32P, _I]
        L.oracle_down_mixing.argtypes = [_F32P, _L, _F32P, _L, _I, _I32P, _I]
        L.oracle_resample.argtypes = [_F32P, _L, _F32P, _L, _I, _F32P, _F32P, _I32P, _F32P, _I, _F, _F, _I]
        L.oracle_num_windows.argtypes = [_I, _I, _I, _I]
        L.oracle_num_windows.restype = _I
        L.oracle_hann_window.argtypes = [_F32P, _I]
        L.oracle_spectrogram_f64.argtypes = [_F32P, _L, _F64P, _L, _L, _I, _I32P, _I, _I, _F32P, _I, _I, _I, _I, _I,
                                             _I, _F32P, _I]
        L.oracle_mel_filter_bank.argtypes = [_F32P, _L, _L, _F32P, _L, _L, _I, _I32P, _F, _F, _I, _I, _F, _I]
        L.oracle_mel_filter_bank_f64.argtypes = [_F64P, _L, _L, _F64P, _L, _L, _I, _I32P, _F, _F, _I, _I, _F, _I]
        L.oracle_mel_tables.argtypes = [_I, _F, _F, _I, _F, _I, _I, _I32P, _F32P, _F32P, _I32P]
        L.oracle_to_decibels.argtypes = [_F32P, _L, _L, _F32P, _L, _L, _I, _U32P, _F, _F, _F]
        L.oracle_to_decibels_f64.argtypes = [_F64P, _L, _L, _F64P, _I, _I32P, _I32P, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double]
        L.oracle_nsr.argtypes = [_F32P, _L, _I, _I32P, _I32P, _I32P, _F, _I, _F, _I, _F32P, _F32P]
        L.oracle_windowed_sinc.argtypes = [_I, _I, _F32P, _F32P]
        L.oracle_normalize_2d.argtypes = [_F32P, _L, _L, _F32P, _L, _L, _I, ctypes.c_uint, _F32P, _F32P, _I, _F, _F,
                                          _U32P]
        L.oracle_normalize_2d.restype = _I
        L.oracle_slice.argtypes = [ctypes.c_void_p, _L, _L, ctypes.c_void_p, _L, _L, _I, _I, _I32P, _I32P, _U32P,
                                   ctypes.c_void_p, _I, _I]
        _LP = ctypes.POINTER(_L)
        L.oracle_normalize_nd.argtypes = [ctypes.c_void_p, _I, _LP, _I, _I32P, ctypes.c_void_p, _I, _LP, _I, _I, _I,
                                          ctypes.c_uint, _F32P, _F32P, _I, _F, _F, _U32P]
        L.oracle_normalize_nd.restype = _I
        L.oracle_slice_nd.argtypes = [ctypes.c_void_p, _LP, ctypes.c_void_p, _LP, _I32P, _I, _I, _I, _I32P, _I32P,
                                      _U32P, ctypes.c_void_p, _I, _I]

    def windowed_sinc(self, coeffs, lobes):
        """The test suite's Hann-windowed sinc table: (lut, scale, center, lobes)."""
        lut = np.zeros(coeffs + 5, np.float32)
        out = np.zeros(3, np.float32)
        self.lib.oracle_windowed_sinc(int(coeffs), int(lobes), _p(lut, _F32P), _p(out, _F32P))
        return lut, float(out[0]), float(out[1]), int(out[2])

    # Each method takes numpy arrays laid out as the descriptors describe ([n][stride...]).
    def pre_emphasis(self, src, dst, lengths, coeff, border):
        n, ss = src.shape
        self.lib.oracle_pre_emphasis(_p(src, _F32P), ss, _p(dst, _F32P), dst.shape[1], n,
                                     _p(np.ascontiguousarray(lengths, np.int32), _I32P), _p(_f32(coeff), _F32P),
                                     int(border))
        return dst

    def down_mixing(self, src, dst, dims, normalize):
        n = src.shape[0]
        self.lib.oracle_down_mixing(_p(src, _F32P), src.shape[1], _p(dst, _F32P), dst.shape[1], n,
                                    _p(np.ascontiguousarray(dims, np.int32), _I32P), int(normalize))
        return dst

    def resample(self, src, dst, in_rate, out_rate, dims, lut, scale, center, lobes):
        n = src.shape[0]
        lut = _f32(lut)
        self.lib.oracle_resample(_p(src, _F32P), src.shape[1], _p(dst, _F32P), dst.shape[1], n,
                                 _p(_f32(in_rate), _F32P), _p(_f32(out_rate), _F32P),
                                 _p(np.ascontiguousarray(dims, np.int32), _I32P), _p(lut, _F32P), len(lut),
                                 float(scale), float(center), int(lobes))
        return dst

    def num_windows(self, length, window_length, window_step, center):
        return self.lib.oracle_num_windows(int(length), int(window_length), int(window_step), int(center))

    def hann(self, W):
        w = np.zeros(W, np.float32)
        self.lib.oracle_hann_window(_p(w, _F32P), W)
        return w

    def spectrogram_f64(self, src, lengths, center, reflect, window, nfft, power, W, hop, nft, max_frames=None,
                        preemph_coeff=None, border=0):
        """FP64 spectrogram; returns double [n][bins][maxFrames] (NFT) or [n][maxFrames][bins]."""
        n, ss = src.shape
        lengths = np.ascontiguousarray(lengths, np.int32)
        nfft_e = nfft or W
        bins = nfft_e // 2 + 1
        if max_frames is None:
            max_frames = max(self.num_windows(l, W, hop, center) for l in lengths)
        shape = (n, bins, max_frames) if nft else (n, max_frames, bins)
        dst = np.zeros(shape, np.float64)
        hstride = max_frames if nft else bins
        win = _f32(window) if window is not None else None
        coeff = _f32(preemph_coeff) if preemph_coeff is not None else np.zeros(n, np.float32)
        self.lib.oracle_spectrogram_f64(_p(src, _F32P), ss, _p(dst, _F64P), dst.shape[1] * dst.shape[2], hstride, n,
                                        _p(lengths, _I32P), int(center), int(reflect),
                                        _p(win, _F32P) if win is not None else None, int(nfft), int(power), int(W),
                                        int(hop), int(nft), int(preemph_coeff is not None), _p(coeff, _F32P),
                                        int(border))
        return dst

    def mel_filter_bank(self, src, dst, dims, max_freq, min_freq, formula, num_filter, sample_rate, normalize):
        n = src.shape[0]
        self.lib.oracle_mel_filter_bank(_p(src, _F32P), src.shape[1] * src.shape[2], src.shape[2], _p(dst, _F32P),
                                        dst.shape[1] * dst.shape[2], dst.shape[2], n,
                                        _p(np.ascontiguousarray(dims, np.int32), _I32P), float(max_freq),
                                        float(min_freq), int(formula), int(num_filter), float(sample_rate),
                                        int(normalize))
        return dst

    def mel_filter_bank_f64(self, src, dims, max_freq, min_freq, formula, num_filter, sample_rate, normalize):
        n = src.shape[0]
        dst = np.zeros((n, num_filter, src.shape[2]), np.float64)
        self.lib.oracle_mel_filter_bank_f64(_p(src, _F64P), src.shape[1] * src.shape[2], src.shape[2],
                                            _p(dst, _F64P), dst.shape[1] * dst.shape[2], dst.shape[2], n,
                                            _p(np.ascontiguousarray(dims, np.int32), _I32P), float(max_freq),
                                            float(min_freq), int(formula), int(num_filter), float(sample_rate),
                                            int(normalize))
        return dst

    def mel_tables(self, formula, min_freq, max_freq, num_filter, sample_rate, normalize, nfft):
        bins = nfft // 2 + 1
        interval = np.zeros(bins + 1, np.int32)
        wd = np.zeros(bins + 1, np.float32)
        norm = np.zeros(num_filter + 1, np.float32)
        rng = np.zeros(2, np.int32)
        self.lib.oracle_mel_tables(int(formula), float(min_freq), float(max_freq), int(num_filter),
                                   float(sample_rate), int(normalize), int(nfft), _p(interval, _I32P),
                                   _p(wd, _F32P), _p(norm, _F32P), _p(rng, _I32P))
        return interval[:bins], wd[:bins], norm[:num_filter], (int(rng[0]), int(rng[1]))

    def to_decibels(self, src, dst, dims_wh, cutoff_db, multiplier, ref_mag):
        """src/dst shaped [n][rows][hStride] (2-D) or [n][stride] (1-D); dims_wh [n][2] = (width, height)."""
        n = src.shape[0]
        hs = src.shape[2] if src.ndim == 3 else 1
        dhs = dst.shape[2] if dst.ndim == 3 else 1
        ns = int(np.prod(src.shape[1:]))
        dns = int(np.prod(dst.shape[1:]))
        self.lib.oracle_to_decibels(_p(src, _F32P), ns, hs, _p(dst, _F32P), dns, dhs, n,
                                    _p(np.ascontiguousarray(dims_wh, np.uint32), _U32P), float(cutoff_db),
                                    float(multiplier), float(ref_mag))
        return dst

    def to_decibels_f64(self, src, rows, cols, cutoff_db, multiplier, ref_mag):
        n = src.shape[0]
        dst = np.zeros_like(src)
        self.lib.oracle_to_decibels_f64(_p(src, _F64P), src.shape[1] * src.shape[2], src.shape[2], _p(dst, _F64P), n,
                                        _p(np.ascontiguousarray(rows, np.int32), _I32P),
                                        _p(np.ascontiguousarray(cols, np.int32), _I32P), float(cutoff_db),
                                        float(multiplier), float(ref_mag))
        return dst

    def normalize_2d(self, src, dst, axis_mask, mean, std, compute, scale, shift, roi):
        """src/dst float32 [n][rows][cols]; mean/std float32 arrays updated in place as the
        reference does; roi uint32 n*4 (begin0, begin1, length0, length1).  Returns dst."""
        n, R, C = src.shape
        st = self.lib.oracle_normalize_2d(_p(src, _F32P), R * C, C, _p(dst, _F32P), dst.shape[1] * dst.shape[2],
                                          dst.shape[2], n, int(axis_mask), _p(mean, _F32P), _p(std, _F32P),
                                          int(compute), float(scale), float(shift),
                                          _p(np.ascontiguousarray(roi, np.uint32), _U32P))
        assert st == 0
        return dst

    def slice(self, src, dst, anchor, shape, roi, fill, enable_padding, num_dims):
        """src/dst: [n][stride0] (1-D) or [n][rows][stride1] (2-D) float32 or uint8 arrays; dst is
        updated in place (fill + box copy) and returned."""
        n = src.shape[0]
        es = src.dtype.itemsize
        s0 = int(np.prod(src.shape[1:]))
        d0 = int(np.prod(dst.shape[1:]))
        s1 = src.shape[-1] if num_dims == 2 else 0
        d1 = dst.shape[-1] if num_dims == 2 else 0
        f = np.array([fill], dtype=src.dtype)
        self.lib.oracle_slice(src.ctypes.data, s0, s1, dst.ctypes.data, d0, d1, n, int(num_dims),
                              _p(np.ascontiguousarray(anchor, np.int32), _I32P),
                              _p(np.ascontiguousarray(shape, np.int32), _I32P),
                              _p(np.ascontiguousarray(roi, np.uint32), _U32P), f.ctypes.data, int(enable_padding), es)
        return dst

    def slice_nd(self, src, dst, anchor, shape, roi, fill, enable_padding, layout):
        """3-D or 4-D slice of dense [n][...] float32 or uint8 arrays (numDims = src.ndim - 1) in the
        given layout (0 NCHW, 1 NHWC, 2 NCDHW, 3 NDHWC); dst is updated in place and returned."""
        nd = src.ndim - 1
        def strides(a):
            return (_L * (nd + 1))(*[st // a.itemsize for st in a.strides])
        dims = np.ascontiguousarray(src.shape[1:], np.int32)
        f = np.array([fill], dtype=src.dtype)
        self.lib.oracle_slice_nd(src.ctypes.data, strides(src), dst.ctypes.data, strides(dst), _p(dims, _I32P),
                                 src.shape[0], nd, int(layout),
                                 _p(np.ascontiguousarray(anchor, np.int32), _I32P),
                                 _p(np.ascontiguousarray(shape, np.int32), _I32P),
                                 _p(np.ascontiguousarray(roi, np.uint32), _U32P), f.ctypes.data, int(enable_padding),
                                 src.dtype.itemsize)
        return dst

    NORMALIZE_TYPES = {np.dtype(np.float32): 0, np.dtype(np.float16): 1, np.dtype(np.uint8): 2, np.dtype(np.int8): 3}

    def normalize_nd(self, src, dst, axis_mask, mean, std, compute, scale, shift, roi, src_layout=0, dst_layout=0):
        """rppt_normalize on dense [n][...] arrays of any rank and element type (float32, float16,
        uint8, int8): the F32 3-D branch or the N-D branch of the reference host path (the F32 2-D
        branch is normalize_2d).  mean / std are in-out arrays as in the reference; dst is updated in
        place and returned."""
        T = src.ndim - 1
        def strides(a):
            return (_L * (T + 1))(*[st // a.itemsize for st in a.strides])
        dims = np.ascontiguousarray(src.shape[1:], np.int32)
        st = self.lib.oracle_normalize_nd(src.ctypes.data, self.NORMALIZE_TYPES[src.dtype], strides(src), int(src_layout),
                                          _p(dims, _I32P), dst.ctypes.data, self.NORMALIZE_TYPES[dst.dtype],
                                          strides(dst), int(dst_layout), src.shape[0], T, int(axis_mask),
                                          _p(mean, _F32P), _p(std, _F32P), int(compute), float(scale), float(shift),
                                          _p(np.ascontiguousarray(roi, np.uint32), _U32P))
        assert st == 0, st
        return dst

    def nsr(self, src, lengths, cutoff_db, window_length, ref_power, reset_interval, want_mms=False):
        n, ss = src.shape
        begin = np.zeros(n, np.int32)
        length = np.zeros(n, np.int32)
        mms = np.zeros_like(src) if want_mms else None
        cut = np.zeros(n, np.float32)
        self.lib.oracle_nsr(_p(src, _F32P), ss, n, _p(np.ascontiguousarray(lengths, np.int32), _I32P),
                            _p(begin, _I32P), _p(length, _I32P), float(cutoff_db), int(window_length),
                            float(ref_power), int(reset_interval), _p(mms, _F32P) if want_mms else None,
                            _p(cut, _F32P))
        return (begin, length, mms, cut) if want_mms else (begin, length)


class Reference:
    """The reference's own host audio library (oracle/_ref/librpp_audio_ref.so)."""

    def __init__(self, threads=None, batch_slots=1, path=None):
        path = path or _REF_SO
        if not os.path.isfile(path):
            raise FileNotFoundError(f"reference host library missing: {path} (run oracle/build_ref.sh)")
        L = self.lib = ctypes.CDLL(path)
        L.ref_create.argtypes = [ctypes.c_size_t, ctypes.c_uint]
        L.ref_create.restype = ctypes.c_void_p
        L.ref_destroy.argtypes = [ctypes.c_void_p]
        L.ref_slice_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _I32P, _I32P,
                                    ctypes.c_void_p, ctypes.c_bool, _U32P, ctypes.c_void_p]
        L.ref_slice_u8.argtypes = L.ref_slice_f32.argtypes
        D = ctypes.POINTER(RpptDesc)
        V = ctypes.c_void_p
        L.rppt_pre_emphasis_filter_host.argtypes = [V, D, V, D, _I32P, _F32P, _I, V]
        L.rppt_down_mixing_host.argtypes = [V, D, V, D, _I32P, ctypes.c_bool, V]
        L.rppt_spectrogram_host.argtypes = [V, D, V, D, _I32P, ctypes.c_bool, ctypes.c_bool, _F32P, _I, _I, _I, _I, V]
        L.rppt_mel_filter_bank_host.argtypes = [V, D, V, D, _I32P, _F, _F, _I, _I, _F, ctypes.c_bool, V]
        L.rppt_to_decibels_host.argtypes = [V, D, V, D, ctypes.POINTER(RpptImagePatch), _F, _F, _F, V]
        L.rppt_non_silent_region_detection_host.argtypes = [V, D, _I32P, _I32P, _I32P, _F, _I, _F, _I, V]
        L.ref_resample.argtypes = [V, D, V, D, _F32P, _F32P, _I32P, _F32P, _I, _F, _F, _I, _I, V]
        for f in ("rppt_pre_emphasis_filter_host", "rppt_down_mixing_host", "rppt_spectrogram_host",
                  "rppt_mel_filter_bank_host", "rppt_to_decibels_host", "rppt_non_silent_region_detection_host",
                  "ref_resample"):
            getattr(L, f).restype = _I
        self.threads = threads or os.cpu_count()
        self.batch_slots = 0
        self.h = None
        self.ensure_slots(batch_slots)

    def ensure_slots(self, slots):
        """The host handle mallocs 99,532,800 floats of scratch per batch slot
        (src/modules/handle_host.cpp:50); the spectrogram needs n*maxFrames*nfft of them."""
        slots = max(1, int(slots))
        if slots <= self.batch_slots:
            return
        if self.h:
            self.lib.ref_destroy(self.h)
        self.h = self.lib.ref_create(slots, self.threads)
        if not self.h:
            raise RuntimeError("rppCreate(host) failed")
        self.batch_slots = slots

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _v(a):
        return ctypes.c_void_p(a.ctypes.data)

    def pre_emphasis_filter(self, src, sd, dst, dd, lengths, coeff, border):
        return self.lib.rppt_pre_emphasis_filter_host(self._v(src), ctypes.byref(sd), self._v(dst), ctypes.byref(dd),
                                                      _p(lengths, _I32P), _p(coeff, _F32P), int(border), self.h)

    def down_mixing(self, src, sd, dst, dd, dims, normalize):
        return self.lib.rppt_down_mixing_host(self._v(src), ctypes.byref(sd), self._v(dst), ctypes.byref(dd),
                                              _p(dims, _I32P), bool(normalize), self.h)

    def spectrogram(self, src, sd, dst, dd, lengths, center, reflect, window, nfft, power, W, hop):
        nf = max(int(dd.w if dd.layout == 5 else dd.h), 1)
        self.ensure_slots(-(-sd.n * nf * max(nfft, W) // 99532800))
        return self.lib.rppt_spectrogram_host(self._v(src), ctypes.byref(sd), self._v(dst), ctypes.byref(dd),
                                              _p(lengths, _I32P), bool(center), bool(reflect),
                                              _p(window, _F32P) if window is not None else None, int(nfft),
                                              int(power), int(W), int(hop), self.h)

    def mel_filter_bank(self, src, sd, dst, dd, dims, max_freq, min_freq, formula, num_filter, sample_rate,
                        normalize):
        return self.lib.rppt_mel_filter_bank_host(self._v(src), ctypes.byref(sd), self._v(dst), ctypes.byref(dd),
                                                  _p(dims, _I32P), float(max_freq), float(min_freq), int(formula),
                                                  int(num_filter), float(sample_rate), bool(normalize), self.h)

    def to_decibels(self, src, sd, dst, dd, patches, cutoff_db, multiplier, ref_mag):
        return self.lib.rppt_to_decibels_host(self._v(src), ctypes.byref(sd), self._v(dst), ctypes.byref(dd),
                                              patches, float(cutoff_db), float(multiplier), float(ref_mag), self.h)

    def nsr(self, src, sd, lengths, begin, length, cutoff_db, window_length, ref_power, reset_interval):
        return self.lib.rppt_non_silent_region_detection_host(self._v(src), ctypes.byref(sd), _p(lengths, _I32P),
                                                              _p(begin, _I32P), _p(length, _I32P), float(cutoff_db),
                                                              int(window_length), float(ref_power),
                                                              int(reset_interval), self.h)

    def resample(self, src, sd, dst, dd, in_rate, out_rate, dims, lut, scale, center, lobes, coeffs):
        lut = np.ascontiguousarray(lut, np.float32)
        return self.lib.ref_resample(self._v(src), ctypes.byref(sd), self._v(dst), ctypes.byref(dd),
                                     _p(in_rate, _F32P), _p(out_rate, _F32P), _p(dims, _I32P), _p(lut, _F32P),
                                     len(lut), float(scale), float(center), int(lobes), int(coeffs), self.h)


def _reference_slice(self, src, dst, anchor, shape, roi, fill, enable_padding, num_dims):
    """The reference's host slice on the same arrays as Oracle.slice (dst updated in place)."""
    from rpp_b200.types import generic_desc, RpptDataType
    dt = RpptDataType.U8 if src.dtype == np.uint8 else RpptDataType.F32
    sd = generic_desc(src.shape, dt)
    dd = generic_desc(dst.shape, dt)
    f = np.array([fill], dtype=src.dtype)
    fn = self.lib.ref_slice_u8 if src.dtype == np.uint8 else self.lib.ref_slice_f32
    st = fn(src.ctypes.data, ctypes.addressof(sd), dst.ctypes.data, ctypes.addressof(dd),
            _p(np.ascontiguousarray(anchor, np.int32), _I32P), _p(np.ascontiguousarray(shape, np.int32), _I32P),
            f.ctypes.data, bool(enable_padding), _p(np.ascontiguousarray(roi, np.uint32), _U32P), self.h)
    assert st == 0, st
    return dst


Reference.slice = _reference_slice


def _reference_slice_nd(self, src, dst, anchor, shape, roi, fill, enable_padding, layout):
    """The reference's host slice on 3-D / 4-D arrays in the given layout (dst updated in place)."""
    from rpp_b200.types import generic_desc, RpptDataType
    dt = RpptDataType.U8 if src.dtype == np.uint8 else RpptDataType.F32
    sd = generic_desc(src.shape, dt, layout)
    dd = generic_desc(dst.shape, dt, layout)
    f = np.array([fill], dtype=src.dtype)
    fn = self.lib.ref_slice_nd_u8 if src.dtype == np.uint8 else self.lib.ref_slice_nd_f32
    fn.argtypes = self.lib.ref_slice_f32.argtypes
    st = fn(src.ctypes.data, ctypes.addressof(sd), dst.ctypes.data, ctypes.addressof(dd),
            _p(np.ascontiguousarray(anchor, np.int32), _I32P), _p(np.ascontiguousarray(shape, np.int32), _I32P),
            f.ctypes.data, bool(enable_padding), _p(np.ascontiguousarray(roi, np.uint32), _U32P), self.h)
    assert st == 0, st
    return dst


Reference.slice_nd = _reference_slice_nd


def _reference_normalize_2d(self, src, dst, axis_mask, mean, std, compute, scale, shift, roi):
    """The reference's host normalize (F32, 2-D) on the same arrays as Oracle.normalize_2d."""
    from rpp_b200.types import generic_desc
    sd, dd = generic_desc(src.shape), generic_desc(dst.shape)
    L = self.lib
    L.ref_normalize_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                                    _F32P, _F32P, ctypes.c_ubyte, _F, _F, _U32P, ctypes.c_void_p]
    st = L.ref_normalize_f32(src.ctypes.data, ctypes.addressof(sd), dst.ctypes.data, ctypes.addressof(dd),
                             int(axis_mask), _p(mean, _F32P), _p(std, _F32P), int(compute), float(scale), float(shift),
                             _p(np.ascontiguousarray(roi, np.uint32), _U32P), self.h)
    assert st == 0, st
    return dst


Reference.normalize_2d = _reference_normalize_2d


def _reference_normalize_nd(self, src, dst, axis_mask, mean, std, compute, scale, shift, roi, src_layout=0,
                            dst_layout=0):
    """The reference's host normalize (F32 any rank; U8; I8 through its unsigned destination) on
    the same arrays as Oracle.normalize_nd."""
    from rpp_b200.types import generic_desc, RpptDataType
    dt = {np.dtype(np.float32): RpptDataType.F32, np.dtype(np.uint8): RpptDataType.U8,
          np.dtype(np.int8): RpptDataType.I8}
    sd, dd = generic_desc(src.shape, dt[src.dtype], src_layout), generic_desc(dst.shape, dt[dst.dtype], dst_layout)
    L = self.lib
    L.ref_normalize_nd.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                                   _F32P, _F32P, ctypes.c_ubyte, _F, _F, _U32P, ctypes.c_void_p]
    st = L.ref_normalize_nd(src.ctypes.data, ctypes.addressof(sd), dst.ctypes.data, ctypes.addressof(dd),
                            int(axis_mask), _p(mean, _F32P), _p(std, _F32P), int(compute), float(scale), float(shift),
                            _p(np.ascontiguousarray(roi, np.uint32), _U32P), self.h)
    assert st == 0, st
    return dst


Reference.normalize_nd = _reference_normalize_nd
