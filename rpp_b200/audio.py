"""Python front of the B200 audio path, mirroring the reference's rppt_* audio interface.

Each function takes the same arguments as the reference's C entry point (descriptors, per-sample
tensors, scalars, handle) and returns its RppStatus; tensors are torch CUDA tensors (or pinned /
host tensors for the per-sample arguments, as the C API allows) or raw integer addresses.  The
call goes straight through the C ABI of librppb.so (rpp_b200/lib.py); nothing here computes.
"""
import ctypes

from . import lib as _lib
from .types import RpptImagePatch, RpptResamplingWindow, RppStatus


def _addr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if isinstance(t, ctypes.Array):
        return ctypes.addressof(t)
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    if hasattr(t, "ctypes"):
        return t.ctypes.data
    raise TypeError(f"cannot take the address of {type(t)}")


def _h(handle):
    return handle.value if hasattr(handle, "value") else handle


def _status(v):
    try:
        return RppStatus(v)
    except ValueError:
        return v


def non_silent_region_detection(src, src_desc, src_length, detected_index, detection_length, cut_off_db,
                                window_length, reference_power, reset_interval, handle):
    L = _lib.load()
    return _status(L.rppt_non_silent_region_detection_gpu(
        _addr(src), ctypes.byref(src_desc), _addr(src_length), _addr(detected_index), _addr(detection_length),
        float(cut_off_db), int(window_length), float(reference_power), int(reset_interval), _h(handle)))


def to_decibels(src, src_desc, dst, dst_desc, src_dims, cut_off_db, multiplier, reference_magnitude, handle):
    L = _lib.load()
    return _status(L.rppt_to_decibels_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                          _addr(src_dims), float(cut_off_db), float(multiplier),
                                          float(reference_magnitude), _h(handle)))


def pre_emphasis_filter(src, src_desc, dst, dst_desc, src_length, coeff, border_type, handle):
    L = _lib.load()
    return _status(L.rppt_pre_emphasis_filter_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst),
                                                  ctypes.byref(dst_desc), _addr(src_length), _addr(coeff),
                                                  int(border_type), _h(handle)))


def down_mixing(src, src_desc, dst, dst_desc, src_dims, normalize_weights, handle):
    L = _lib.load()
    return _status(L.rppt_down_mixing_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                          _addr(src_dims), bool(normalize_weights), _h(handle)))


def spectrogram(src, src_desc, dst, dst_desc, src_length, center_windows, reflect_padding, window_function, nfft,
                power, window_length, window_step, handle):
    L = _lib.load()
    return _status(L.rppt_spectrogram_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                          _addr(src_length), bool(center_windows), bool(reflect_padding),
                                          _addr(window_function), int(nfft), int(power), int(window_length),
                                          int(window_step), _h(handle)))


def mel_filter_bank(src, src_desc, dst, dst_desc, src_dims, max_freq, min_freq, mel_formula, num_filter,
                    sample_rate, normalize, handle):
    L = _lib.load()
    return _status(L.rppt_mel_filter_bank_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                              _addr(src_dims), float(max_freq), float(min_freq), int(mel_formula),
                                              int(num_filter), float(sample_rate), bool(normalize), _h(handle)))


def resampling_window(lut, scale, center, lobes, coeffs=None):
    """RpptResamplingWindow whose lookupPinned points at `lut` (a torch tensor, pinned or device,
    or a host array kept alive by the caller)."""
    w = RpptResamplingWindow()
    w.scale = float(scale)
    w.center = float(center)
    w.lobes = int(lobes)
    w.coeffs = int(coeffs if coeffs is not None else len(lut) - 5)
    w.lookupSize = int(len(lut))
    w.lookupPinned = _addr(lut)
    for i in range(4):
        w.pCenter[i] = w.center
        w.pScale[i] = w.scale
    return w


def resample(src, src_desc, dst, dst_desc, in_rate, out_rate, src_dims, window, handle):
    L = _lib.load()
    return _status(L.rppt_resample_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                       _addr(in_rate), _addr(out_rate), _addr(src_dims), ctypes.byref(window),
                                       _h(handle)))


def image_patches(widths, heights):
    """Host array of RpptImagePatch {width, height} (keep it alive during the call)."""
    arr = (RpptImagePatch * len(widths))()
    for i, (w, h) in enumerate(zip(widths, heights)):
        arr[i].width = int(w)
        arr[i].height = int(h)
    return arr


def frontend(src, src_desc, dst, dst_desc, src_length, coeff, params, handle):
    """rppb_frontend_gpu: the fused pre-emphasis -> spectrogram -> mel -> decibels chain."""
    L = _lib.load()
    return _status(L.rppb_frontend_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                       _addr(src_length), _addr(coeff), ctypes.byref(params), _h(handle)))


def frontend_host(src, src_desc, dst, dst_desc, src_length, coeff, params, num_chunks, handle):
    """rppb_frontend_host_gpu: the fused chain on host tensors (pinned for overlap), chunked so that
    copies in, kernels and copies out overlap.  Asynchronous on the handle stream."""
    L = _lib.load()
    return _status(L.rppb_frontend_host_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                            _addr(src_length), _addr(coeff), ctypes.byref(params), int(num_chunks),
                                            _h(handle)))


def frontend_tune(src, src_desc, dst, dst_desc, src_length, coeff, params, handle, reps=3):
    """rppb_frontend_tune_gpu: times the schedule candidates of rppb_frontend_gpu on this batch and
    writes the fastest into `params` (in place).  Returns (status, best ms)."""
    L = _lib.load()
    ms = ctypes.c_float(0.0)
    st = L.rppb_frontend_tune_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                  _addr(src_length), _addr(coeff), ctypes.byref(params), int(reps), ctypes.byref(ms),
                                  _h(handle))
    return _status(st), ms.value


def slice(src, src_desc, dst, dst_desc, anchor, shape, fill_value, enable_padding, roi, handle):
    """rppt_slice_gpu (api/rppt_tensor_geometric_augmentations.h:486); fill_value: a one-element
    array or tensor of the data type (host, pinned or device)."""
    L = _lib.load()
    return _status(L.rppt_slice_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                    _addr(anchor), _addr(shape), _addr(fill_value), bool(enable_padding), _addr(roi),
                                    _h(handle)))


def normalize(src, src_desc, dst, dst_desc, axis_mask, mean, std_dev, compute_mean_stddev, scale, shift, roi, handle):
    """rppt_normalize_gpu (api/rppt_tensor_statistical_operations.h:193): U8 / F16 / F32 / I8, ranks 1-4."""
    L = _lib.load()
    return _status(L.rppt_normalize_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                        int(axis_mask), _addr(mean), _addr(std_dev), int(compute_mean_stddev),
                                        float(scale), float(shift), _addr(roi), _h(handle)))


def pcm16_to_f32(src, src_desc, dst, dst_desc, src_length, handle):
    """rppb_pcm16_to_f32_gpu: int16 PCM (interleaved channels) to float / 32768 on the device."""
    L = _lib.load()
    return _status(L.rppb_pcm16_to_f32_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                           _addr(src_length), _h(handle)))


def mel_filter_bank_tc(src, src_desc, dst, dst_desc, src_dims, max_freq, min_freq, mel_formula, num_filter,
                       sample_rate, normalize, precision, handle):
    """rppb_mel_filter_bank_tc_gpu: the mel filter bank as a tensor-core GEMM (precision study)."""
    L = _lib.load()
    return _status(L.rppb_mel_filter_bank_tc_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst),
                                                 ctypes.byref(dst_desc), _addr(src_dims), float(max_freq),
                                                 float(min_freq), int(mel_formula), int(num_filter), float(sample_rate),
                                                 bool(normalize), int(precision), _h(handle)))


def device_error(handle):
    """Reads and clears the handle's device error word (synchronizes the handle stream)."""
    L = _lib.load()
    v = ctypes.c_int32(0)
    st = L.rppb_get_device_error(_h(handle), ctypes.byref(v))
    if st != 0:
        raise RuntimeError(f"rppb_get_device_error failed with status {st}")
    return v.value


def set_wait_fault_injection(handle, enable):
    """rppb_set_wait_fault_injection (test hook): the fused front end's decibel items wait for a tile
    that is never counted and give up after ~0.1 ms, setting the device error word."""
    L = _lib.load()
    return _status(L.rppb_set_wait_fault_injection(_h(handle), bool(enable)))


def set_tc_materialized_frames(handle, materialize):
    """rppb_set_tc_materialized_frames: the tensor-core spectrogram writes frame rows out instead of
    reading overlapping rows through its tensor map (same bits)."""
    L = _lib.load()
    return _status(L.rppb_set_tc_materialized_frames(_h(handle), bool(materialize)))


def downmix_resample(src, src_desc, dst, dst_desc, in_rate, out_rate, src_dims, normalize_weights, lut, scale, center,
                     lobes, handle):
    """rppb_downmix_resample_gpu: down-mix to mono and resample in one launch."""
    L = _lib.load()
    return _status(L.rppb_downmix_resample_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                               _addr(in_rate), _addr(out_rate), _addr(src_dims),
                                               bool(normalize_weights), _addr(lut), int(len(lut)), float(scale),
                                               float(center), int(lobes), _h(handle)))


TC_BF16, TC_BF16_HILO3, TC_TF32, TC_FP8_E4M3 = 0, 1, 2, 3   # RppbTensorCorePrecision


def spectrogram_tc(src, src_desc, dst, dst_desc, src_length, coeff, border_type, center_windows, reflect_padding, nfft,
                   power, window_length, window_step, precision, handle):
    """rppb_spectrogram_tc_gpu: the tensor-core spectrogram of the precision study (precision: one of
    TC_BF16, TC_BF16_HILO3, TC_TF32, TC_FP8_E4M3)."""
    L = _lib.load()
    return _status(L.rppb_spectrogram_tc_gpu(_addr(src), ctypes.byref(src_desc), _addr(dst), ctypes.byref(dst_desc),
                                             _addr(src_length), _addr(coeff), int(border_type), bool(center_windows),
                                             bool(reflect_padding), int(nfft), int(power), int(window_length),
                                             int(window_step), int(precision), _h(handle)))
