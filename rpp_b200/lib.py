"""ctypes binding of rpp_b200/librppb.so — the same C ABI a C/C++ caller of the reference links.

Loading fails loudly when the library is missing: there is no CPU fallback.  Build it with
``python -m rpp_b200.build`` (or ``__graft_entry__.build()``).
"""
import ctypes
import os

from .types import (RpptGenericDesc, RpptDesc, RpptImagePatch, RpptResamplingWindow, RppBackend, RppbFrontendParams, RppbServerConfig,
                    RppbCompletion)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "librppb.so")
# The checked build (`python -m rpp_b200.build --checked`): every global access of the kernels checked against
# the regions of its call.  RPPB_LIBRARY=checked loads it instead of LIB_PATH; RPPB_LIBRARY=<path> loads <path>.
CHECKED_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "librppb_checked.so")

# Every symbol the public headers (include/*.h) declare.
EXPORTED = (
    "rppCreate", "rppDestroy", "rppSetBatchSize", "rppGetBatchSize", "rppSetStream", "rppGetStream",
    "rppSetAllocator", "rppGetKernelTime", "rppEnableProfiling",
    "rppt_non_silent_region_detection_gpu", "rppt_to_decibels_gpu", "rppt_pre_emphasis_filter_gpu",
    "rppt_down_mixing_gpu", "rppt_spectrogram_gpu", "rppt_mel_filter_bank_gpu", "rppt_resample_gpu",
    "rppbGetLastError", "rppbGetLaunchCount", "rppb_frontend_gpu", "rppb_get_device_error", "rppb_set_wait_fault_injection",
    "rppb_downmix_resample_gpu", "rppt_to_decibels_gpu_static", "rppb_frontend_clips_gpu",
    "rppb_spectrogram_tc_gpu", "rppb_set_tc_materialized_frames",
    "rppb_frontend_host_gpu", "rppb_frontend_tune_gpu",
    "rppb_server_create", "rppb_server_destroy", "rppb_server_frames", "rppb_server_submit", "rppb_server_poll",
    "rppb_server_arena_used",
    "rppt_slice_gpu", "rppt_normalize_gpu", "rppb_pcm16_to_f32_gpu", "rppb_mel_filter_bank_tc_gpu",
    "rppb_check_shrink_next_tensors",
)

_lib = None

_V = ctypes.c_void_p
_D = ctypes.POINTER(RpptDesc)
_I = ctypes.c_int
_F = ctypes.c_float
_B = ctypes.c_bool


def load(path=None):
    """Loads the library once and declares every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    env = os.environ.get("RPPB_LIBRARY", "")
    p = path or (CHECKED_LIB_PATH if env == "checked" else env) or LIB_PATH
    if not os.path.isfile(p):
        raise FileNotFoundError(f"{p} is missing: build it with `python -m rpp_b200.build` (no CPU fallback)")
    L = ctypes.CDLL(p)
    L.rppCreate.argtypes = [ctypes.POINTER(_V), ctypes.c_size_t, ctypes.c_uint, _V, _I]
    L.rppDestroy.argtypes = [_V, _I]
    L.rppSetBatchSize.argtypes = [_V, ctypes.c_size_t]
    L.rppGetBatchSize.argtypes = [_V, ctypes.POINTER(ctypes.c_size_t)]
    L.rppSetStream.argtypes = [_V, _V]
    L.rppGetStream.argtypes = [_V, ctypes.POINTER(_V)]
    L.rppSetAllocator.argtypes = [_V, _V, _V, _V]
    L.rppGetKernelTime.argtypes = [_V, ctypes.POINTER(_F)]
    L.rppEnableProfiling.argtypes = [_V, _B]
    for f in ("rppCreate", "rppDestroy", "rppSetBatchSize", "rppGetBatchSize", "rppSetStream", "rppGetStream",
              "rppSetAllocator", "rppGetKernelTime", "rppEnableProfiling"):
        getattr(L, f).restype = _I
    L.rppt_non_silent_region_detection_gpu.argtypes = [_V, _D, _V, _V, _V, _F, _I, _F, _I, _V]
    L.rppt_to_decibels_gpu.argtypes = [_V, _D, _V, _D, _V, _F, _F, _F, _V]
    L.rppt_pre_emphasis_filter_gpu.argtypes = [_V, _D, _V, _D, _V, _V, _I, _V]
    L.rppt_down_mixing_gpu.argtypes = [_V, _D, _V, _D, _V, _B, _V]
    L.rppt_spectrogram_gpu.argtypes = [_V, _D, _V, _D, _V, _B, _B, _V, _I, _I, _I, _I, _V]
    L.rppt_mel_filter_bank_gpu.argtypes = [_V, _D, _V, _D, _V, _F, _F, _I, _I, _F, _B, _V]
    L.rppt_resample_gpu.argtypes = [_V, _D, _V, _D, _V, _V, _V, ctypes.POINTER(RpptResamplingWindow), _V]
    for f in ("rppt_non_silent_region_detection_gpu", "rppt_to_decibels_gpu", "rppt_pre_emphasis_filter_gpu",
              "rppt_down_mixing_gpu", "rppt_spectrogram_gpu", "rppt_mel_filter_bank_gpu", "rppt_resample_gpu"):
        getattr(L, f).restype = _I
    L.rppb_frontend_gpu.argtypes = [_V, _D, _V, _D, _V, _V, ctypes.POINTER(RppbFrontendParams), _V]
    L.rppb_frontend_gpu.restype = _I
    L.rppb_downmix_resample_gpu.argtypes = [_V, _D, _V, _D, _V, _V, _V, _B, _V, _I, _F, _F, _I, _V]
    L.rppb_downmix_resample_gpu.restype = _I
    L.rppb_frontend_clips_gpu.argtypes = [_V, _I, _F, _V, _I, _F, _F, _I, _F, ctypes.POINTER(RppbFrontendParams), _V]
    L.rppb_frontend_clips_gpu.restype = _I
    L.rppb_frontend_host_gpu.argtypes = [_V, _D, _V, _D, _V, _V, ctypes.POINTER(RppbFrontendParams), _I, _V]
    L.rppb_frontend_host_gpu.restype = _I
    L.rppb_frontend_tune_gpu.argtypes = [_V, _D, _V, _D, _V, _V, ctypes.POINTER(RppbFrontendParams), _I,
                                         ctypes.POINTER(ctypes.c_float), _V]
    L.rppb_frontend_tune_gpu.restype = _I
    L.rppb_spectrogram_tc_gpu.argtypes = [_V, _D, _V, _D, _V, _V, _I, _B, _B, _I, _I, _I, _I, _I, _V]
    L.rppb_spectrogram_tc_gpu.restype = _I
    L.rppt_to_decibels_gpu_static.argtypes = [_V, _D, _V, _D, _V, _F, _F, _F, _V]
    L.rppt_to_decibels_gpu_static.restype = _I
    L.rppt_slice_gpu.argtypes = [_V, ctypes.POINTER(RpptGenericDesc), _V, ctypes.POINTER(RpptGenericDesc), _V, _V, _V,
                                 _B, _V, _V]
    L.rppt_slice_gpu.restype = _I
    L.rppt_normalize_gpu.argtypes = [_V, ctypes.POINTER(RpptGenericDesc), _V, ctypes.POINTER(RpptGenericDesc),
                                     ctypes.c_uint32, _V, _V, ctypes.c_uint8, _F, _F, _V, _V]
    L.rppt_normalize_gpu.restype = _I
    L.rppb_pcm16_to_f32_gpu.argtypes = [_V, _D, _V, _D, _V, _V]
    L.rppb_pcm16_to_f32_gpu.restype = _I
    L.rppb_mel_filter_bank_tc_gpu.argtypes = [_V, _D, _V, _D, _V, _F, _F, _I, _I, _F, _B, _I, _V]
    L.rppb_mel_filter_bank_tc_gpu.restype = _I
    L.rppb_check_shrink_next_tensors.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    L.rppb_check_shrink_next_tensors.restype = _I
    L.rppb_server_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(RppbServerConfig)]
    L.rppb_server_create.restype = _I
    L.rppb_server_destroy.argtypes = [_V]
    L.rppb_server_destroy.restype = _I
    L.rppb_server_frames.argtypes = [_V, ctypes.c_int32, _F]
    L.rppb_server_frames.restype = ctypes.c_int32
    L.rppb_server_submit.argtypes = [_V, _V, _V, _V, _V, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]
    L.rppb_server_submit.restype = _I
    L.rppb_server_poll.argtypes = [_V, ctypes.POINTER(RppbCompletion), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
    L.rppb_server_poll.restype = _I
    L.rppb_server_arena_used.argtypes = [_V]
    L.rppb_server_arena_used.restype = ctypes.c_uint64
    L.rppb_get_device_error.argtypes = [_V, ctypes.POINTER(ctypes.c_int32)]
    L.rppb_get_device_error.restype = _I
    L.rppb_set_wait_fault_injection.argtypes = [_V, _B]
    L.rppb_set_wait_fault_injection.restype = _I
    L.rppb_set_tc_materialized_frames.argtypes = [_V, _B]
    L.rppb_set_tc_materialized_frames.restype = _I
    L.rppbGetLaunchCount.argtypes = []
    L.rppbGetLaunchCount.restype = ctypes.c_longlong
    L.rppbGetLastError.argtypes = []
    L.rppbGetLastError.restype = ctypes.c_char_p
    _lib = L
    return L


def last_error():
    return load().rppbGetLastError().decode()


class Handle:
    """rppCreate/rppDestroy around a CUDA stream (an int handle, e.g. torch's stream.cuda_stream)."""

    def __init__(self, batch_size=1, stream=0):
        L = load()
        h = _V()
        st = L.rppCreate(ctypes.byref(h), batch_size, 0, _V(stream), int(RppBackend.RPP_HIP_BACKEND))
        if st != 0:
            raise RuntimeError(f"rppCreate failed with status {st}")
        self.ptr = h

    def set_stream(self, stream):
        st = load().rppSetStream(self.ptr, _V(stream))
        if st != 0:
            raise RuntimeError(f"rppSetStream failed with status {st}")

    @property
    def value(self):
        return self.ptr

    def close(self):
        if self.ptr:
            load().rppDestroy(self.ptr, int(RppBackend.RPP_HIP_BACKEND))
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
