"""ctypes mirrors of the audio path's ABI types (include/rppdefs.h).

Layouts follow the reference's api/rppdefs.h: RpptDesc (:581-589), RpptStrides (:570-576),
RpptImagePatch (:645-649) and RpptResamplingWindow (:751-790); enum values follow
RppStatus (:121-176), RppBackend (:181-186), RpptDataType (:397-405), RpptLayout (:410-419),
RpptAudioBorderType (:464-469) and RpptMelScaleFormula (:474-478).
"""
import ctypes
import enum


class RppStatus(enum.IntEnum):
    RPP_SUCCESS = 0
    RPP_ERROR = -1
    RPP_ERROR_INVALID_ARGUMENTS = -2
    RPP_ERROR_LOW_OFFSET = -3
    RPP_ERROR_ZERO_DIVISION = -4
    RPP_ERROR_HIGH_SRC_DIMENSION = -5
    RPP_ERROR_NOT_IMPLEMENTED = -6
    RPP_ERROR_INVALID_SRC_CHANNELS = -7
    RPP_ERROR_INVALID_DST_CHANNELS = -8
    RPP_ERROR_INVALID_SRC_LAYOUT = -9
    RPP_ERROR_INVALID_DST_LAYOUT = -10
    RPP_ERROR_INVALID_SRC_DATATYPE = -11
    RPP_ERROR_INVALID_DST_DATATYPE = -12
    RPP_ERROR_INVALID_SRC_OR_DST_DATATYPE = -13
    RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH = -14
    RPP_ERROR_INVALID_PARAMETER_DATATYPE = -15
    RPP_ERROR_NOT_ENOUGH_MEMORY = -16
    RPP_ERROR_OUT_OF_BOUND_SRC_ROI = -17
    RPP_ERROR_LAYOUT_MISMATCH = -18
    RPP_ERROR_INVALID_CHANNELS = -19
    RPP_ERROR_INVALID_OUTPUT_TILE_LENGTH = -20
    RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE = -21
    RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE = -22
    RPP_ERROR_INVALID_SRC_DIMS = -23
    RPP_ERROR_INVALID_DST_DIMS = -24
    RPP_ERROR_INVALID_DIM_LENGTHS = -25
    RPP_ERROR_INVALID_AXIS = -26


class RppHandleStatus(enum.IntEnum):
    rppStatusSuccess = 0
    rppStatusBadParm = -1
    rppStatusUnknownError = -2
    rppStatusNotInitialized = -3
    rppStatusInvalidValue = -4
    rppStatusAllocFailed = -5
    rppStatusInternalError = -6
    rppStatusNotImplemented = -7
    rppStatusUnsupportedOp = -8


class RppBackend(enum.IntEnum):
    RPP_HOST_BACKEND = 0
    RPP_HIP_BACKEND = 1
    RPP_OCL_BACKEND = 2


class RpptDataType(enum.IntEnum):
    U8 = 0
    F32 = 1
    F16 = 2
    I8 = 3
    I16 = 4


class RpptLayout(enum.IntEnum):
    NCHW = 0
    NHWC = 1
    NCDHW = 2
    NDHWC = 3
    NHW = 4
    NFT = 5
    NTF = 6


class RpptAudioBorderType(enum.IntEnum):
    ZERO = 0
    CLAMP = 1
    REFLECT = 2


class RpptMelScaleFormula(enum.IntEnum):
    SLANEY = 0
    HTK = 1


class RpptStrides(ctypes.Structure):
    _fields_ = [("nStride", ctypes.c_uint32), ("cStride", ctypes.c_uint32),
                ("hStride", ctypes.c_uint32), ("wStride", ctypes.c_uint32)]


class RpptDesc(ctypes.Structure):
    _fields_ = [("numDims", ctypes.c_size_t), ("offsetInBytes", ctypes.c_uint32),
                ("dataType", ctypes.c_int), ("n", ctypes.c_uint32), ("c", ctypes.c_uint32),
                ("h", ctypes.c_uint32), ("w", ctypes.c_uint32), ("strides", RpptStrides),
                ("layout", ctypes.c_int)]


class RpptImagePatch(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class _StdVectorFloat(ctypes.Structure):
    # libstdc++ std::vector<float>: begin, end, end-of-storage pointers
    _fields_ = [("begin", ctypes.c_void_p), ("end", ctypes.c_void_p), ("cap", ctypes.c_void_p)]


class RpptResamplingWindow(ctypes.Structure):
    """Byte image of the reference's RpptResamplingWindow (96 bytes on x86-64).

    Only `lookupPinned` is used to pass the table from Python (the vector stays empty, so
    nothing on the C++ side ever frees Python memory)."""
    _fields_ = [("scale", ctypes.c_float), ("center", ctypes.c_float),
                ("lobes", ctypes.c_int32), ("coeffs", ctypes.c_int32),
                ("lookupSize", ctypes.c_int32), ("_pad0", ctypes.c_int32),
                ("lookupPinned", ctypes.c_void_p), ("lookup", _StdVectorFloat),
                ("_pad1", ctypes.c_uint8 * 8),
                ("pCenter", ctypes.c_float * 4), ("pScale", ctypes.c_float * 4)]


assert ctypes.sizeof(RpptDesc) == 56
assert ctypes.sizeof(RpptResamplingWindow) == 96
assert RpptResamplingWindow.pCenter.offset == 64


def audio_desc(n, max_len, channels=1, num_dims=2, pad_to_8=False):
    """Descriptor of a batch of 1-D (optionally interleaved multi-channel) signals.

    pad_to_8 reproduces the test suite's stride choice, w = (w/8)*8 + 8
    (utilities/test_suite/rpp_test_suite_audio.h:84-99)."""
    d = RpptDesc()
    d.numDims = num_dims
    d.offsetInBytes = 0
    d.dataType = RpptDataType.F32
    d.n, d.h, d.c = n, 1, channels
    d.w = (max_len // 8) * 8 + 8 if pad_to_8 else max_len
    d.strides.nStride = d.c * d.w * d.h
    d.strides.hStride = d.c * d.w
    d.strides.wStride = d.c
    d.strides.cStride = 1
    d.layout = RpptLayout.NFT
    return d


def spectra_desc(n, height, width, layout=RpptLayout.NFT):
    """Descriptor of a batch of 2-D spectra [height][width] per sample (numDims 3)."""
    d = RpptDesc()
    d.numDims = 3
    d.offsetInBytes = 0
    d.dataType = RpptDataType.F32
    d.n, d.c, d.h, d.w = n, 1, height, width
    d.strides.nStride = height * width
    d.strides.hStride = width
    d.strides.wStride = 1
    d.strides.cStride = 1
    d.layout = layout
    return d


class RppbFrontendParams(ctypes.Structure):
    """include/rppb_frontend.h: parameters of the fused pre-emphasis -> spectrogram -> mel -> dB call."""
    _fields_ = [("borderType", ctypes.c_int), ("centerWindows", ctypes.c_bool), ("reflectPadding", ctypes.c_bool),
                ("windowFunction", ctypes.c_void_p), ("nfft", ctypes.c_int32), ("power", ctypes.c_int32),
                ("windowLength", ctypes.c_int32), ("windowStep", ctypes.c_int32), ("maxFreq", ctypes.c_float),
                ("minFreq", ctypes.c_float), ("melFormula", ctypes.c_int), ("numFilter", ctypes.c_int32),
                ("sampleRate", ctypes.c_float), ("normalize", ctypes.c_bool), ("cutOffDB", ctypes.c_float),
                ("multiplier", ctypes.c_float), ("referenceMagnitude", ctypes.c_float),
                ("lookahead", ctypes.c_int32), ("tileFrames", ctypes.c_int32), ("dbFrames", ctypes.c_int32),
                ("ctasPerSm", ctypes.c_int32), ("spectrumEngine", ctypes.c_int32)]


assert ctypes.sizeof(RppbFrontendParams) == 88   # sizeof in C (the engine field fills the tail padding)

# RppbSpectrumEngine
ENGINE_FP32_FFT = 0
ENGINE_TENSOR_CORE_F16X3 = 1


def frontend_params(nfft=512, window_length=400, window_step=160, num_filter=128, sample_rate=16000.0,
                    min_freq=0.0, max_freq=8000.0, mel_formula=0, normalize=True, cut_off_db=-80.0,
                    multiplier=10.0, reference_magnitude=0.0, border=0, center=True, reflect=True, power=2,
                    window=None, lookahead=0, tile_frames=0, db_frames=0, ctas_per_sm=0, engine=0):
    p = RppbFrontendParams()
    p.borderType = int(border)
    p.centerWindows = bool(center)
    p.reflectPadding = bool(reflect)
    p.windowFunction = window
    p.nfft, p.power, p.windowLength, p.windowStep = int(nfft), int(power), int(window_length), int(window_step)
    p.maxFreq, p.minFreq = float(max_freq), float(min_freq)
    p.melFormula, p.numFilter, p.sampleRate, p.normalize = int(mel_formula), int(num_filter), float(sample_rate), \
        bool(normalize)
    p.cutOffDB, p.multiplier, p.referenceMagnitude = float(cut_off_db), float(multiplier), float(reference_magnitude)
    p.lookahead = int(lookahead)
    p.tileFrames, p.dbFrames, p.ctasPerSm = int(tile_frames), int(db_frames), int(ctas_per_sm)
    p.spectrumEngine = int(engine)
    return p


class RppbServerConfig(ctypes.Structure):
    """include/rppb_server.h: configuration of the continuous-batching server."""
    _fields_ = [("budgetBytes", ctypes.c_uint64), ("maxClipsPerStep", ctypes.c_int32), ("tables", ctypes.c_int32),
                ("outRate", ctypes.c_float), ("lookup", ctypes.c_void_p), ("lookupSize", ctypes.c_int32),
                ("scale", ctypes.c_float), ("center", ctypes.c_float), ("lobes", ctypes.c_int32),
                ("preemphCoeff", ctypes.c_float), ("params", RppbFrontendParams), ("plainChain", ctypes.c_int32),
                ("maxSamples", ctypes.c_int32)]


class RppbCompletion(ctypes.Structure):
    """include/rppb_server.h: one finished request (steady-clock nanoseconds)."""
    _fields_ = [("id", ctypes.c_uint64), ("submitNs", ctypes.c_int64), ("finishNs", ctypes.c_int64)]


class RpptGenericDesc(ctypes.Structure):
    """include/rppdefs.h RpptGenericDesc (api/rppdefs.h:591-602): dims[0] is the batch."""
    _fields_ = [("numDims", ctypes.c_size_t), ("offsetInBytes", ctypes.c_uint32), ("dataType", ctypes.c_int),
                ("dims", ctypes.c_uint32 * 5), ("strides", ctypes.c_uint32 * 5), ("layout", ctypes.c_int)]


def generic_desc(shape, dtype=None, layout=None):
    """Dense generic descriptor of a [n, d1, ...] tensor (numDims = len(shape))."""
    d = RpptGenericDesc()
    d.numDims = len(shape)
    d.offsetInBytes = 0
    d.dataType = int(RpptDataType.F32 if dtype is None else dtype)
    for i, v in enumerate(shape):
        d.dims[i] = int(v)
    st = 1
    for i in range(len(shape) - 1, -1, -1):
        d.strides[i] = st
        st *= int(shape[i])
    d.layout = int(RpptLayout.NCHW if layout is None else layout)
    return d
