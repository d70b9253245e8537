/*
 * rppb — B200-native drop-in for RPP's batched audio tensor path.
 *
 * ABI types of the audio path.  Every struct and enum here keeps the byte layout and the
 * numeric values of the reference's api/rppdefs.h, so code compiled against the reference
 * headers can call this library unchanged:
 *   RppStatus            api/rppdefs.h:121-176
 *   RppBackend           api/rppdefs.h:181-186
 *   rppStatus_t          api/rppdefs.h:190-202
 *   RpptDataType         api/rppdefs.h:397-405
 *   RpptLayout           api/rppdefs.h:410-419
 *   RpptAudioBorderType  api/rppdefs.h:464-469
 *   RpptMelScaleFormula  api/rppdefs.h:474-478
 *   RpptStrides          api/rppdefs.h:570-576
 *   RpptDesc             api/rppdefs.h:581-589
 *   RpptImagePatch       api/rppdefs.h:645-649
 *   RpptGenericDesc      api/rppdefs.h:591-602 (rppt_slice_gpu)
 *   RpptResamplingWindow api/rppdefs.h:751-790 (C++ only: it holds a std::vector and __m128)
 * Only the subset the audio entry points use is restated.
 */
#ifndef RPPB_RPPDEFS_H
#define RPPB_RPPDEFS_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif
#ifdef __cplusplus
#include <vector>
#if defined(__x86_64__) || defined(_M_X64)
#include <xmmintrin.h>
#endif
#endif

typedef unsigned char      Rpp8u;
typedef signed char        Rpp8s;
typedef unsigned short     Rpp16u;
typedef short              Rpp16s;
typedef unsigned int       Rpp32u;
typedef int                Rpp32s;
typedef unsigned long long Rpp64u;
typedef long long          Rpp64s;
typedef float              Rpp32f;
typedef double             Rpp64f;
typedef void*              RppPtr_t;
typedef size_t             RppSize_t;

/* Status codes returned by every rppt_* entry point (values as in the reference). */
typedef enum
{
    RPP_SUCCESS                                = 0,
    RPP_ERROR                                  = -1,
    RPP_ERROR_INVALID_ARGUMENTS                = -2,
    RPP_ERROR_LOW_OFFSET                       = -3,
    RPP_ERROR_ZERO_DIVISION                    = -4,
    RPP_ERROR_HIGH_SRC_DIMENSION               = -5,
    RPP_ERROR_NOT_IMPLEMENTED                  = -6,
    RPP_ERROR_INVALID_SRC_CHANNELS             = -7,
    RPP_ERROR_INVALID_DST_CHANNELS             = -8,
    RPP_ERROR_INVALID_SRC_LAYOUT               = -9,
    RPP_ERROR_INVALID_DST_LAYOUT               = -10,
    RPP_ERROR_INVALID_SRC_DATATYPE             = -11,
    RPP_ERROR_INVALID_DST_DATATYPE             = -12,
    RPP_ERROR_INVALID_SRC_OR_DST_DATATYPE      = -13,
    RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH   = -14,
    RPP_ERROR_INVALID_PARAMETER_DATATYPE       = -15,
    RPP_ERROR_NOT_ENOUGH_MEMORY                = -16,
    RPP_ERROR_OUT_OF_BOUND_SRC_ROI             = -17,
    RPP_ERROR_LAYOUT_MISMATCH                  = -18,
    RPP_ERROR_INVALID_CHANNELS                 = -19,
    RPP_ERROR_INVALID_OUTPUT_TILE_LENGTH       = -20,
    RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE  = -21,
    RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE = -22,
    RPP_ERROR_INVALID_SRC_DIMS                 = -23,
    RPP_ERROR_INVALID_DST_DIMS                 = -24,
    RPP_ERROR_INVALID_DIM_LENGTHS              = -25,
    RPP_ERROR_INVALID_AXIS                     = -26
} RppStatus;

/* Backend selector of rppCreate/rppDestroy.  This library implements the GPU backend only;
 * RPP_HIP_BACKEND (=1) is the value callers of the reference's GPU path already pass. */
typedef enum
{
    RPP_HOST_BACKEND,
    RPP_HIP_BACKEND,
    RPP_OCL_BACKEND
} RppBackend;

/* Status codes of the handle API. */
typedef enum
{
    rppStatusSuccess        = 0,
    rppStatusBadParm        = -1,
    rppStatusUnknownError   = -2,
    rppStatusNotInitialized = -3,
    rppStatusInvalidValue   = -4,
    rppStatusAllocFailed    = -5,
    rppStatusInternalError  = -6,
    rppStatusNotImplemented = -7,
    rppStatusUnsupportedOp  = -8
} rppStatus_t;

typedef enum
{
    U8,
    F32,
    F16,
    I8,
    I16
} RpptDataType;

typedef enum
{
    NCHW,
    NHWC,
    NCDHW,
    NDHWC,
    NHW,
    NFT,    /* batch - frequency - time: frequency-major spectra (spectrogram / mel) */
    NTF     /* batch - time - frequency: time-major spectra */
} RpptLayout;

/* Value used for the sample before the first one in pre_emphasis_filter. */
typedef enum
{
    ZERO = 0,
    CLAMP,
    REFLECT
} RpptAudioBorderType;

/* Hz <-> mel conversion used to place the mel filters. */
typedef enum
{
    SLANEY = 0,
    HTK
} RpptMelScaleFormula;

typedef struct
{
    Rpp32u nStride;
    Rpp32u cStride;
    Rpp32u hStride;
    Rpp32u wStride;
} RpptStrides;

/* Batched tensor descriptor.  Strides are in elements; offsetInBytes is carried for ABI
 * compatibility and, as in the reference audio path, not applied to the data pointers. */
typedef struct
{
    RppSize_t numDims;
    Rpp32u offsetInBytes;
    RpptDataType dataType;
    Rpp32u n, c, h, w;
    RpptStrides strides;
    RpptLayout layout;
} RpptDesc, *RpptDescPtr;

/* Per-sample 2-D extent (width = columns / frames, height = rows). */
typedef struct
{
    Rpp32u width;
    Rpp32u height;
} RpptImagePatch, *RpptImagePatchPtr;

typedef size_t RppSize_t;
#define RPPT_MAX_DIMS (5)

/* N-dimensional tensor descriptor: dims[0] is the batch, strides in elements. */
typedef struct
{
    RppSize_t numDims;
    Rpp32u offsetInBytes;
    RpptDataType dataType;
    Rpp32u dims[RPPT_MAX_DIMS];
    Rpp32u strides[RPPT_MAX_DIMS];
    RpptLayout layout;
} RpptGenericDesc, *RpptGenericDescPtr;

#ifdef __cplusplus
/* Resampling window: a lookup table of the windowed-sinc kernel, sampled so that
 * lookup[x * scale + center] is the weight of an input sample x input periods away from
 * the output position, with `lobes` zero crossings on each side.  The GPU entry point reads
 * lookupPinned when it is set (pinned or device memory, as the reference's GPU path does)
 * and otherwise lookup.data().  Layout identical to the reference, including the std::vector
 * and the two __m128 members, so it can be passed by reference across the C ABI. */
typedef struct RpptResamplingWindow
{
    inline void input_range(Rpp32f x, Rpp32s *loc0, Rpp32s *loc1)
    {
        Rpp32s xc = (Rpp32s)__builtin_ceilf(x);
        *loc0 = xc - lobes;
        *loc1 = xc + lobes;
    }

    Rpp32f scale = 1, center = 1;
    Rpp32s lobes = 0, coeffs = 0;
    Rpp32s lookupSize = 0;
    Rpp32f *lookupPinned = nullptr;
    std::vector<Rpp32f> lookup;
#if defined(__x86_64__) || defined(_M_X64)
    __m128 pCenter, pScale;
#else
    alignas(16) float pCenter[4];
    alignas(16) float pScale[4];
#endif
} RpptResamplingWindow;
#endif

#endif /* RPPB_RPPDEFS_H */
