/*
 * rppb — the slice entry point of the reference's geometric augmentations, the step of the audio
 * pipeline that cuts each clip's detected region (non_silent_region_detection's begin/length)
 * before the front end.
 *
 * Replaces api/rppt_tensor_geometric_augmentations.h:486 (rppt_slice_gpu), same arguments:
 *  - srcPtr/dstPtr device memory; F32 -> F32 or U8 -> U8 (other types: the reference's
 *    RPP_ERROR_INVALID_SRC/DST_DATATYPE; different types: RPP_ERROR_NOT_IMPLEMENTED);
 *  - generic descriptors with numDims 2 (a batch of 1-D signals) or 3 (a batch of 2-D tensors,
 *    e.g. spectra), any layout; numDims 4 (images, NCHW or NHWC) or 5 (volumes, NCDHW or NDHWC),
 *    other layouts of those returning RPP_ERROR_NOT_IMPLEMENTED; layouts must match
 *    (RPP_ERROR_LAYOUT_MISMATCH);
 *  - 3-D / 4-D: the box covers the spatial dims (H, W or D, H, W; the channel entries of anchor,
 *    shape and roi are not read), every channel is copied; channel-first layouts step the
 *    destination by the source's channel stride between channels, as the reference does.  Both
 *    tensors must hold the same channels, contiguous rows (channel-last: rows of width x channels
 *    elements), and destination strides that nest (each at least the next dim's extent);
 *    otherwise RPP_ERROR_INVALID_ARGUMENTS.  Boxes are clipped to the destination's dims too;
 *  - anchorTensor, shapeTensor (n * (numDims - 1)) and roiTensor (n * (numDims - 1) * 2: begins,
 *    then lengths; the begins are not read, as in the reference host path) may be device, pinned
 *    or pageable memory; fillValue points to one element of the tensor's type.
 * Per sample: the box [anchor, anchor + min(shape, length - anchor)) is copied to the start of
 * the destination sample; if any anchor + shape exceeds the length and enablePadding is set, the
 * first dstStride0 - 1 elements of the sample are filled first (the reference host path's
 * src/modules/tensor/cpu/kernel/slice.cpp:61-228, results equal bit for bit).  Asynchronous on
 * the handle stream.
 */
#ifndef RPPB_RPPT_TENSOR_GEOMETRIC_AUGMENTATIONS_H
#define RPPB_RPPT_TENSOR_GEOMETRIC_AUGMENTATIONS_H

#include "rpp.h"
#include "rppdefs.h"

#ifdef __cplusplus
extern "C" {
#endif

SHARED_PUBLIC RppStatus rppt_slice_gpu(RppPtr_t srcPtr, RpptGenericDescPtr srcGenericDescPtr, RppPtr_t dstPtr,
                                       RpptGenericDescPtr dstGenericDescPtr, Rpp32s* anchorTensor,
                                       Rpp32s* shapeTensor, RppPtr_t fillValue, bool enablePadding,
                                       Rpp32u* roiTensor, rppHandle_t rppHandle);

#ifdef __cplusplus
}
#endif

#endif
