/*
 * rppb — the normalize entry point of the reference's statistical operations, the step after the
 * audio front end in RNN-T-style pipelines (per-feature mean / std-dev normalisation of the
 * decibel spectra).
 *
 * Replaces api/rppt_tensor_statistical_operations.h:193 (rppt_normalize_gpu), same arguments:
 *  - srcPtr/dstPtr device memory, F32; generic descriptors with numDims 3 (a batch of 2-D
 *    tensors, e.g. [n][filters][frames]); other types and ranks return RPP_ERROR_NOT_IMPLEMENTED;
 *  - axisMask: 1 reduces over dimension 0 (one parameter per column), 2 over dimension 1 (one
 *    per row, e.g. per mel filter over time), 3 over both (one per sample); others give
 *    RPP_ERROR_INVALID_ARGUMENTS;
 *  - roiTensor: n * 4 (begin0, begin1, length0, length1), device, pinned or pageable (read on the
 *    host); the begins are not read, as in the reference host path;
 *  - computeMeanStddev bit 0 / bit 1: the mean / inverse std dev are computed and written to
 *    meanTensor / stdDevTensor (n x maxSize, maxSize = the largest parameter count of a sample);
 *    a clear bit reads the caller's values; both clear: one shared set of maxSize means and std
 *    devs, the std devs turned into scale / stdDev (1 where 0) without changing the caller's array.
 * Output: the destination sample is zeroed, then (x - mean) * invStdDev + shift over the roi.  The
 * sums follow the reference host path's recursive halving tree bit for bit
 * (src/modules/tensor/cpu/kernel/normalize.cpp:29-120, :417-600); the inverse square root is
 * correctly rounded where the reference refines the SSE estimate (~1e-7 relative apart).
 * Synchronization: the roi lengths size the work list on the host, so unless roiTensor is pageable
 * host memory the call first synchronizes the handle stream (a device roiTensor is copied back; a
 * pinned or managed one is read once earlier work on the stream, which may have written it, is
 * done).  This is the one call of the library that synchronizes; everything after the roi read is
 * asynchronous on the handle stream.
 */
#ifndef RPPB_RPPT_TENSOR_STATISTICAL_OPERATIONS_H
#define RPPB_RPPT_TENSOR_STATISTICAL_OPERATIONS_H

#include "rpp.h"
#include "rppdefs.h"

#ifdef __cplusplus
extern "C" {
#endif

SHARED_PUBLIC RppStatus rppt_normalize_gpu(RppPtr_t srcPtr, RpptGenericDescPtr srcGenericDescPtr, RppPtr_t dstPtr,
                                           RpptGenericDescPtr dstGenericDescPtr, Rpp32u axisMask, Rpp32f* meanTensor,
                                           Rpp32f* stdDevTensor, Rpp8u computeMeanStddev, Rpp32f scale, Rpp32f shift,
                                           Rpp32u* roiTensor, rppHandle_t rppHandle);

#ifdef __cplusplus
}
#endif

#endif
