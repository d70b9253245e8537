/*
 * rppb — the normalize entry point of the reference's statistical operations, the step after the
 * audio front end in RNN-T-style pipelines (per-feature mean / std-dev normalisation of the
 * decibel spectra).
 *
 * Replaces api/rppt_tensor_statistical_operations.h:193 (rppt_normalize_gpu), same arguments:
 *  - srcPtr/dstPtr device memory; U8 -> U8, F16 -> F16, F32 -> F32 or I8 -> I8 (other pairs:
 *    RPP_ERROR_NOT_IMPLEMENTED); generic descriptors with numDims 2 to 5 (tensors of rank 1-4);
 *  - axisMask: bit i reduces over dimension i (e.g. 2-D: 1 one parameter per column, 2 one per
 *    row, such as per mel filter over time, 3 one per sample); 0 or bits beyond the rank give
 *    RPP_ERROR_INVALID_ARGUMENTS;
 *  - roiTensor: n * rank * 2 (begins, then lengths), device, pinned or pageable (read on the host);
 *  - computeMeanStddev bit 0 / bit 1: the mean / inverse std dev are computed and written to
 *    meanTensor / stdDevTensor (n x maxSize, maxSize = the largest parameter count of a sample);
 *    a clear bit reads the caller's values; both clear: one shared set of maxSize means and std
 *    devs, the std devs turned into scale / stdDev (1 where 0) without changing the caller's array.
 * The three branches of the reference host path (src/modules/tensor/cpu/kernel/normalize.cpp):
 *  - F32, rank 2 (:417-600): the roi begins are not read; the destination sample is zeroed, then
 *    (x - mean) * invStdDev + shift over the roi;
 *  - F32, rank 3 (:592-730): statistics over the roi from its first two begins; the result is
 *    written for NHWC -> NHWC (any mask) and NHWC -> NCHW (mask 3) only, other layout pairs get
 *    a zeroed destination and the statistics;
 *  - every other type and rank (:731-868): consecutive normalized dimensions are merged as the
 *    reference merges them, the roi is read as a dense block of its lengths from its begin offset
 *    and written densely from the sample start, and the sums are added to the values already in
 *    meanTensor / stdDevTensor (pass zeros for plain statistics); a roi whose block does not fit
 *    the sample gives RPP_ERROR_INVALID_ARGUMENTS.
 * The sums follow the reference's recursive halving tree in its order, bit for bit; the inverse
 * square root is correctly rounded where the reference refines an SSE/AVX estimate (~1e-7 relative
 * apart).  Results are stored as the destination type: U8 / I8 clamped to their range, then
 * truncated (the reference host path truncates too; its out-of-range conversion is undefined),
 * F16 rounded to nearest even; I8 values are read and written as signed numbers, as the
 * reference's GPU path does (its host path reads them through an unsigned cast).
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
