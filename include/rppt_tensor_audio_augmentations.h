/*
 * rppb — the seven GPU audio entry points.
 *
 * Each prototype is the reference's `rppt_<op>_gpu` from api/rppt_tensor_audio_augmentations.h,
 * with the same argument order, types and meaning; the line each one replaces is cited.
 *
 * Conventions shared by every entry point (reference: api/rppt_tensor_audio_augmentations.h
 * parameter docs and src/modules/tensor/rppt_tensor_audio_augmentations.cpp:332-629):
 *  - srcPtr/dstPtr are device memory; data type F32 only.
 *  - Per-sample tensors (lengths, dims, coefficients, rates, NSR outputs) may be device memory,
 *    pinned host memory, or pageable host memory (pageable inputs are staged through the
 *    handle; pageable NSR outputs are written back by a stream-ordered copy, so read them after
 *    synchronizing the handle stream).
 *  - Every call is asynchronous on the handle's stream: no call synchronizes the stream
 *    (the reference's spectrogram and to_decibels synchronize internally; these do not).
 *  - Outputs are written only inside each sample's valid region (mel_filter_bank also zeroes
 *    up to 8 columns past the valid frames, as the reference host path does).
 *  - Status codes match the reference's GPU dispatch for the same invalid inputs; CUDA errors
 *    return RPP_ERROR and never exit the process.
 */
#ifndef RPPB_RPPT_TENSOR_AUDIO_AUGMENTATIONS_H
#define RPPB_RPPT_TENSOR_AUDIO_AUGMENTATIONS_H

#include "rpp.h"
#include "rppdefs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Non-silent region: moving mean square over windowLength samples, restarted every
 * resetInterval samples (-1: never), cutoff = (referencePower, or the per-sample maximum when
 * it is 0) * 10^(cutOffDB/10); outputs the first index and length of the region whose power is
 * at or above the cutoff, the begin moved back by windowLength-1.
 * srcDesc numDims = 2.  resetInterval must be -1 or > 0 (0 would never terminate in the
 * reference and is rejected with RPP_ERROR_INVALID_ARGUMENTS).
 * Replaces api/rppt_tensor_audio_augmentations.h:86. */
SHARED_PUBLIC RppStatus rppt_non_silent_region_detection_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, Rpp32s *srcLengthTensor,
                                                             Rpp32s *detectedIndexTensor, Rpp32s *detectionLengthTensor,
                                                             Rpp32f cutOffDB, Rpp32s windowLength, Rpp32f referencePower,
                                                             Rpp32s resetInterval, rppHandle_t rppHandle);

/* y = multiplier * log10(max(10^(cutOffDB/multiplier), x / ref)); ref = referenceMagnitude, or
 * the per-sample maximum over the srcDims ROI when it is 0.  srcDims[i].width == 1 means a 1-D
 * sample of srcDims[i].height contiguous values; otherwise height rows of width values at
 * hStride.  Replaces api/rppt_tensor_audio_augmentations.h:122. */
SHARED_PUBLIC RppStatus rppt_to_decibels_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                             RpptImagePatchPtr srcDims, Rpp32f cutOffDB, Rpp32f multiplier,
                                             Rpp32f referenceMagnitude, rppHandle_t rppHandle);

/* Allocation-free to_decibels for callers that cannot allocate device memory: code running inside
 * another runtime's memory pool or under a fixed device-memory budget, real-time audio threads that
 * must not block on cudaMalloc (it can synchronize the device and take driver locks), and callers
 * without an rppHandle_t (creating one sets up a workspace).  No counterpart in the reference.
 *
 * Same arguments and results as rppt_to_decibels_gpu, except that it takes the CUDA stream directly
 * instead of a handle, srcDims must be in device or pinned memory, and it allocates nothing: its
 * scratch (work list and per-sample maxima, ~98 KB) is a fixed array inside the library that every
 * GPU loading the library holds until the process exits.  Limit: at most 8192 samples per call;
 * larger batches return RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE (split them).  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress, with that device current): make
 * that first call before any stream capture.  All calls share the one array, so calls that can run
 * on the GPU at the same time (different streams, overlapping graphs) race: order them on one
 * stream or with events.  Launch failures are read right after each launch; a CUDA error that earlier
 * work left pending on the calling thread makes the call return RPP_ERROR without launching (the
 * error is left in place for its owner). */
SHARED_PUBLIC RppStatus rppt_to_decibels_gpu_static(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                    RpptDescPtr dstDescPtr, RpptImagePatchPtr srcDims, Rpp32f cutOffDB,
                                                    Rpp32f multiplier, Rpp32f referenceMagnitude,
                                                    rppAcceleratorQueue_t stream);

/* y[0] = x[0] - coeff * border, y[i] = x[i] - coeff * x[i-1] for 0 < i < length, with border
 * 0 (ZERO), x[0] (CLAMP) or x[1] (REFLECT).  srcDesc numDims = 2.
 * Replaces api/rppt_tensor_audio_augmentations.h:156. */
SHARED_PUBLIC RppStatus rppt_pre_emphasis_filter_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                                     Rpp32s *srcLengthTensor, Rpp32f *coeffTensor,
                                                     RpptAudioBorderType borderType, rppHandle_t rppHandle);

/* Mono mix of interleaved channels with equal weights 1/channels (normalized to sum 1 when
 * normalizeWeights).  srcDimsTensor = {length, channels} per sample.
 * Replaces api/rppt_tensor_audio_augmentations.h:188. */
SHARED_PUBLIC RppStatus rppt_down_mixing_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                             Rpp32s *srcDimsTensor, bool normalizeWeights, rppHandle_t rppHandle);

/* Short-time power (power == 2) or magnitude (power == 1) spectrum of each sample: frames of
 * windowLength samples every windowStep samples, centred on multiples of windowStep when
 * centerWindows (reflect or zero padding at the edges), multiplied by windowFunction (host
 * pointer; nullptr = Hann), placed in the middle of an nfft-point buffer (nfft 0 = windowLength)
 * and transformed.  dst is NFT [nfft/2+1][frames] or NTF [frames][nfft/2+1] per sample.
 * srcDesc numDims = 2, dstDesc numDims = 3.  A CTA stages a tile of frames with their input span in
 * shared memory: for nfft 2048 with a window and step of over ~1000 samples the tile does not fit, and
 * the call returns RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE.  Replaces
 * api/rppt_tensor_audio_augmentations.h:232. */
SHARED_PUBLIC RppStatus rppt_spectrogram_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                             Rpp32s *srcLengthTensor, bool centerWindows, bool reflectPadding,
                                             Rpp32f *windowFunction, Rpp32s nfft, Rpp32s power, Rpp32s windowLength,
                                             Rpp32s windowStep, rppHandle_t rppHandle);

/* Mel filter bank over an NFT spectrum: numFilter triangular filters evenly spaced on the
 * mel scale between minFreq and maxFreq (0 = sampleRate/2), optionally area-normalized.
 * srcDimsTensor = {bins, frames} per sample; nfft is derived per sample as (bins-1)*2.
 * src/dst layout NFT, numDims = 3.  The filter tables and a spectrum tile sit in shared memory: bins and
 * filters whose tables exceed a CTA's share return RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE.
 * Replaces api/rppt_tensor_audio_augmentations.h:274. */
SHARED_PUBLIC RppStatus rppt_mel_filter_bank_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                                 Rpp32s *srcDimsTensor, Rpp32f maxFreq, Rpp32f minFreq,
                                                 RpptMelScaleFormula melFormula, Rpp32s numFilter, Rpp32f sampleRate,
                                                 bool normalize, rppHandle_t rppHandle);

#ifdef __cplusplus
/* Band-limited resampling from inRateTensor[i] to outRateTensor[i] with the caller's windowed
 * sinc table; output length ceil(length * outRate / inRate).  srcDimsTensor = {length,
 * channels}.  Replaces api/rppt_tensor_audio_augmentations.h:310. */
SHARED_PUBLIC RppStatus rppt_resample_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                          Rpp32f *inRateTensor, Rpp32f *outRateTensor, Rpp32s *srcDimsTensor,
                                          RpptResamplingWindow &window, rppHandle_t rppHandle);
#endif

#ifdef __cplusplus
}
#endif

#endif /* RPPB_RPPT_TENSOR_AUDIO_AUGMENTATIONS_H */
