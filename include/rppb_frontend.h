/*
 * rppb — fused audio front end (extension; no single counterpart in the reference).
 *
 * rppb_frontend_gpu computes, in one persistent launch, exactly what this sequence of the
 * reference's entry points computes (api/rppt_tensor_audio_augmentations.h:156, :232, :274, :122):
 *
 *   rppt_pre_emphasis_filter_gpu(src -> pre, srcLength, coeff, borderType)
 *   rppt_spectrogram_gpu(pre -> spec NFT, srcLength, centerWindows, reflectPadding, windowFunction,
 *                        nfft, power, windowLength, windowStep)
 *   rppt_mel_filter_bank_gpu(spec -> mel NFT, {nfft/2+1, frames}, maxFreq, minFreq, melFormula,
 *                            numFilter, sampleRate, normalize)
 *   rppt_to_decibels_gpu(mel -> dst, {frames, numFilter}, cutOffDB, multiplier, referenceMagnitude)
 *
 * and, with the default FP32 spectrum engine, its outputs are bit-identical to that sequence run
 * through this library (the tensor-core engine, RppbSpectrumEngine, computes the spectrum as a factored
 * DFT on tcgen05 tensor cores instead, within ~1e-6 of each frame's largest bin).  The
 * intermediate pre-emphasized signal, spectrum and mel tensors never reach memory except the mel
 * power, which is written into dst and converted to decibels in place once the clip's maximum is
 * known.  dst is NFT [numFilter][frames] per sample (hStride >= frames); only the valid frames
 * are written.  nfft must be a power of two from 128 to 2048.  The tables, a frame tile's span and its
 * power tile sit in shared memory: a window, step or numFilter too large for a CTA's share returns
 * RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE.  Asynchronous on the handle stream; capturable in a CUDA
 * graph after one uncaptured call has sized the handle workspace.
 */
#ifndef RPPB_FRONTEND_H
#define RPPB_FRONTEND_H

#include "rpp.h"
#include "rppdefs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    /* pre_emphasis_filter */
    RpptAudioBorderType borderType;
    /* spectrogram */
    bool centerWindows;
    bool reflectPadding;
    Rpp32f* windowFunction; /* host pointer, windowLength floats; nullptr = Hann */
    Rpp32s nfft;
    Rpp32s power;           /* 2: power, 1: magnitude */
    Rpp32s windowLength;
    Rpp32s windowStep;
    /* mel_filter_bank */
    Rpp32f maxFreq;         /* 0: sampleRate / 2 */
    Rpp32f minFreq;
    RpptMelScaleFormula melFormula;
    Rpp32s numFilter;
    Rpp32f sampleRate;
    bool normalize;
    /* to_decibels */
    Rpp32f cutOffDB;
    Rpp32f multiplier;
    Rpp32f referenceMagnitude; /* 0: per-sample maximum */
    /* schedule: clips by which the decibel tiles trail the spectrum tiles (0 = default 32) */
    Rpp32s lookahead;
    /* schedule (never the results; rppb_frontend_tune_gpu picks them): frames per spectrum item
     * (0 = 2 tiles, else 1, 2 or 4 times the FFT plan's tile of 16 frames for nfft >= 512, 32
     * below), frames per decibel item (0 = 128, else a power of two from 16 to 256), CTAs per SM
     * (0 = as many as fit) */
    Rpp32s tileFrames;
    Rpp32s dbFrames;
    Rpp32s ctasPerSm;
    /* spectrum engine (RppbSpectrumEngine): the FP32 register FFT, whose results are bit-identical to
     * the four plain calls, or the factored DFT on the tensor cores (nfft 512 only) */
    Rpp32s spectrumEngine;
} RppbFrontendParams;

/* Spectrum engines of the fused front end. */
typedef enum
{
    /* FP32 register FFT: the outputs are bit for bit those of the four plain calls */
    RPPB_ENGINE_FP32_FFT = 0,
    /* The 512-point real DFT factored as 16 x 32 and computed as two GEMM stages on tcgen05 tensor cores
     * (32-point real DFTs, an FP32 twiddle, 16-point complex DFTs).  Each frame is scaled by a power of
     * two, every operand is split into F16 hi + lo, and hi*hi + hi*lo + lo*hi is accumulated in FP32:
     * the spectrum stays within ~1e-6 of each frame's largest bin against FP64 (the mel and decibel
     * steps are the FP32 engine's), so the outputs are close to, not bit-identical with, the plain
     * calls.  nfft must be 512 (windowLength <= 512, tileFrames 0, 16, 32 or 64); otherwise
     * RPP_ERROR_NOT_IMPLEMENTED. */
    RPPB_ENGINE_TENSOR_CORE_F16X3 = 1
} RppbSpectrumEngine;

/* srcDesc numDims = 2 (F32 1-D signals); dstDesc numDims = 3, layout NFT, F32.
 * srcLengthTensor and coeffTensor as for rppt_pre_emphasis_filter_gpu. */
SHARED_PUBLIC RppStatus rppb_frontend_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                                          Rpp32s* srcLengthTensor, Rpp32f* coeffTensor, const RppbFrontendParams* params,
                                          rppHandle_t rppHandle);

/* Down-mix to mono and resample in one launch: equal, bit for bit, to rppt_down_mixing_gpu
 * (normalizeWeights) followed by a mono rppt_resample_gpu with the window described by
 * lookup/lookupSize/scale/center/lobes (the RpptResamplingWindow fields, passed as plain values so C
 * callers can use it; lookup in device or pinned memory, or pageable host memory).  srcDimsTensor =
 * {length, channels} per sample of interleaved input; dst receives mono samples at outRate.
 * Extension used by the multi-rate front end (no single counterpart in the reference). */
SHARED_PUBLIC RppStatus rppb_downmix_resample_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                  RpptDescPtr dstDescPtr, Rpp32f* inRateTensor, Rpp32f* outRateTensor,
                                                  Rpp32s* srcDimsTensor, bool normalizeWeights, const Rpp32f* lookup,
                                                  Rpp32s lookupSize, Rpp32f scale, Rpp32f center, Rpp32s lobes,
                                                  rppHandle_t rppHandle);

/* One clip of a serving batch: buffers anywhere in device memory. */
typedef struct
{
    const Rpp32f* src;   /* mono input at inRate, `length` samples */
    Rpp32f* work;        /* scratch for the signal resampled to outRate: ceil(length * outRate / inRate) floats */
    Rpp32f* dst;         /* decibels, NFT [numFilter][dstStride] */
    Rpp32s length;
    Rpp32f inRate;
    Rpp32s dstStride;    /* frames dst holds per filter row (>= the clip's frame count) */
    Rpp32s pad;
} RppbClip;

/* The whole multi-rate front end over a table of clips: resample every clip to outRate
 * (rppt_resample_gpu semantics, mono) into its `work` buffer, then rppb_frontend_gpu on it into
 * `dst`.  Two launches (+ their work-list scans), no host synchronization, graph-capturable: the
 * table is read on the device, so a captured graph replays over whatever clips the table holds
 * (a clip of length 0 is skipped).  clips: device or pinned memory, numClips entries.
 * Extension for continuous-batching servers (no counterpart in the reference). */
SHARED_PUBLIC RppStatus rppb_frontend_clips_gpu(const RppbClip* clips, Rpp32s numClips, Rpp32f outRate,
                                                const Rpp32f* lookup, Rpp32s lookupSize, Rpp32f scale, Rpp32f center,
                                                Rpp32s lobes, Rpp32f preemphCoeff, const RppbFrontendParams* params,
                                                rppHandle_t rppHandle);

/* Autotuner of the schedule of rppb_frontend_gpu (extension; no counterpart in the reference): runs
 * the call on the given batch once per candidate (frames per spectrum tile, frames per decibel item,
 * lookahead, CTAs per SM; outputs are identical for all of them), times `reps` runs of each with
 * CUDA events on the handle stream, and writes the fastest into params->tileFrames, dbFrames,
 * lookahead and ctasPerSm (bestMs, if not null, receives its time).  dstPtr is overwritten with
 * the call's result.  Winners are remembered per device and call shape for the process, and in the
 * file named by the RPPB_TUNE_CACHE environment variable if set.  Synchronizes the handle stream;
 * not capturable. */
SHARED_PUBLIC RppStatus rppb_frontend_tune_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                               RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor, Rpp32f* coeffTensor,
                                               RppbFrontendParams* params, Rpp32s reps, Rpp32f* bestMs,
                                               rppHandle_t rppHandle);

/* The fused front end on HOST tensors: srcHost, dstHost, srcLengthHost and coeffHost are host memory
 * (pinned for overlap; pageable works but serializes the copies), laid out as for rppb_frontend_gpu.
 * The batch is split into numChunks contiguous runs of clips (<= 0: 16) with about equal sample
 * counts, except that from 6 chunks on the first and last carry a quarter and the second and
 * second-to-last half of a middle chunk's samples (the copy-in before the first kernel and the
 * copy-out after the last one run with the other direction idle, so they are kept short); chunk
 * c's valid samples are copied in on one stream while chunk c-1 is computed and chunk c-2's
 * valid output rows (numFilter x frames per clip) are copied out on another, through double-buffered
 * device staging in the handle workspace.  Output equals rppb_frontend_gpu on the same data and
 * only the valid region of dstHost is written.  Asynchronous: synchronize the handle stream before
 * reading dstHost.  Extension (no counterpart in the reference). */
SHARED_PUBLIC RppStatus rppb_frontend_host_gpu(const Rpp32f* srcHost, RpptDescPtr srcDescPtr, Rpp32f* dstHost,
                                               RpptDescPtr dstDescPtr, const Rpp32s* srcLengthHost,
                                               const Rpp32f* coeffHost, const RppbFrontendParams* params,
                                               Rpp32s numChunks, rppHandle_t rppHandle);

/* 16-bit PCM ingest (extension; the reference converts WAV data on the host in its test suite,
 * utilities/test_suite/rpp_test_suite_audio.h:143-178): srcDesc dataType I16, dstDesc F32, both
 * [n][nStride] with c interleaved channels; converts srcLengthTensor[b] frames x c samples of each
 * clip to float / 32768 (exact), leaving the destination tail as it was.  Lengths may be device,
 * pinned or pageable memory; srcPtr/dstPtr device memory. */
SHARED_PUBLIC RppStatus rppb_pcm16_to_f32_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                              RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor, rppHandle_t rppHandle);

/* Operand precision of the tensor-core spectrogram; every variant accumulates in FP32. */
typedef enum
{
    RPPB_TC_BF16 = 0,        /* BF16 operands, one pass */
    RPPB_TC_BF16_HILO3 = 1,  /* x = hi + lo, both BF16; hi*hi + hi*lo + lo*hi */
    RPPB_TC_TF32 = 2,        /* FP32 rounded to TF32 */
    RPPB_TC_FP8_E4M3 = 3     /* E4M3 with one scale per frame (largest sample -> 448) */
} RppbTensorCorePrecision;

/* Tensor-core spectrogram (precision study): the short-time DFT as a GEMM on tcgen05 tensor cores
 * with the window folded into the DFT basis.  Same framing and output layouts as
 * rppt_spectrogram_gpu with the Hann window (no windowFunction argument); coeffTensor (nullable)
 * applies pre-emphasis first, as rppt_pre_emphasis_filter_gpu with borderType would.  Requires nfft a
 * multiple of 256, windowLength <= nfft, and windowStep a multiple of 8 (BF16) or 4 (TF32); otherwise
 * RPP_ERROR_NOT_IMPLEMENTED.  Extension for the precision study (no counterpart in the reference). */
SHARED_PUBLIC RppStatus rppb_spectrogram_tc_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor, Rpp32f* coeffTensor,
                                                RpptAudioBorderType borderType, bool centerWindows,
                                                bool reflectPadding, Rpp32s nfft, Rpp32s power, Rpp32s windowLength,
                                                Rpp32s windowStep, RppbTensorCorePrecision precision,
                                                rppHandle_t rppHandle);

/* Tensor-core mel projection (precision study; extension, no counterpart in the reference): the
 * mel filter bank of rppt_mel_filter_bank_gpu (same arguments and tables) as a GEMM on tcgen05
 * tensor cores, spectrum frames x dense filter matrix, with the operand precision of `precision`
 * (FP8: per-frame spectrum scale and one power-of-two weight scale) and FP32 accumulation.
 * NFT in and out, numFilter <= 256; the spectrum's bin count is srcDesc->h.  Only the valid frames
 * (srcDimsTensor) are written; the sums are in the tensor core's order, so the results carry the
 * operand precision's error instead of matching the reference bit for bit. */
SHARED_PUBLIC RppStatus rppb_mel_filter_bank_tc_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                    RpptDescPtr dstDescPtr, Rpp32s* srcDimsTensor, Rpp32f maxFreq,
                                                    Rpp32f minFreq, RpptMelScaleFormula melFormula, Rpp32s numFilter,
                                                    Rpp32f sampleRate, bool normalize,
                                                    RppbTensorCorePrecision precision, rppHandle_t rppHandle);

/* Reads (and clears) the handle's device error word: nonzero when a fused launch gave up
 * waiting for a clip's spectrum tiles (a bounded wait; the affected tiles are left unconverted).
 * Synchronizes the handle stream. */
SHARED_PUBLIC RppStatus rppb_get_device_error(rppHandle_t rppHandle, Rpp32s* errorCode);

/* Failure-detection test hook; no counterpart in the reference.  While enabled, every decibel item
 * of the fused front end (rppb_frontend_gpu, rppb_frontend_host_gpu, rppb_frontend_clips_gpu) waits
 * for one spectrum tile more than its clip has, a count that nothing reaches, and gives up after
 * ~1024 polls (about 0.1 ms) instead of a few seconds: the kernel sets the device error word, leaves
 * that item's mel power unconverted and finishes, so the context stays usable.  Lets a test check the
 * timeout path without a fault or a hang.  Off by default; affects only this handle. */
SHARED_PUBLIC RppStatus rppb_set_wait_fault_injection(rppHandle_t rppHandle, bool enable);

/* Tensor-core spectrogram setting; no counterpart in the reference.  rppb_spectrogram_tc_gpu reads the
 * BF16/TF32 frames in place, through a tensor map whose rows (frames) start windowStep samples apart
 * and overlap; when the driver refuses such a map it writes every frame out as a [frame][kPad] row
 * first.  With materialize = true this handle always takes the second form (more memory traffic,
 * the same bits), e.g. to test it.  Off by default; affects only this handle. */
SHARED_PUBLIC RppStatus rppb_set_tc_materialized_frames(rppHandle_t rppHandle, bool materialize);

/* Bounds-checked build (librppb_checked.so, built with `python -m rpp_b200.build --checked`); no
 * counterpart in the reference.  In that library every global load and store of the kernels is checked
 * against the device regions of the call that launched it: the caller's tensors as their descriptors
 * describe them, the per-sample tensors, the handle's workspace and tables.  An access outside them is
 * skipped (loads read a dummy, stores write one), and the call returns RPP_ERROR_OUT_OF_BOUND_SRC_ROI
 * for a stray read or RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH for a stray write, with the file, line,
 * address and count in rppbGetLastError().  Calls run one at a time and synchronize their stream at
 * the end (a captured call's record is read by the next uncaptured one).  This test hook registers the
 * next call's source and destination tensors sourceBytes and destinationBytes shorter than their
 * descriptors say (0: as described), so that the call's last in-bounds loads or stores are reported (and
 * skipped) as out of bounds.  It returns RPP_ERROR_NOT_IMPLEMENTED in the ordinary library. */
SHARED_PUBLIC RppStatus rppb_check_shrink_next_tensors(Rpp64u sourceBytes, Rpp64u destinationBytes);

#ifdef __cplusplus
}
#endif

#endif /* RPPB_FRONTEND_H */
