/*
 * rppb — continuous-batching server for the multi-rate audio front end (extension; no counterpart in
 * the reference, whose entry points are one-shot batch calls).
 *
 * Requests of 1..k mono clips at any input rate are submitted from any thread at any time.  A
 * scheduler thread owned by the server
 *   - admits requests first come, first served when all their device buffers (input at its rate,
 *     the outRate signal, the decibel output) fit in a fixed device arena (the memory budget);
 *   - copies each admitted request's clips in on an upload stream: clips in pinned (device-mapped)
 *     memory are read by one copy kernel per admission round, pageable ones by one DMA copy each;
 *   - runs steps on a compute stream: every uploaded, not yet processed clip (up to maxClipsPerStep)
 *     gets an entry in a pinned clip table, and one CUDA graph (table copy + rppb_frontend_clips_gpu:
 *     resample -> pre-emphasis -> STFT -> mel -> decibels) is replayed; up to `tables` steps are in
 *     flight and requests that arrive meanwhile join the next step;
 *   - copies each finished clip's decibels [numFilter][frames] to the request's output on a
 *     download stream (one copy kernel per retired step for pinned outputs, a DMA copy each for
 *     pageable ones), and reports the request complete when all of its copies have ended.
 * Two step paths: the fused front end (rppb_frontend_clips_gpu), or, with plainChain set, the plain
 * FP32 path -- resample, then the four calls rppt_pre_emphasis_filter_gpu, rppt_spectrogram_gpu,
 * rppt_mel_filter_bank_gpu and rppt_to_decibels_gpu on a batch buffer of maxClipsPerStep rows of
 * maxSamples samples (the clips are copied in and the decibels out by kernels).
 * Every clip's result depends only on that clip, so a request gives the same bits alone and in any
 * mix of requests.  Host clip and output buffers must stay valid until the request completes;
 * pinned memory lets the copies run asynchronously.
 */
#ifndef RPPB_SERVER_H
#define RPPB_SERVER_H

#include "rppb_frontend.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct RppbServer* rppbServer_t;

typedef struct
{
    Rpp64u budgetBytes;       /* device arena for request buffers */
    Rpp32s maxClipsPerStep;
    Rpp32s tables;            /* steps in flight, one captured graph each */
    Rpp32f outRate;           /* rate entering the spectrogram */
    const Rpp32f* lookup;     /* host resampling window LUT (as RpptResamplingWindow) */
    Rpp32s lookupSize;
    Rpp32f scale;
    Rpp32f center;
    Rpp32s lobes;
    Rpp32f preemphCoeff;
    RppbFrontendParams params; /* windowFunction must be null (Hann) */
    Rpp32s plainChain;         /* 0: fused front end; 1: the plain FP32 four-call path per step */
    Rpp32s maxSamples;         /* plain path: longest clip at outRate (0: 30 s); longer requests are refused */
} RppbServerConfig;

typedef struct
{
    Rpp64u id;
    Rpp64s submitNs;          /* steady clock at rppb_server_submit */
    Rpp64s finishNs;          /* steady clock when the scheduler saw the last output copy end */
} RppbCompletion;

/* Creates the server on the current CUDA device: arena, streams, clip tables, captured graphs and
 * the scheduler thread. */
SHARED_PUBLIC RppStatus rppb_server_create(rppbServer_t* server, const RppbServerConfig* config);
/* Stops the scheduler after the requests in flight have completed and frees everything. */
SHARED_PUBLIC RppStatus rppb_server_destroy(rppbServer_t server);
/* Frames of the output of a clip of `length` samples at `rate` (outputs are [numFilter][frames],
 * at least one frame of storage). */
SHARED_PUBLIC Rpp32s rppb_server_frames(rppbServer_t server, Rpp32s length, Rpp32f rate);
/* Queues a request; clips[i] holds lengths[i] samples at rates[i], outputs[i] receives
 * numFilter x max(frames, 1) floats.  RPP_ERROR_NOT_ENOUGH_MEMORY if the request can never fit
 * the arena. */
SHARED_PUBLIC RppStatus rppb_server_submit(rppbServer_t server, const Rpp32f* const* clips, const Rpp32s* lengths,
                                           const Rpp32f* rates, Rpp32f* const* outputs, Rpp32s numClips,
                                           Rpp64u* requestId);
/* Moves up to `capacity` completions (in completion order) into `done`. */
SHARED_PUBLIC RppStatus rppb_server_poll(rppbServer_t server, RppbCompletion* done, Rpp32s capacity, Rpp32s* count);
/* Arena bytes held by admitted, unfinished requests. */
SHARED_PUBLIC Rpp64u rppb_server_arena_used(rppbServer_t server);

#ifdef __cplusplus
}
#endif

#endif
