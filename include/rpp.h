/*
 * rppb — handle API of the B200 audio path.
 *
 * Same entry points and signatures as the reference's api/rpp.h:132-280, with the accelerator
 * queue being a CUDA stream (the reference's GPU build uses hipStream_t, api/rpp.h:49).
 *
 * A handle owns: the CUDA stream every rppt_*_gpu call is enqueued on, a device workspace
 * that grows on demand (never a fixed scratch cap), pinned staging for per-sample tensors
 * that callers pass in pageable host memory, and cached device tables (windows, twiddles).
 * A handle is not thread-safe; use one handle per host thread.
 */
#ifndef RPPB_RPP_H
#define RPPB_RPP_H

#include "rppdefs.h"

#if defined(_WIN32)
#define SHARED_PUBLIC __declspec(dllexport)
#else
#define SHARED_PUBLIC __attribute__((visibility("default")))
#endif

/* cudaStream_t without requiring the CUDA headers (cudaStream_t is `struct CUstream_st *`). */
struct CUstream_st;
typedef struct CUstream_st* rppAcceleratorQueue_t;

/* Opaque handle type, declared as in the reference (api/rpp.h:73). */
struct rppHandle
{
};
typedef struct rppHandle* rppHandle_t;
typedef rppHandle_t RppHandle_t;

/* Custom device allocator hooks (reference api/rpp.h:92-107). */
typedef void* (*rppAllocatorFunction)(void* context, size_t sizeBytes);
typedef void (*rppDeallocatorFunction)(void* context, void* memory);

#ifdef __cplusplus
extern "C" {
#define RPPB_DEFAULT(x) = x
#else
#define RPPB_DEFAULT(x)
#endif

/* Creates a handle bound to `stream` (nullptr: the legacy default stream) on the current CUDA
 * device.  backend must be RPP_HIP_BACKEND (the GPU backend); RPP_HOST_BACKEND returns
 * rppStatusNotImplemented because this library has no CPU path.  numThreads is accepted and
 * ignored.  Replaces api/rpp.h:132 (src/modules/handle_api.cpp:29-44). */
SHARED_PUBLIC rppStatus_t rppCreate(rppHandle_t* handle, size_t nBatchSize, Rpp32u numThreads RPPB_DEFAULT(0),
                                    void* stream RPPB_DEFAULT(nullptr), RppBackend backend RPPB_DEFAULT(RPP_HOST_BACKEND));

/* Releases the handle, its workspace and tables after the handle's stream has drained.
 * Replaces api/rpp.h:150. */
SHARED_PUBLIC rppStatus_t rppDestroy(rppHandle_t handle, RppBackend backend RPPB_DEFAULT(RPP_HOST_BACKEND));

/* Replaces api/rpp.h:168 and :186. */
SHARED_PUBLIC rppStatus_t rppSetBatchSize(rppHandle_t handle, size_t batchSize);
SHARED_PUBLIC rppStatus_t rppGetBatchSize(rppHandle_t handle, size_t* batchSize);

/* Rebinds / reads the handle's CUDA stream.  Replaces api/rpp.h:206 and :224. */
SHARED_PUBLIC rppStatus_t rppSetStream(rppHandle_t handle, rppAcceleratorQueue_t streamID);
SHARED_PUBLIC rppStatus_t rppGetStream(rppHandle_t handle, rppAcceleratorQueue_t* streamID);

/* Routes every device allocation the handle makes (its workspace, its cached tables and its device
 * error word) through the caller's allocator; passing null restores cudaMalloc/cudaFree.  The
 * current workspace is released (after the handle's stream drains) and the next call allocates a
 * new one from the allocator now in force; every other block goes back, when the handle is
 * destroyed, to the deallocator that was in force when it was allocated (none when that was null).
 * Replaces api/rpp.h:244. */
SHARED_PUBLIC rppStatus_t rppSetAllocator(rppHandle_t handle, rppAllocatorFunction allocator,
                                          rppDeallocatorFunction deallocator, void* allocatorContext);

/* Device time in ms of the last rppt_*_gpu call on this handle, when profiling is enabled
 * (CUDA events around the call's launches; reading it synchronizes on the end event).
 * Replaces api/rpp.h:262 and :280. */
SHARED_PUBLIC rppStatus_t rppGetKernelTime(rppHandle_t handle, float* time);
SHARED_PUBLIC rppStatus_t rppEnableProfiling(rppHandle_t handle, bool enable);

#ifdef __cplusplus
}
#endif
#undef RPPB_DEFAULT

#endif /* RPPB_RPP_H */
