// Handle API of the B200 audio path: rppCreate / rppDestroy / batch size / stream / allocator /
// profiling (reference: api/rpp.h:132-280, src/modules/handle_api.cpp:29-101).
#include "handle.hpp"

#include <atomic>
#include <tuple>
#include <cstring>
#include <stdexcept>

namespace rppb {

void fail(RppStatus status, const std::string& what) { throw Error{status, what}; }

void check_cuda(cudaError_t err, const char* what)
{
    if (err != cudaSuccess)
        fail(err == cudaErrorMemoryAllocation ? RPP_ERROR_NOT_ENOUGH_MEMORY : RPP_ERROR,
             std::string(what) + ": " + cudaGetErrorString(err));
}

Handle::Handle(size_t batchSize, cudaStream_t stream) : stream_(stream), batch_(batchSize)
{
    check_cuda(cudaGetDevice(&device_), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device_), "sm count");
    check_cuda(cudaEventCreateWithFlags(&pinned_free_, cudaEventDisableTiming), "cudaEventCreate");
}

Handle::~Handle()
{
    cudaStreamSynchronize(stream_);
    for (cudaStream_t s : aux_)
        if (s)
        {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    if (ws_) dev_free(ws_);
    for (auto& kv : tables_) block_free(kv.second);
    block_free(flags_);
    if (pinned_) cudaFreeHost(pinned_);
    if (pinned_free_) cudaEventDestroy(pinned_free_);
    if (ev_begin_) cudaEventDestroy(ev_begin_);
    if (ev_end_) cudaEventDestroy(ev_end_);
}

void* Handle::dev_alloc(size_t bytes)
{
    void* p = nullptr;
    if (alloc_fn_)
    {
        p = alloc_fn_(alloc_ctx_, bytes);
        if (!p) fail(RPP_ERROR_NOT_ENOUGH_MEMORY, "custom allocator returned null");
        return p;
    }
    check_cuda(cudaMalloc(&p, bytes), "cudaMalloc(workspace)");
    return p;
}

void Handle::dev_free(void* p)
{
    if (alloc_fn_ || free_fn_)
    {
        if (free_fn_) free_fn_(alloc_ctx_, p);
        return;
    }
    cudaFree(p);
}

Handle::Block Handle::block_alloc(size_t bytes)
{
    Block b;
    b.p = dev_alloc(bytes);
    b.bytes = bytes;
    b.custom = alloc_fn_ != nullptr;
    b.free_fn = free_fn_;
    b.ctx = alloc_ctx_;
    return b;
}

void Handle::block_free(const Block& b)
{
    if (!b.p) return;
    if (b.custom)
    {
        if (b.free_fn) b.free_fn(b.ctx, b.p);
        return;
    }
    cudaFree(b.p);
}

void* Handle::workspace(size_t bytes)
{
    if (bytes <= ws_bytes_) return ws_;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(stream_, &cap), "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
        fail(RPP_ERROR_NOT_ENOUGH_MEMORY,
             "workspace must grow while the stream is being captured; run the call once before capture");
    // The old block may still be read by earlier launches on this stream.
    check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize(grow workspace)");
    if (ws_) dev_free(ws_);
    ws_ = nullptr;
    ws_bytes_ = 0;
    size_t grown = bytes + bytes / 4 + (1 << 20);
    ws_ = dev_alloc(grown);
    ws_bytes_ = grown;
#ifdef RPPB_CHECKED
    check_dirty_ = check_active_;
#endif
    return ws_;
}

cudaStream_t Handle::aux_stream(int i)
{
    if (!aux_[i]) check_cuda(cudaStreamCreateWithFlags(&aux_[i], cudaStreamNonBlocking), "cudaStreamCreate(aux)");
    return aux_[i];
}

cudaEvent_t Handle::event(int i)
{
    while (int(events_.size()) <= i)
    {
        cudaEvent_t e;
        check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate(pool)");
        events_.push_back(e);
    }
    return events_[i];
}

void* Handle::staging(size_t bytes)
{
    if (pinned_pending_)
    {
        check_cuda(cudaEventSynchronize(pinned_free_), "cudaEventSynchronize(staging)");
        pinned_pending_ = false;
    }
    if (bytes > pinned_bytes_)
    {
        if (pinned_) cudaFreeHost(pinned_);
        pinned_ = nullptr;
        pinned_bytes_ = 0;
        size_t grown = bytes + bytes / 2 + 4096;
        check_cuda(cudaMallocHost(&pinned_, grown), "cudaMallocHost(staging)");
        pinned_bytes_ = grown;
    }
    return pinned_;
}

void Handle::staging_done()
{
    check_cuda(cudaEventRecord(pinned_free_, stream_), "cudaEventRecord(staging)");
    pinned_pending_ = true;
}

void Handle::upload(void* dDst, const void* hSrc, size_t bytes)
{
    if (bytes == 0) return;
    void* st = staging(bytes);
    std::memcpy(st, hSrc, bytes);
    check_cuda(cudaMemcpyAsync(dDst, st, bytes, cudaMemcpyHostToDevice, stream_), "cudaMemcpyAsync(H2D)");
    staging_done();
}

const void* Handle::device_view(const void* p, size_t bytes, void* dst)
{
    if (p == nullptr) fail(RPP_ERROR_INVALID_ARGUMENTS, "null per-sample tensor");
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        attr.type = cudaMemoryTypeUnregistered;
    }
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged)
    {
        check_add(p, bytes, false);
        return p;
    }
    if (attr.type == cudaMemoryTypeHost && attr.devicePointer != nullptr)
    {
        check_add(attr.devicePointer, bytes, false);
        return attr.devicePointer;
    }
    upload(dst, p, bytes);
    return dst;
}

bool Handle::device_writable(const void* p, void** devicePtr)
{
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged)
    {
        *devicePtr = const_cast<void*>(p);
        return true;
    }
    if (attr.type == cudaMemoryTypeHost && attr.devicePointer != nullptr)
    {
        *devicePtr = attr.devicePointer;
        return true;
    }
    return false;
}

const float* Handle::table(const std::string& key, size_t count, void (*build)(float*, size_t, const void*),
                           const void* ctx)
{
    auto it = tables_.find(key);
    if (it != tables_.end()) return static_cast<const float*>(it->second.p);
    std::vector<float> host(count);
    build(host.data(), count, ctx);
    const Block b = block_alloc(count * sizeof(float));
    // Synchronous copy from pageable memory: tables are built once per key, before any capture.
    const cudaError_t e = cudaMemcpy(b.p, host.data(), count * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) block_free(b);
    check_cuda(e, "cudaMemcpy(table)");
    tables_[key] = b;
#ifdef RPPB_CHECKED
    check_dirty_ = check_active_;
#endif
    return static_cast<const float*>(b.p);
}

void* Handle::device_table(const std::string& key, size_t bytes, bool* fresh)
{
    *fresh = false;
    auto it = tables_.find(key);
    if (it != tables_.end()) return it->second.p;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(stream_, &cap), "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone) return nullptr;
    const Block b = block_alloc(bytes);
    tables_[key] = b;
    *fresh = true;
#ifdef RPPB_CHECKED
    check_dirty_ = check_active_;
#endif
    return b.p;
}

int* Handle::device_flags()
{
    if (!flags_.p)
    {
        const Block b = block_alloc(64 * sizeof(int));
        const cudaError_t e = cudaMemset(b.p, 0, 64 * sizeof(int));
        if (e != cudaSuccess) block_free(b);
        check_cuda(e, "cudaMemset(flags)");
        flags_ = b;
#ifdef RPPB_CHECKED
        check_dirty_ = check_active_;
#endif
    }
    return static_cast<int*>(flags_.p);
}

#ifdef RPPB_CHECKED
void Handle::check_add(const void* p, size_t bytes, bool writable)
{
    if (!check_active_ || !p || !bytes) return;
    check_spans_.push_back(CheckSpan{p, bytes, writable});
    check_dirty_ = true;
}

void Handle::check_src(const void* p, size_t bytes)
{
    const unsigned long long shrink = check_take_shrink(false);
    check_add(p, shrink < bytes ? bytes - shrink : 0, false);
}

void Handle::check_dst(const void* p, size_t bytes)
{
    const unsigned long long shrink = check_take_shrink(true);
    check_add(p, shrink < bytes ? bytes - shrink : 0, true);
}

void Handle::check_flush() const
{
    std::vector<CheckSpan> spans = check_spans_;
    if (ws_) spans.push_back(CheckSpan{ws_, ws_bytes_, true});
    for (const auto& kv : tables_) spans.push_back(CheckSpan{kv.second.p, kv.second.bytes, true});
    if (flags_.p) spans.push_back(CheckSpan{flags_.p, flags_.bytes, true});
    check_dirty_ = false;
    check_upload(stream_, true, spans);
}

void Handle::check_begin()
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(stream_, &cap), "cudaStreamIsCapturing");
    if (cap == cudaStreamCaptureStatusNone)
    {
        // a record left by an earlier call that ended in an exception is not this call's
        check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize(check)");
        check_reset();
    }
    check_spans_.clear();
    check_active_ = true;
    check_dirty_ = true;
}

void Handle::check_suspend()
{
    check_active_ = false;
    check_dirty_ = false;
    check_upload(stream_, false, {});
}

RppStatus Handle::check_end(RppStatus st)
{
    check_active_ = false;
    check_dirty_ = false;
    check_upload(stream_, false, {});
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(stream_, &cap), "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone) return st;   // read by the next uncaptured call
    check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize(check)");
    return check_collect(st);
}
#endif

void Handle::set_allocator(rppAllocatorFunction a, rppDeallocatorFunction d, void* ctx)
{
    check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize(set allocator)");
    if (ws_) dev_free(ws_);
    ws_ = nullptr;
    ws_bytes_ = 0;
    alloc_fn_ = a;
    free_fn_ = a ? d : nullptr;
    alloc_ctx_ = a ? ctx : nullptr;
}

void Handle::enable_profiling(bool on)
{
    profiling_ = on;
    if (on && !ev_begin_)
    {
        check_cuda(cudaEventCreate(&ev_begin_), "cudaEventCreate");
        check_cuda(cudaEventCreate(&ev_end_), "cudaEventCreate");
    }
}

void Handle::begin_call()
{
    if (profiling_) check_cuda(cudaEventRecord(ev_begin_, stream_), "cudaEventRecord");
}

void Handle::end_call()
{
    if (profiling_)
    {
        check_cuda(cudaEventRecord(ev_end_, stream_), "cudaEventRecord");
        timed_ = true;
    }
}

float Handle::last_call_ms()
{
    if (!profiling_ || !timed_) return 0.f;
    float ms = 0.f;
    check_cuda(cudaEventSynchronize(ev_end_), "cudaEventSynchronize");
    check_cuda(cudaEventElapsedTime(&ms, ev_begin_, ev_end_), "cudaEventElapsedTime");
    return ms;
}

Handle& deref(rppHandle_t h)
{
    if (h == nullptr) fail(RPP_ERROR_INVALID_ARGUMENTS, "null rppHandle_t");
    return *reinterpret_cast<Handle*>(h);
}

static std::atomic<long long> g_launches{0};

void count_launch(int kernels) { g_launches.fetch_add(kernels, std::memory_order_relaxed); }

long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

int persistent_grid(const Handle& h, const void* kernel, int threads, size_t smem)
{
    // Cached per (kernel, device, threads, smem) so that repeated calls, including calls made while
    // a stream is being captured into a CUDA graph, make no further non-stream CUDA API calls.  The
    // kernel's dynamic shared-memory limit only ever grows (one kernel serves several sizes).
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
    static std::map<std::pair<const void*, int>, size_t> smemLimit;
    const auto key = std::make_tuple(kernel, h.device(), threads, smem);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    size_t& limit = smemLimit[std::make_pair(kernel, h.device())];
    // without the opt-in attribute, static + dynamic shared memory must stay within 48 KB
    cudaFuncAttributes fa{};
    check_cuda(cudaFuncGetAttributes(&fa, kernel), "cudaFuncGetAttributes");
    int optin = 0;
    check_cuda(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h.device()), "smem limit");
    if (smem + fa.sharedSizeBytes > size_t(optin))
        fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "the call's tile needs more shared memory than a CTA has");
    if (smem + fa.sharedSizeBytes > 48 * 1024 && smem > limit)
    {
        check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "smem attr");
        limit = smem;
    }
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem), "occupancy");
    if (per_sm < 1) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "kernel does not fit on an SM");
    const int grid = per_sm * h.num_sms();
    cache[key] = grid;
    return grid;
}

}  // namespace rppb

using rppb::Handle;

template <class F>
static rppStatus_t handle_try(F&& f)
{
    try
    {
        f();
        return rppStatusSuccess;
    }
    catch (const rppb::Error& e)
    {
        switch (e.status)
        {
            case RPP_ERROR_INVALID_ARGUMENTS: return rppStatusBadParm;
            case RPP_ERROR_NOT_ENOUGH_MEMORY: return rppStatusAllocFailed;
            case RPP_ERROR_NOT_IMPLEMENTED: return rppStatusNotImplemented;
            default: return rppStatusInternalError;
        }
    }
    catch (const std::bad_alloc&)
    {
        return rppStatusAllocFailed;
    }
    catch (...)
    {
        return rppStatusUnknownError;
    }
}

extern "C" SHARED_PUBLIC rppStatus_t rppCreate(rppHandle_t* handle, size_t nBatchSize, Rpp32u, void* stream,
                                               RppBackend backend)
{
    if (handle == nullptr) return rppStatusBadParm;
    if (backend == RPP_HOST_BACKEND || backend == RPP_OCL_BACKEND) return rppStatusNotImplemented;
    if (backend != RPP_HIP_BACKEND) return rppStatusBadParm;
    return handle_try([&] {
        auto* h = new Handle(nBatchSize, static_cast<cudaStream_t>(stream));
        *handle = reinterpret_cast<rppHandle_t>(h);
    });
}

extern "C" SHARED_PUBLIC rppStatus_t rppDestroy(rppHandle_t handle, RppBackend)
{
    if (handle == nullptr) return rppStatusBadParm;
    return handle_try([&] { delete reinterpret_cast<Handle*>(handle); });
}

extern "C" SHARED_PUBLIC rppStatus_t rppSetBatchSize(rppHandle_t handle, size_t batchSize)
{
    return handle_try([&] { rppb::deref(handle).set_batch_size(batchSize); });
}

extern "C" SHARED_PUBLIC rppStatus_t rppGetBatchSize(rppHandle_t handle, size_t* batchSize)
{
    if (batchSize == nullptr) return rppStatusBadParm;
    return handle_try([&] { *batchSize = rppb::deref(handle).batch_size(); });
}

extern "C" SHARED_PUBLIC rppStatus_t rppSetStream(rppHandle_t handle, rppAcceleratorQueue_t streamID)
{
    return handle_try([&] { rppb::deref(handle).set_stream(reinterpret_cast<cudaStream_t>(streamID)); });
}

extern "C" SHARED_PUBLIC rppStatus_t rppGetStream(rppHandle_t handle, rppAcceleratorQueue_t* streamID)
{
    if (streamID == nullptr) return rppStatusBadParm;
    return handle_try([&] { *streamID = reinterpret_cast<rppAcceleratorQueue_t>(rppb::deref(handle).stream()); });
}

extern "C" SHARED_PUBLIC rppStatus_t rppSetAllocator(rppHandle_t handle, rppAllocatorFunction allocator,
                                                     rppDeallocatorFunction deallocator, void* allocatorContext)
{
    return handle_try([&] { rppb::deref(handle).set_allocator(allocator, deallocator, allocatorContext); });
}

extern "C" SHARED_PUBLIC rppStatus_t rppGetKernelTime(rppHandle_t handle, float* time)
{
    if (time == nullptr) return rppStatusBadParm;
    return handle_try([&] { *time = rppb::deref(handle).last_call_ms(); });
}

// Kernels launched by this library in this process so far.
extern "C" SHARED_PUBLIC long long rppbGetLaunchCount() { return rppb::launch_count(); }

extern "C" SHARED_PUBLIC rppStatus_t rppEnableProfiling(rppHandle_t handle, bool enable)
{
    return handle_try([&] { rppb::deref(handle).enable_profiling(enable); });
}
