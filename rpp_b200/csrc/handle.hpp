// Internal handle of the B200 audio path (behind the opaque rppHandle_t of include/rpp.h).
//
// Plays the role of the reference's rpp::Handle (src/include/common/handle.hpp:63-180,
// src/modules/handle_hip.cpp:100-240) with a different memory model: instead of a fixed
// 1.49 GB device scratch and an 8.3 M-float pinned scratch allocated at creation
// (handle_hip.cpp:216-234), the workspace is sized from each call and grows on demand, so
// there is no scratch cap and no RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rpp.h"

namespace rppb {

// Thrown inside the library and converted to a status code at the C boundary.
struct Error
{
    RppStatus status;
    std::string what;
};

[[noreturn]] void fail(RppStatus status, const std::string& what);
// Sets the calling thread's message returned by rppbGetLastError.
void record_error(const std::string& what);
void check_cuda(cudaError_t err, const char* what);

// Checked build (RPPB_CHECKED, check.cu): a device region a call's kernels may touch.
struct CheckSpan
{
    const void* p;
    size_t bytes;
    bool writable;
};
#ifdef RPPB_CHECKED
std::recursive_mutex& check_mutex();
// Uploads the table of `spans` (merged where they touch) on stream s; enabled = false switches checks off.
void check_upload(cudaStream_t s, bool enabled, std::vector<CheckSpan> spans);
// Reads and clears the violation record: st when there was none, else the violation's status code.
RppStatus check_collect(RppStatus st);
void check_reset();
// The byte count rppb_check_shrink_next_tensors set for the next source or destination tensor (0 when
// none), cleared by the read.
unsigned long long check_take_shrink(bool destination);
#endif

// Bump allocator over one workspace block: measure with base == nullptr, then carve.
class Carver
{
  public:
    explicit Carver(void* base) : base_(static_cast<char*>(base)) {}
    template <class T>
    T* take(size_t count)
    {
        size_t off = (used_ + 255) & ~size_t(255);
        used_ = off + count * sizeof(T);
        return base_ ? reinterpret_cast<T*>(base_ + off) : nullptr;
    }
    size_t used() const { return (used_ + 255) & ~size_t(255); }

  private:
    char* base_;
    size_t used_ = 0;
};

class Handle
{
  public:
    Handle(size_t batchSize, cudaStream_t stream);
    ~Handle();

#ifdef RPPB_CHECKED
    // uploads the call's region table first when it changed (check.cu)
    cudaStream_t stream() const
    {
        if (check_dirty_) check_flush();
        return stream_;
    }
#else
    cudaStream_t stream() const { return stream_; }
#endif
    void set_stream(cudaStream_t s) { stream_ = s; }
    size_t batch_size() const { return batch_; }
    void set_batch_size(size_t b) { batch_ = b; }
    int device() const { return device_; }
    int num_sms() const { return num_sms_; }

    // Device workspace valid for the current call; contents are undefined on entry.
    void* workspace(size_t bytes);

    // Makes a per-sample tensor readable by kernels.  Device, managed and pinned pointers are
    // returned as device addresses; pageable host memory is copied through pinned staging into
    // the workspace region `dst` (which must hold `bytes`).
    const void* device_view(const void* p, size_t bytes, void* dst);
    // True when the device can write `p` directly (device, managed or pinned memory).
    bool device_writable(const void* p, void** devicePtr);

    // Cached device tables keyed by a string (window functions, twiddles).  The host builder
    // fills `host` once; the table is uploaded and kept until the handle is destroyed.
    const float* table(const std::string& key, size_t count, void (*build)(float*, size_t, const void*),
                       const void* ctx);
    // Cached device buffer of `bytes` for tables that a kernel builds: returns the buffer for `key`
    // and sets *fresh when it was just allocated (the caller then fills it on stream() before any
    // use).  While stream() is being captured a missing key returns nullptr (nothing is allocated
    // during capture) and the caller builds the tables some other way.
    void* device_table(const std::string& key, size_t bytes, bool* fresh);
    // Uploads `bytes` of host data to a device region that stays valid for this call.
    void upload(void* dDst, const void* hSrc, size_t bytes);

    void set_allocator(rppAllocatorFunction a, rppDeallocatorFunction d, void* ctx);

    // Profiling (rppEnableProfiling / rppGetKernelTime).
    void enable_profiling(bool on);
    void begin_call();
    void end_call();
    float last_call_ms();

    // A small zeroed device word array that kernels set on bounded-wait timeouts.
    int* device_flags();
    // Test setting (rppb_set_wait_fault_injection): the fused front end's decibel items wait for one
    // spectrum tile more than their clip has, with a short poll limit, so the wait runs out.
    void set_wait_injection(bool on) { wait_injection_ = on; }
    bool wait_injection() const { return wait_injection_; }
    // rppb_set_tc_materialized_frames: the tensor-core spectrogram writes frame rows out instead of
    // reading overlapping rows through its tensor map.
    void set_tc_materialize(bool on) { tc_materialize_ = on; }
    bool tc_materialize() const { return tc_materialize_; }

    // Checked build: regions of the current call beyond the handle's own blocks (caller tensors,
    // per-sample tensors, pinned host buffers); check_src / check_dst register a caller's source /
    // destination tensor.
    // check_begin starts a call, check_end ends it and returns the status of any violation.
#ifdef RPPB_CHECKED
    void check_add(const void* p, size_t bytes, bool writable);
    void check_src(const void* p, size_t bytes);
    void check_dst(const void* p, size_t bytes);
    void check_begin();
    RppStatus check_end(RppStatus st);
    // the rest of the call is not checked (its regions cannot be listed)
    void check_suspend();
#else
    void check_add(const void*, size_t, bool) {}
    void check_src(const void*, size_t) {}
    void check_dst(const void*, size_t) {}
    void check_begin() {}
    RppStatus check_end(RppStatus st) { return st; }
#endif

    // Extra streams of this handle (created on first use, non-blocking), for copies that overlap
    // the kernels on stream(); every call that uses them joins them back into stream() before it
    // returns, so stream order on stream() still covers all of the handle's work.
    cudaStream_t aux_stream(int i);
    // Event i of the handle's pool (timing disabled), created on first use.
    cudaEvent_t event(int i);

    // Scratch of size `bytes` in pinned host memory, reused after the previous user's copy ended.
    void* staging(size_t bytes);
    void staging_done();

  private:
    // A device block and the deallocator it must go back to (the allocator in force when it was
    // allocated: rppSetAllocator may change it while blocks are alive).
    struct Block
    {
        void* p = nullptr;
        rppDeallocatorFunction free_fn = nullptr;
        void* ctx = nullptr;
        bool custom = false;
        size_t bytes = 0;
    };
    void* dev_alloc(size_t bytes);
    void dev_free(void* p);
    Block block_alloc(size_t bytes);
    static void block_free(const Block& b);

    int device_ = 0;
    int num_sms_ = 148;
    cudaStream_t stream_ = nullptr;
    size_t batch_ = 1;

    void* ws_ = nullptr;
    size_t ws_bytes_ = 0;

    void* pinned_ = nullptr;
    size_t pinned_bytes_ = 0;
    cudaEvent_t pinned_free_ = nullptr;
    bool pinned_pending_ = false;

    cudaStream_t aux_[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> events_;

    std::map<std::string, Block> tables_;
    Block flags_;
    bool wait_injection_ = false;
    bool tc_materialize_ = false;

    rppAllocatorFunction alloc_fn_ = nullptr;
    rppDeallocatorFunction free_fn_ = nullptr;
    void* alloc_ctx_ = nullptr;

    bool profiling_ = false;
    cudaEvent_t ev_begin_ = nullptr, ev_end_ = nullptr;
    bool timed_ = false;

#ifdef RPPB_CHECKED
    void check_flush() const;
    mutable std::vector<CheckSpan> check_spans_;
    mutable bool check_dirty_ = false;
    bool check_active_ = false;
#endif
};

Handle& deref(rppHandle_t h);

// Counts kernel launches made by this library (reported by rppbGetLaunchCount).
void count_launch(int kernels = 1);
long long launch_count();

// Number of CTAs for a persistent launch of `kernel` with `threads` threads and `smem` bytes.
int persistent_grid(const Handle& h, const void* kernel, int threads, size_t smem);

}  // namespace rppb
