// Device helpers shared by the audio kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

namespace rppb {

void count_launch(int kernels);
void check_cuda(cudaError_t err, const char* what);

// ---------------------------------------------------------------- checked build
// Every global load and store of the kernels names its address through RPPB_RD / RPPB_WR.  In the
// library these expand to the address itself.  Built with -DRPPB_CHECKED (librppb_checked.so,
// `python -m rpp_b200.build --checked`), each access is first compared with the device regions the
// current call may touch (check.cu): the caller's tensors as their descriptors describe them, the
// per-sample tensors, the workspace and the handle's tables.  An access outside them is recorded
// (site, address, size; the first one of the call) and redirected to a dummy buffer, so it neither
// reads nor writes out of bounds, and the call returns a status code for it.
constexpr unsigned check_file_hash(const char* path)
{
    const char* base = path;
    for (const char* q = path; *q; ++q)
        if (*q == '/') base = q + 1;
    unsigned h = 2166136261u;   // FNV-1a of the file's base name
    for (; *base; ++base) h = (h ^ static_cast<unsigned char>(*base)) * 16777619u;
    return h & 0xffffu;
}
template <unsigned kV>
struct CheckConst
{
    static constexpr unsigned value = kV;
};
#define RPPB_SITE ((::rppb::CheckConst<::rppb::check_file_hash(__FILE__)>::value << 16) | (__LINE__ & 0xffff))
#ifdef RPPB_CHECKED
__device__ void* check_addr(const void* p, unsigned bytes, bool write, unsigned site);
template <class T>
__device__ __forceinline__ T* check_ptr(T* p, bool write, unsigned site)
{
    return static_cast<T*>(check_addr(p, unsigned(sizeof(T)), write, site));
}
// a range of `bytes` (bulk copies, prefetches): true when it lies inside one region
__device__ bool check_range(const void* p, unsigned long long bytes, bool write, unsigned site);
#define RPPB_RD(p) ::rppb::check_ptr((p), false, RPPB_SITE)
#define RPPB_WR(p) ::rppb::check_ptr((p), true, RPPB_SITE)
#define RPPB_RANGE_OK(p, bytes) ::rppb::check_range((p), (bytes), false, RPPB_SITE)
#else
#define RPPB_RD(p) (p)
#define RPPB_WR(p) (p)
#define RPPB_RANGE_OK(p, bytes) true
#endif

// ---------------------------------------------------------------- ragged batches
// A batch of uneven samples is addressed as one flat list of work units (chunks, frame tiles,
// reset blocks ...).  prefix[b] is the number of units of samples 0..b-1 (prefix[n] = total),
// computed on the device from the per-sample tensors, so no call reads lengths on the host.

// Largest b in [0, n) with prefix[b] <= w (w < prefix[n]); empty samples are skipped.
// `prefix` may point to global or shared memory (see cache_prefix).
__device__ __forceinline__ int ragged_find(const long long* prefix, int n, long long w)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        int mid = (lo + hi + 1) >> 1;
        if (*RPPB_RD(prefix + mid) <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Shared-memory copy of prefix[0..n] when it fits (batches up to kPrefixCache - 1 samples), so the
// per-unit binary search costs shared-memory rather than global-memory latency.  All threads of
// the CTA must call it; it ends with __syncthreads.
constexpr int kPrefixCache = 512;
template <int CAP = kPrefixCache>
__device__ __forceinline__ const long long* cache_prefix(const long long* prefix, int n, long long* s_cache)
{
    if (n + 1 > CAP)
    {
        __syncthreads();
        return prefix;
    }
    for (int i = threadIdx.x; i <= n; i += blockDim.x) s_cache[i] = *RPPB_RD(prefix + i);
    __syncthreads();
    return s_cache;
}

// One CTA of 1024 threads: prefix[0..n] = exclusive scan of count(b), and zero[0..zeroWords) = 0
// (the work counters of the kernel that follows).  It lets a kernel launched after it with
// programmatic stream serialization (launch_dependent) start at once; that kernel runs its
// independent setup, then grid_dependency_wait() before it reads what this kernel writes.
template <class Count>
__global__ void __launch_bounds__(1024) ragged_prefix_kernel(Count count, int n, long long* __restrict__ prefix,
                                                             unsigned* __restrict__ zero, int zeroWords)
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    for (int i = threadIdx.x; i < zeroWords; i += 1024) *RPPB_WR(zero + i) = 0u;
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int b0 = t * per, b1 = min(n, b0 + per);
    long long s = 0;
    for (int b = b0; b < b1; ++b) s += count(b);
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1)
    {
        long long v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = t ? part[t - 1] : 0;
    for (int b = b0; b < b1; ++b)
    {
        *RPPB_WR(prefix + b) = run;
        run += count(b);
    }
    if (t == 1023) *RPPB_WR(prefix + n) = part[1023];
}

template <class Count>
inline void launch_ragged_prefix(Count count, int n, long long* prefix, cudaStream_t s, unsigned* zero = nullptr,
                                 int zeroWords = 0)
{
    ragged_prefix_kernel<Count><<<1, 1024, 0, s>>>(count, n, prefix, zero, zeroWords);
    count_launch(1);
}

// In a kernel launched by launch_dependent: waits until the kernel before it in the stream has
// completed and its writes are visible (a no-op for a kernel launched the ordinary way).
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launches `kernel` with programmatic stream serialization: it may start while the kernel before
// it (which must allow it, as ragged_prefix_kernel does) is still running, so its setup overlaps
// that kernel and the launch gap; it must call grid_dependency_wait() before touching that
// kernel's results.  Kernels earlier in the stream have completed by then.
template <class... KArgs, class... Args>
inline void launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             const char* what, Args&&... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    check_cuda(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...), what);
}

// ---------------------------------------------------------------- float helpers
// Monotone map of float to uint32 so that atomicMax on the key is a float max (NaN excluded).
// Asks L2 to fetch the bytes of [begin, end) (rounded inward to 16-byte boundaries; nothing when
// that leaves no whole 16-byte block).  A hint: no completion to wait for.
__device__ __forceinline__ void l2_prefetch(const float* begin, const float* end)
{
    const uintptr_t b = (reinterpret_cast<uintptr_t>(begin) + 15) & ~uintptr_t(15);
    const uintptr_t e = reinterpret_cast<uintptr_t>(end) & ~uintptr_t(15);
    if (e <= b) return;
    const uintptr_t n = e - b;
    const uint32_t bytes = n < (uintptr_t(1) << 20) ? uint32_t(n) : (1u << 20);
    if (!RPPB_RANGE_OK(reinterpret_cast<const void*>(b), bytes)) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"(bytes) : "memory");
}

__device__ __forceinline__ unsigned float_key(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned k)
{
    unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Reflect an out-of-range index into [minLoc, maxLoc) the way the reference does
// (src/modules/tensor/cpu/kernel/spectrogram.cpp:55-69): mirror without repeating the edge,
// repeatedly for short signals; a signal shorter than 2 maps everything to its last sample.
// The reference's repeated mirroring is periodic with period 2 * (len - 1), so it is evaluated
// in closed form; the result is always inside [minLoc, maxLoc).
__device__ __forceinline__ int reflect_index(int loc, int minLoc, int maxLoc)
{
    const int len = maxLoc - minLoc;
    if (len < 2) return maxLoc - 1;
    const int period = 2 * (len - 1);
    int r = (loc - minLoc) % period;
    if (r < 0) r += period;
    return minLoc + (r < len ? r : period - r);
}

// Resampled length ceil(length * outRate / inRate) in the reference's float arithmetic
// (resample.cpp:57); equal rates keep the length.
__host__ __device__ __forceinline__ int resampled_length(int L, float inRate, float outRate)
{
#ifdef __CUDA_ARCH__
    return inRate == outRate ? L : int(ceilf(__fdiv_rn(__fmul_rn(float(L), outRate), inRate)));
#else
    return inRate == outRate ? L : int(ceilf(float(L) * outRate / inRate));
#endif
}

// Frames of a sample (spectrogram.cpp:47-52), never negative.
__host__ __device__ __forceinline__ int num_windows(int length, int windowLength, int windowStep, bool center)
{
    if (!center) length -= windowLength;
    int f = length / windowStep + 1;
    return f < 0 ? 0 : f;
}

}  // namespace rppb
