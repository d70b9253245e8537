// to_decibels: y = multiplier * log10(2) * log2(max(minRatio, x / ref)).
//
// Reference: src/modules/tensor/cpu/kernel/to_decibels.cpp:39-95.  ref is the caller's
// referenceMagnitude, or (when that is 0) the per-sample maximum over the srcDims ROI, seeded
// with -FLT_MAX; 1/ref is taken as 1 when ref is 0.  srcDims[i].width == 1 selects a 1-D sample
// of `height` contiguous values, otherwise `height` rows of `width` values at hStride.
//
// Two launches, no host synchronization (the reference's GPU path synchronizes the stream
// twice, hip/kernel/to_decibels.cpp:282,295):
//   1. when ref is 0: a max pass over the ROIs, one float-ordered atomicMax per CTA into an
//      n-entry scratch array;
//   2. the decibel pass.
// Both walk the same flat list of units: 4096-value chunks of a 1-D sample, or 4096-column
// chunks of one row of a 2-D sample.  The log is CUDA's log2f (1 ulp): results agree with the
// host path within 1e-5 dB, far inside the 1e-3 dB parity bound.
#include <cfloat>

#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 4096;

struct DecibelCount
{
    const uint32_t* dims;
    __device__ long long operator()(int b) const
    {
        long long wdt = dims[2 * b], hgt = dims[2 * b + 1];
        if (wdt == 1) return (hgt + kChunk - 1) / kChunk;
        return hgt * ((wdt + kChunk - 1) / kChunk);
    }
};

// Unit w of sample b -> row, first column, column count.
struct UnitSpan
{
    uint32_t row, col0, cols;
};
__device__ __forceinline__ UnitSpan unit_span(uint32_t wdt, uint32_t hgt, long long u)
{
    UnitSpan s;
    if (wdt == 1)
    {
        s.row = 0;
        s.col0 = uint32_t(u) * kChunk;
        s.cols = min(uint32_t(kChunk), hgt - s.col0);
    }
    else
    {
        uint32_t chunks = (wdt + kChunk - 1) / kChunk;
        s.row = uint32_t(u / chunks);
        s.col0 = uint32_t(u % chunks) * kChunk;
        s.cols = min(uint32_t(kChunk), wdt - s.col0);
    }
    return s;
}

__global__ void __launch_bounds__(kThreads) decibel_max_kernel(const float* __restrict__ src, uint32_t nStride,
                                                               uint32_t hStride, const uint32_t* __restrict__ dims,
                                                               unsigned* __restrict__ maxKey,
                                                               const long long* __restrict__ prefix, int n)
{
    __shared__ float warpMax[kThreads / 32];
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const uint32_t wdt = dims[2 * b], hgt = dims[2 * b + 1];
        const UnitSpan s = unit_span(wdt, hgt, w - prefix[b]);
        const float* x = src + size_t(b) * nStride + size_t(s.row) * hStride + s.col0;
        float m = -FLT_MAX;
        for (uint32_t c = threadIdx.x; c < s.cols; c += kThreads) m = fmaxf(m, x[c]);
        m = warp_max(m);
        if ((threadIdx.x & 31) == 0) warpMax[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32)
        {
            float v = threadIdx.x < kThreads / 32 ? warpMax[threadIdx.x] : -FLT_MAX;
            v = warp_max(v);
            if (threadIdx.x == 0) atomicMax(maxKey + b, float_key(v));
        }
        __syncthreads();
    }
}

template <bool kUseMax>
__global__ void __launch_bounds__(kThreads) decibel_kernel(const float* __restrict__ src, uint32_t srcNStride,
                                                           uint32_t srcHStride, float* __restrict__ dst,
                                                           uint32_t dstNStride, uint32_t dstHStride,
                                                           const uint32_t* __restrict__ dims,
                                                           const unsigned* __restrict__ maxKey, float refMag,
                                                           float minRatio, float multiplier,
                                                           const long long* __restrict__ prefix, int n)
{
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const uint32_t wdt = dims[2 * b], hgt = dims[2 * b + 1];
        const UnitSpan s = unit_span(wdt, hgt, w - prefix[b]);
        float ref = refMag;
        if (kUseMax)
        {
            unsigned k = maxKey[b];
            ref = k == 0u ? -FLT_MAX : fmaxf(-FLT_MAX, key_float(k));
        }
        const float inv = ref != 0.f ? __fdiv_rn(1.f, ref) : 1.0f;
        const float* x = src + size_t(b) * srcNStride + size_t(s.row) * srcHStride + s.col0;
        float* y = dst + size_t(b) * dstNStride + size_t(s.row) * dstHStride + s.col0;
        for (uint32_t c = threadIdx.x; c < s.cols; c += kThreads)
        {
            float v = __fmul_rn(x[c], inv);
            v = minRatio < v ? v : minRatio;
            y[c] = __fmul_rn(multiplier, log2f(v));
        }
    }
}

}  // namespace

void launch_to_decibels(Handle& h, void* scratch, const DecibelArgs& a)
{
    if (a.n <= 0) return;
    Carver cv(scratch);
    long long* prefix = cv.take<long long>(a.n + 1);
    unsigned* maxKey = cv.take<unsigned>(a.n);
    launch_ragged_prefix(DecibelCount{a.dims}, a.n, prefix, h.stream());
    const bool useMax = (a.referenceMagnitude == 0.f);
    if (useMax)
    {
        check_cuda(cudaMemsetAsync(maxKey, 0, size_t(a.n) * sizeof(unsigned), h.stream()), "memset(max)");
        int grid = persistent_grid(h, reinterpret_cast<const void*>(decibel_max_kernel), kThreads, 0);
        decibel_max_kernel<<<grid, kThreads, 0, h.stream()>>>(a.src, a.srcNStride, a.srcHStride, a.dims, maxKey,
                                                              prefix, a.n);
        count_launch();
        check_cuda(cudaGetLastError(), "decibel_max_kernel");
        grid = persistent_grid(h, reinterpret_cast<const void*>(decibel_kernel<true>), kThreads, 0);
        decibel_kernel<true><<<grid, kThreads, 0, h.stream()>>>(a.src, a.srcNStride, a.srcHStride, a.dst, a.dstNStride,
                                                                a.dstHStride, a.dims, maxKey, 0.f, a.minRatio,
                                                                a.multiplier, prefix, a.n);
        count_launch();
    }
    else
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(decibel_kernel<false>), kThreads, 0);
        decibel_kernel<false><<<grid, kThreads, 0, h.stream()>>>(a.src, a.srcNStride, a.srcHStride, a.dst,
                                                                 a.dstNStride, a.dstHStride, a.dims, nullptr,
                                                                 a.referenceMagnitude, a.minRatio, a.multiplier,
                                                                 prefix, a.n);
        count_launch();
    }
    check_cuda(cudaGetLastError(), "decibel_kernel");
}

}  // namespace rppb
