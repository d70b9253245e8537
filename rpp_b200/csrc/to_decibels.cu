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
// chunks of one row of a 2-D sample.  The log is CUDA's __log2f intrinsic (the hardware base-2
// logarithm: 2^-22.6 absolute error on [0.5, 2], 2 ulp elsewhere), so results agree with the host
// path within about 1e-5 dB, far inside the 1e-3 dB parity bound; the fused front end uses the
// same intrinsic, which keeps the two paths bit-identical.
#include <cfloat>
#include <cmath>
#include <mutex>

#include "../../include/rppt_tensor_audio_augmentations.h"
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 4096;

constexpr int kRowsPerUnit = 8;   // rows of a 2-D sample per work unit

struct DecibelCount
{
    const uint32_t* dims;
    __device__ long long operator()(int b) const
    {
        long long wdt = *RPPB_RD(dims + 2 * b), hgt = *RPPB_RD(dims + (2 * b + 1));
        if (wdt == 1) return (hgt + kChunk - 1) / kChunk;
        return ((hgt + kRowsPerUnit - 1) / kRowsPerUnit) * ((wdt + kChunk - 1) / kChunk);
    }
};

// Unit u of a sample -> first row, row count, first column, column count.
struct UnitSpan
{
    uint32_t row, rows, col0, cols;
};
__device__ __forceinline__ UnitSpan unit_span(uint32_t wdt, uint32_t hgt, long long u)
{
    UnitSpan s;
    if (wdt == 1)
    {
        s.row = 0;
        s.rows = 1;
        s.col0 = uint32_t(u) * kChunk;
        s.cols = min(uint32_t(kChunk), hgt - s.col0);
    }
    else
    {
        const uint32_t chunks = (wdt + kChunk - 1) / kChunk;
        s.row = uint32_t(u / chunks) * kRowsPerUnit;
        s.rows = min(uint32_t(kRowsPerUnit), hgt - s.row);
        s.col0 = uint32_t(u % chunks) * kChunk;
        s.cols = min(uint32_t(kChunk), wdt - s.col0);
    }
    return s;
}

// Both kernels walk a unit's elements in (row, column) runs: warp wi takes rows s.row + wi,
// s.row + wi + 8, ...; its lanes walk the row 4 columns at a time (16-byte accesses when the strides
// and addresses allow), so no element index is divided.  A 1-D unit (one row of up to 4096 values)
// is walked by all threads.
__global__ void __launch_bounds__(kThreads) decibel_max_kernel(const float* __restrict__ src, uint32_t nStride,
                                                               uint32_t hStride, const uint32_t* __restrict__ dims,
                                                               unsigned* __restrict__ maxKey,
                                                               const long long* __restrict__ prefix, int n, bool vec)
{
    __shared__ float warpMax[kThreads / 32];
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const uint32_t wdt = *RPPB_RD(dims + 2 * b), hgt = *RPPB_RD(dims + (2 * b + 1));
        const UnitSpan s = unit_span(wdt, hgt, w - prefix[b]);
        const float* base = src + size_t(b) * nStride + size_t(s.row) * hStride + s.col0;
        // a lane loads 4 column steps (16 values) before folding them, so the loads overlap
        float m = -FLT_MAX;
        const bool oneD = wdt == 1;
        const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
        const uint32_t step = oneD ? 4u * kThreads : 128u;
        const uint32_t first = oneD ? 4u * threadIdx.x : 4u * lane;
        const uint32_t r0 = oneD ? 0u : uint32_t(wi), rstep = oneD ? 1u : uint32_t(kThreads / 32);
        constexpr int kBatch = 4;
        for (uint32_t r = r0; r < s.rows; r += rstep)
        {
            const float* p = base + size_t(r) * hStride;
            for (uint32_t c0 = first; c0 < s.cols; c0 += kBatch * step)
            {
                float4 x[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; ++k)
                {
                    const uint32_t c = c0 + k * step;
                    x[k] = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX);
                    if (vec && c + 4 <= s.cols) x[k] = __ldg(RPPB_RD(reinterpret_cast<const float4*>(p + c)));
                    else
                    {
                        if (c < s.cols) x[k].x = __ldg(RPPB_RD(p + c));
                        if (c + 1 < s.cols) x[k].y = __ldg(RPPB_RD(p + c + 1));
                        if (c + 2 < s.cols) x[k].z = __ldg(RPPB_RD(p + c + 2));
                        if (c + 3 < s.cols) x[k].w = __ldg(RPPB_RD(p + c + 3));
                    }
                }
#pragma unroll
                for (int k = 0; k < kBatch; ++k) m = fmaxf(m, fmaxf(fmaxf(x[k].x, x[k].y), fmaxf(x[k].z, x[k].w)));
            }
        }
        m = warp_max(m);
        if ((threadIdx.x & 31) == 0) warpMax[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32)
        {
            float v = threadIdx.x < kThreads / 32 ? warpMax[threadIdx.x] : -FLT_MAX;
            v = warp_max(v);
            if (threadIdx.x == 0) atomicMax(RPPB_WR(maxKey + b), float_key(v));
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
                                                           const long long* __restrict__ prefix, int n, bool vec)
{
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const uint32_t wdt = *RPPB_RD(dims + 2 * b), hgt = *RPPB_RD(dims + (2 * b + 1));
        const UnitSpan s = unit_span(wdt, hgt, w - prefix[b]);
        float ref = refMag;
        if (kUseMax)
        {
            unsigned k = *RPPB_RD(maxKey + b);
            ref = k == 0u ? -FLT_MAX : fmaxf(-FLT_MAX, key_float(k));
        }
        const float inv = ref != 0.f ? __fdiv_rn(1.f, ref) : 1.0f;
        auto db = [&](float x) {
            float t = __fmul_rn(x, inv);
            t = minRatio < t ? t : minRatio;
            return __fmul_rn(multiplier, __log2f(t));
        };
        // in-place calls alias src and dst: every element is loaded before its own store.  A lane
        // loads 4 column steps (16 values) before converting and storing them, so the loads overlap.
        const float* xb = src + size_t(b) * srcNStride + size_t(s.row) * srcHStride + s.col0;
        float* yb = dst + size_t(b) * dstNStride + size_t(s.row) * dstHStride + s.col0;
        const bool oneD = wdt == 1;
        const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
        const uint32_t step = oneD ? 4u * kThreads : 128u;
        const uint32_t first = oneD ? 4u * threadIdx.x : 4u * lane;
        const uint32_t r0 = oneD ? 0u : uint32_t(wi), rstep = oneD ? 1u : uint32_t(kThreads / 32);
        constexpr int kBatch = 4;
        for (uint32_t r = r0; r < s.rows; r += rstep)
        {
            const float* p = xb + size_t(r) * srcHStride;
            float* q = yb + size_t(r) * dstHStride;
            for (uint32_t c0 = first; c0 < s.cols; c0 += kBatch * step)
            {
                float4 x[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; ++k)
                {
                    const uint32_t c = c0 + k * step;
                    x[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (vec && c + 4 <= s.cols) x[k] = *RPPB_RD(reinterpret_cast<const float4*>(p + c));
                    else
                    {
                        if (c < s.cols) x[k].x = *RPPB_RD(p + c);
                        if (c + 1 < s.cols) x[k].y = *RPPB_RD(p + (c + 1));
                        if (c + 2 < s.cols) x[k].z = *RPPB_RD(p + (c + 2));
                        if (c + 3 < s.cols) x[k].w = *RPPB_RD(p + (c + 3));
                    }
                }
#pragma unroll
                for (int k = 0; k < kBatch; ++k)
                {
                    const uint32_t c = c0 + k * step;
                    const float4 y = make_float4(db(x[k].x), db(x[k].y), db(x[k].z), db(x[k].w));
                    if (vec && c + 4 <= s.cols) *RPPB_WR(reinterpret_cast<float4*>(q + c)) = y;
                    else
                    {
                        if (c < s.cols) *RPPB_WR(q + c) = y.x;
                        if (c + 1 < s.cols) *RPPB_WR(q + (c + 1)) = y.y;
                        if (c + 2 < s.cols) *RPPB_WR(q + (c + 2)) = y.z;
                        if (c + 3 < s.cols) *RPPB_WR(q + (c + 3)) = y.w;
                    }
                }
            }
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
    const bool useMax = (a.referenceMagnitude == 0.f);
    // the maxima accumulate with atomicMax from zero keys: the prefix kernel zeroes them
    launch_ragged_prefix(DecibelCount{a.dims}, a.n, prefix, h.stream(), maxKey, useMax ? a.n : 0);
    auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    const bool vecSrc = aligned(a.src) && (a.srcNStride & 3) == 0 && (a.srcHStride & 3) == 0;
    const bool vec = vecSrc && aligned(a.dst) && (a.dstNStride & 3) == 0 && (a.dstHStride & 3) == 0;
    if (useMax)
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(decibel_max_kernel), kThreads, 0);
        decibel_max_kernel<<<grid, kThreads, 0, h.stream()>>>(a.src, a.srcNStride, a.srcHStride, a.dims, maxKey,
                                                              prefix, a.n, vecSrc);
        count_launch();
        check_cuda(cudaGetLastError(), "decibel_max_kernel");
        grid = persistent_grid(h, reinterpret_cast<const void*>(decibel_kernel<true>), kThreads, 0);
        decibel_kernel<true><<<grid, kThreads, 0, h.stream()>>>(a.src, a.srcNStride, a.srcHStride, a.dst, a.dstNStride,
                                                                a.dstHStride, a.dims, maxKey, 0.f, a.minRatio,
                                                                a.multiplier, prefix, a.n, vec);
        count_launch();
    }
    else
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(decibel_kernel<false>), kThreads, 0);
        decibel_kernel<false><<<grid, kThreads, 0, h.stream()>>>(a.src, a.srcNStride, a.srcHStride, a.dst,
                                                                 a.dstNStride, a.dstHStride, a.dims, nullptr,
                                                                 a.referenceMagnitude, a.minRatio, a.multiplier,
                                                                 prefix, a.n, vec);
        count_launch();
    }
    check_cuda(cudaGetLastError(), "decibel_kernel");
}

}  // namespace rppb

// ---------------------------------------------------------------- allocation-free variant
//
// rppt_to_decibels_gpu_static: the same computation as rppt_to_decibels_gpu for callers that
// must not allocate device memory (see include/rppt_tensor_audio_augmentations.h).  Its scratch
// (the work-list prefix and the per-sample maxima) is a file-scope __device__ array that every GPU
// loading this library holds until the process exits; host code reaches it only through the address
// cudaGetSymbolAddress returns for the current device, fetched once per device on the first call.
namespace rppb {
namespace {

constexpr int kStaticMaxSamples = 8192;
constexpr size_t kStaticPrefixBytes = (size_t(kStaticMaxSamples) + 1) * sizeof(long long);
constexpr size_t kStaticScratchBytes = kStaticPrefixBytes + size_t(kStaticMaxSamples) * sizeof(unsigned);

static __device__ __align__(256) unsigned char g_decibel_scratch[kStaticScratchBytes];

constexpr int kStaticMaxDevices = 64;
struct StaticDevice
{
    unsigned char* scratch;   // device address of g_decibel_scratch on this device
    int gridMax, gridTrue, gridFalse;
    bool ready;
};
StaticDevice g_static[kStaticMaxDevices];
std::mutex g_static_mutex;

// Once per device, with that device current: the scratch address and the persistent grid sizes.
cudaError_t static_setup(int device, StaticDevice*& out)
{
    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticDevice& d = g_static[device];
    if (!d.ready)
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_decibel_scratch);
        if (e != cudaSuccess) return e;
        int sms = 0, a = 0, b = 0, c = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, decibel_max_kernel, kThreads, 0)) != cudaSuccess)
            return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, decibel_kernel<true>, kThreads, 0)) != cudaSuccess)
            return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, decibel_kernel<false>, kThreads, 0)) != cudaSuccess)
            return e;
        d.scratch = static_cast<unsigned char*>(p);
        d.gridMax = max(a, 1) * sms;
        d.gridTrue = max(b, 1) * sms;
        d.gridFalse = max(c, 1) * sms;
        d.ready = true;
    }
    out = &d;
    return cudaSuccess;
}

// Device address for a per-sample tensor in device, managed or pinned memory; null otherwise.
const void* device_address(const void* p)
{
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess)
    {
        cudaGetLastError();
        return nullptr;
    }
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) return p;
    if (attr.type == cudaMemoryTypeHost) return attr.devicePointer;
    return nullptr;
}

}  // namespace
}  // namespace rppb

extern "C" SHARED_PUBLIC RppStatus rppt_to_decibels_gpu_static(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                               RpptDescPtr dstDescPtr, RpptImagePatchPtr srcDims,
                                                               Rpp32f cutOffDB, Rpp32f multiplier,
                                                               Rpp32f referenceMagnitude,
                                                               rppAcceleratorQueue_t stream)
{
    using namespace rppb;
    if (srcDescPtr == nullptr || dstDescPtr == nullptr) return RPP_ERROR_INVALID_ARGUMENTS;
    const Rpp32u tensorDims = Rpp32u(srcDescPtr->numDims - 1);
    if (tensorDims != 1 && tensorDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
    if (!multiplier) return RPP_ERROR_ZERO_DIVISION;
    if (srcDescPtr->dataType != F32) return RPP_ERROR_NOT_IMPLEMENTED;
    if (srcPtr == nullptr || dstPtr == nullptr || srcDims == nullptr) return RPP_ERROR_INVALID_ARGUMENTS;
    const int n = int(srcDescPtr->n);
    if (n <= 0) return RPP_SUCCESS;
    if (n > kStaticMaxSamples) return RPP_ERROR_OUT_OF_BOUND_SCRATCH_MEMORY_SIZE;   // batch above the fixed scratch
    const uint32_t* dims = static_cast<const uint32_t*>(device_address(srcDims));
    if (dims == nullptr) return RPP_ERROR_INVALID_ARGUMENTS;   // srcDims must be device or pinned memory
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kStaticMaxDevices) return RPP_ERROR;
    // a CUDA error left pending on this thread by earlier work belongs to its owner: refuse the call
    // without launching (and without clearing it) rather than report it as this call's failure
    if (cudaPeekAtLastError() != cudaSuccess) return RPP_ERROR;
    StaticDevice* sd = nullptr;
    if (static_setup(device, sd) != cudaSuccess) return RPP_ERROR;

    // to_decibels.cpp:40-45
    float minRatio = float(std::pow(10, cutOffDB / multiplier));
    if (minRatio == 0.0f) minRatio = std::nextafter(0.0f, 1.0f);
    const Rpp32f log10Factor = 0.3010299956639812;
    multiplier *= log10Factor;

    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    long long* prefix = reinterpret_cast<long long*>(sd->scratch);
    unsigned* maxKey = reinterpret_cast<unsigned*>(sd->scratch + kStaticPrefixBytes);
    const float* src = static_cast<const float*>(srcPtr);
    float* dst = static_cast<float*>(dstPtr);
    const uint32_t sN = srcDescPtr->strides.nStride, sH = srcDescPtr->strides.hStride;
    const uint32_t dN = dstDescPtr->strides.nStride, dH = dstDescPtr->strides.hStride;
    // every launch is checked at once: the first failure ends the call before later kernels queue
    launch_ragged_prefix(DecibelCount{dims}, n, prefix, s);
    if (cudaGetLastError() != cudaSuccess) return RPP_ERROR;
    auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    const bool vecSrc = aligned(src) && (sN & 3) == 0 && (sH & 3) == 0;
    const bool vec = vecSrc && aligned(dst) && (dN & 3) == 0 && (dH & 3) == 0;
    if (referenceMagnitude == 0.f)
    {
        // the maxima accumulate with atomicMax: start every call from zero keys
        if (cudaMemsetAsync(maxKey, 0, size_t(n) * sizeof(unsigned), s) != cudaSuccess) return RPP_ERROR;
        decibel_max_kernel<<<sd->gridMax, kThreads, 0, s>>>(src, sN, sH, dims, maxKey, prefix, n, vecSrc);
        count_launch();
        if (cudaGetLastError() != cudaSuccess) return RPP_ERROR;
        decibel_kernel<true><<<sd->gridTrue, kThreads, 0, s>>>(src, sN, sH, dst, dN, dH, dims, maxKey, 0.f, minRatio,
                                                               multiplier, prefix, n, vec);
        count_launch();
    }
    else
    {
        decibel_kernel<false><<<sd->gridFalse, kThreads, 0, s>>>(src, sN, sH, dst, dN, dH, dims, nullptr,
                                                                 referenceMagnitude, minRatio, multiplier, prefix, n,
                                                                 vec);
        count_launch();
    }
    return cudaGetLastError() == cudaSuccess ? RPP_SUCCESS : RPP_ERROR;
}
