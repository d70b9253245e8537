// non_silent_region_detection.
//
// Reference: src/modules/tensor/cpu/kernel/non_silent_region_detection.cpp:105-184.  The
// moving mean square (MMS) is a float running sum of squares, restarted every resetInterval
// samples (-1: once per sample) from a fresh sum over the preceding window; the sample's cutoff
// is (referencePower, or the maximum MMS when that is 0) * 10^(cutOffDB/10); the region runs
// from the first to the last MMS at or above the cutoff, its begin moved back by
// windowLength - 1 (clamped at 0); no such MMS gives (0, 0).
//
// The running sum is a dependent float chain, so its value depends on operation order.  Each
// reset block is independent, and one GPU lane replays one block's chain in exactly the
// reference's order (add the new square, store sum * (1/windowLength), subtract the square
// leaving the window; explicit round-to-nearest intrinsics, no FMA): the MMS values, and hence
// the begin/length integers, are bit-identical to the host path.
//   1. mms_kernel:    one warp per (sample, reset block): coalesced loads and squares by the warp,
//                     the chain by one lane, MMS into scratch, block maximum;
//   2. region_kernel: one warp per sample: cutoff from the block maxima, then the first and
//                     last qualifying block are scanned (ballot over 32 MMS at a time).
// Latency-bound by the per-block chain (resetInterval + windowLength dependent steps); the
// parallelism is the number of reset blocks in the batch.
#include <cfloat>

#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kRegionThreads = 256;

__device__ __forceinline__ long long block_len(int L, int reset) { return reset == -1 ? (L > 0 ? L : 1) : reset; }

struct NsrCount
{
    const int* len;
    uint32_t stride;
    int reset;
    __device__ long long operator()(int b) const
    {
        int L = min(len[b], int(stride));
        if (L <= 0) return 0;
        long long R = block_len(L, reset);
        return (L + R - 1) / R;
    }
};

__device__ __forceinline__ float sq(float v) { return __fmul_rn(v, v); }

constexpr int kMmsThreads = 256;
constexpr int kMmsWarps = kMmsThreads / 32;
constexpr int kChunk = 256;   // samples per warp step

// One warp per (sample, reset block).  Per chunk of 256 samples the warp loads the samples entering
// and leaving the window (coalesced), squares them in parallel into shared memory, then lane 0
// runs the block's float chain over the chunk (two dependent adds per sample -- the only serial
// part; squares and the scaled stores are off the chain) and the warp stores the MMS values.  A
// square of zero stands for "nothing leaves the window yet": sum - 0 == sum exactly for the
// non-negative sums of squares, so the chain is bit-identical to the reference's conditional
// subtraction.
__global__ void __launch_bounds__(kMmsThreads) mms_kernel(const float* __restrict__ src, uint32_t stride,
                                                         const int* __restrict__ len, int windowLength, int reset,
                                                         float* __restrict__ mms, float* __restrict__ blockMax,
                                                         const long long* __restrict__ prefix, int n)
{
    __shared__ long long s_prefix[kPrefixCache];
    __shared__ __align__(16) float s_in[kMmsWarps][kChunk];
    __shared__ __align__(16) float s_out[kMmsWarps][kChunk];
    __shared__ __align__(16) float s_val[kMmsWarps][kChunk];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    const float meanFactor = __fdiv_rn(1.0f, float(windowLength));
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    float* qi = s_in[wi];
    float* qo = s_out[wi];
    float* vv = s_val[wi];
    for (long long w = blockIdx.x * (long long)kMmsWarps + wi; w < total; w += (long long)gridDim.x * kMmsWarps)
    {
        const int b = ragged_find(prefix, n, w);
        const int L = min(len[b], int(stride));
        const long long R = block_len(L, reset);
        const int start = int((w - prefix[b]) * R);
        const int end = int(min((long long)L, start + R));
        const float* x = src + size_t(b) * stride;
        float* m = mms + size_t(b) * stride;
        float sum = 0.0f;   // meaningful in lane 0
        // fresh sum over the window that precedes the block (reference :131-133)
        for (int c = max(start - windowLength + 1, 0); c < start; c += kChunk)
        {
            const int cnt = min(kChunk, start - c);
            for (int k = lane; k < cnt; k += 32) qi[k] = sq(__ldg(x + c + k));
            __syncwarp();
            if (lane == 0)
                for (int k = 0; k < cnt; ++k) sum = __fadd_rn(sum, qi[k]);
            __syncwarp();
        }
        float bmax = -FLT_MAX;
        for (int c = start; c < end; c += kChunk)
        {
            const int cnt = min(kChunk, end - c);
            for (int k = lane; k < cnt; k += 32)
            {
                qi[k] = sq(__ldg(x + c + k));
                const int wb = c + k - windowLength + 1;
                qo[k] = wb >= 0 ? sq(__ldg(x + wb)) : 0.0f;
            }
            __syncwarp();
            if (lane == 0)
            {
                int k = 0;
                for (; k + 4 <= cnt; k += 4)
                {
                    const float4 a4 = *reinterpret_cast<const float4*>(qi + k);
                    const float4 o4 = *reinterpret_cast<const float4*>(qo + k);
                    float4 v4;
                    sum = __fadd_rn(sum, a4.x);
                    v4.x = __fmul_rn(sum, meanFactor);
                    sum = __fsub_rn(sum, o4.x);
                    sum = __fadd_rn(sum, a4.y);
                    v4.y = __fmul_rn(sum, meanFactor);
                    sum = __fsub_rn(sum, o4.y);
                    sum = __fadd_rn(sum, a4.z);
                    v4.z = __fmul_rn(sum, meanFactor);
                    sum = __fsub_rn(sum, o4.z);
                    sum = __fadd_rn(sum, a4.w);
                    v4.w = __fmul_rn(sum, meanFactor);
                    sum = __fsub_rn(sum, o4.w);
                    *reinterpret_cast<float4*>(vv + k) = v4;
                }
                for (; k < cnt; ++k)
                {
                    sum = __fadd_rn(sum, qi[k]);
                    vv[k] = __fmul_rn(sum, meanFactor);
                    sum = __fsub_rn(sum, qo[k]);
                }
            }
            __syncwarp();
            for (int k = lane; k < cnt; k += 32)
            {
                const float v = vv[k];
                m[c + k] = v;
                bmax = fmaxf(bmax, v);
            }
            __syncwarp();
        }
        bmax = warp_max(bmax);
        if (lane == 0) blockMax[w] = bmax;
    }
}

__global__ void __launch_bounds__(kRegionThreads) region_kernel(const float* __restrict__ mms, uint32_t stride,
                                                                const int* __restrict__ len, int windowLength,
                                                                int reset, float referencePower, float cutOff,
                                                                const float* __restrict__ blockMax,
                                                                int* __restrict__ outBegin,
                                                                int* __restrict__ outLength,
                                                                const long long* __restrict__ prefix, int n)
{
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * (kRegionThreads / 32) + (threadIdx.x >> 5);
    if (b >= n) return;
    const int L = min(len[b], int(stride));
    if (L <= 0)
    {
        if (lane == 0) { outBegin[b] = 0; outLength[b] = 0; }
        return;
    }
    const long long R = block_len(L, reset);
    const long long u0 = prefix[b], u1 = prefix[b + 1];
    const int nb = int(u1 - u0);
    float base = referencePower;
    if (referencePower == 0.0f)
    {
        float m = -FLT_MAX;
        for (int k = lane; k < nb; k += 32) m = fmaxf(m, blockMax[u0 + k]);
        base = warp_max(m);
    }
    const float cutOffMag = __fmul_rn(base, cutOff);
    const float* m = mms + size_t(b) * stride;

    // first block whose maximum reaches the cutoff, then the first index inside it
    int firstBlock = -1;
    for (int k0 = 0; k0 < nb && firstBlock < 0; k0 += 32)
    {
        const int k = k0 + lane;
        unsigned hit = __ballot_sync(0xffffffffu, k < nb && blockMax[u0 + k] >= cutOffMag);
        if (hit) firstBlock = k0 + __ffs(hit) - 1;
    }
    int detectBegin = 0, detectLength = 0;
    if (firstBlock >= 0)
    {
        int beginIdx = -1;
        const int s0 = int(firstBlock * R), s1 = int(min((long long)L, s0 + R));
        for (int i0 = s0; i0 < s1 && beginIdx < 0; i0 += 32)
        {
            const int i = i0 + lane;
            unsigned hit = __ballot_sync(0xffffffffu, i < s1 && m[i] >= cutOffMag);
            if (hit) beginIdx = i0 + __ffs(hit) - 1;
        }
        int lastBlock = -1;
        for (int k1 = nb - 1; k1 >= 0 && lastBlock < 0; k1 -= 32)
        {
            const int k = k1 - lane;
            unsigned hit = __ballot_sync(0xffffffffu, k >= 0 && blockMax[u0 + k] >= cutOffMag);
            if (hit) lastBlock = k1 - (__ffs(hit) - 1);
        }
        int endIdx = -1;
        const int e0 = int(lastBlock * R), e1 = int(min((long long)L, e0 + R));
        for (int i1 = e1 - 1; i1 >= e0 && endIdx < 0; i1 -= 32)
        {
            const int i = i1 - lane;
            unsigned hit = __ballot_sync(0xffffffffu, i >= e0 && m[i] >= cutOffMag);
            if (hit) endIdx = i1 - (__ffs(hit) - 1);
        }
        detectBegin = beginIdx;
        detectLength = endIdx - beginIdx + 1;
        if (detectBegin != 0 && detectLength != 0)
        {
            const int newBegin = max(detectBegin - (windowLength - 1), 0);
            detectLength += detectBegin - newBegin;
            detectBegin = newBegin;
        }
    }
    if (lane == 0)
    {
        outBegin[b] = detectBegin;
        outLength[b] = detectLength;
    }
}

}  // namespace

size_t nsr_scratch_bytes(int n, uint32_t srcStride, int resetInterval)
{
    size_t blocks = resetInterval == -1 ? size_t(n) : size_t(n) * ((srcStride + resetInterval - 1) / resetInterval);
    Carver cv(nullptr);
    cv.take<long long>(n + 1);
    cv.take<float>(size_t(n) * srcStride);
    cv.take<float>(blocks + 1);
    return cv.used();
}

void launch_nsr(Handle& h, void* scratch, const NsrArgs& a)
{
    if (a.n <= 0) return;
    size_t blocks = a.resetInterval == -1 ? size_t(a.n)
                                          : size_t(a.n) * ((a.srcStride + a.resetInterval - 1) / a.resetInterval);
    Carver cv(scratch);
    long long* prefix = cv.take<long long>(a.n + 1);
    float* mms = cv.take<float>(size_t(a.n) * a.srcStride);
    float* blockMax = cv.take<float>(blocks + 1);
    launch_ragged_prefix(NsrCount{a.len, a.srcStride, a.resetInterval}, a.n, prefix, h.stream());
    int grid = persistent_grid(h, reinterpret_cast<const void*>(mms_kernel), kMmsThreads, 0);
    mms_kernel<<<grid, kMmsThreads, 0, h.stream()>>>(a.src, a.srcStride, a.len, a.windowLength, a.resetInterval, mms,
                                             blockMax, prefix, a.n);
    count_launch();
    check_cuda(cudaGetLastError(), "mms_kernel");
    const int rgrid = (a.n + kRegionThreads / 32 - 1) / (kRegionThreads / 32);
    region_kernel<<<rgrid, kRegionThreads, 0, h.stream()>>>(mms, a.srcStride, a.len, a.windowLength, a.resetInterval,
                                                            a.referencePower, a.cutOff, blockMax, a.begin, a.length,
                                                            prefix, a.n);
    count_launch();
    check_cuda(cudaGetLastError(), "region_kernel");
}

}  // namespace rppb
