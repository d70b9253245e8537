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
//   1. mms_kernel:    one warp per 4 (sample, reset block) units: coalesced loads and squares by
//                     the warp, the 4 chains by 4 lanes together, MMS into scratch, block maxima;
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
        int L = min(*RPPB_RD(len + b), int(stride));
        if (L <= 0) return 0;
        long long R = block_len(L, reset);
        return (L + R - 1) / R;
    }
};

__device__ __forceinline__ float sq(float v) { return __fmul_rn(v, v); }

constexpr int kMmsThreads = 256;
constexpr int kMmsWarps = kMmsThreads / 32;
constexpr int kBlocksPerWarp = 4;            // chains per warp (lanes 0, 8, 16, 24): 2 and 8 measured slower
constexpr int kChunk = 128;                  // samples of each block per warp step
constexpr int kRowPitch = kChunk + 4;        // rows 16-byte aligned, the 4 chain lanes' quads in distinct banks
constexpr int kWarpFloats = 3 * kBlocksPerWarp * kRowPitch;   // entering, leaving, MMS rows

// One warp per 4 consecutive (sample, reset block) units; lane 8j replays block j's float chain.
// Per step of 128 samples per block the warp loads the samples entering and leaving each block's
// window (coalesced), squares them in parallel into shared memory, then the 4 chain lanes run
// their blocks' chains together over the step (two dependent adds per sample -- the only serial
// part; squares and the scaled stores are off the chain) and the warp stores the MMS values.  A
// square of zero stands for "nothing enters / leaves": sum + 0 and sum - 0 == sum exactly for the
// non-negative sums of squares, so the chain is bit-identical to the reference's conditional
// subtraction, and the padding past a shorter block's end neither changes its stored values nor
// raises its maximum.
__global__ void __launch_bounds__(kMmsThreads) mms_kernel(const float* __restrict__ src, uint32_t stride,
                                                         const int* __restrict__ len, int windowLength, int reset,
                                                         float* __restrict__ mms, float* __restrict__ blockMax,
                                                         const long long* __restrict__ prefix, int n)
{
    extern __shared__ __align__(16) float s_mms[];
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    const float meanFactor = __fdiv_rn(1.0f, float(windowLength));
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    float* qi = s_mms + wi * kWarpFloats;                 // [4][kRowPitch]
    float* qo = qi + kBlocksPerWarp * kRowPitch;
    float* vv = qo + kBlocksPerWarp * kRowPitch;
    constexpr int kLaneGap = 32 / kBlocksPerWarp;
    const int chainBlock = lane / kLaneGap;               // the block this lane replays (lanes kLaneGap * j)
    const bool chainLane = lane % kLaneGap == 0;
    // group g = 4 consecutive units; groups go to CTAs first, so every SM gets work
    for (long long g = blockIdx.x + (long long)wi * gridDim.x; g * kBlocksPerWarp < total;
         g += (long long)gridDim.x * kMmsWarps)
    {
        int bb[kBlocksPerWarp], st[kBlocksPerWarp], en[kBlocksPerWarp], pre[kBlocksPerWarp];
        int preMax = 0, blkMax = 0;
#pragma unroll
        for (int j = 0; j < kBlocksPerWarp; ++j)
        {
            const long long w = g * kBlocksPerWarp + j;
            bb[j] = 0, st[j] = 0, en[j] = 0, pre[j] = 0;
            if (w < total)
            {
                bb[j] = ragged_find(prefix, n, w);
                const int L = min(*RPPB_RD(len + bb[j]), int(stride));
                const long long R = block_len(L, reset);
                st[j] = int((w - prefix[bb[j]]) * R);
                en[j] = int(min((long long)L, st[j] + R));
                pre[j] = max(st[j] - windowLength + 1, 0);   // fresh-sum range [pre, st) (reference :131-133)
            }
            preMax = max(preMax, st[j] - pre[j]);
            blkMax = max(blkMax, en[j] - st[j]);
        }
        float sum = 0.0f, bmax = -FLT_MAX;   // meaningful in the chain lanes
        for (int c = 0; c < preMax; c += kChunk)
        {
            // all of the step's loads are in flight before the first is used
            float r[kBlocksPerWarp][kChunk / 32];
#pragma unroll
            for (int j = 0; j < kBlocksPerWarp; ++j)
            {
                const float* x = src + size_t(bb[j]) * stride;
#pragma unroll
                for (int t = 0; t < kChunk / 32; ++t)
                {
                    const int i = pre[j] + c + lane + 32 * t;
                    r[j][t] = i < st[j] ? __ldg(RPPB_RD(x + i)) : 0.0f;
                }
            }
            if (lane < kBlocksPerWarp)   // the next steps' samples, from L2
            {
                const int i0 = pre[lane] + c + 2 * kChunk;
                l2_prefetch(src + size_t(bb[lane]) * stride + i0,
                            src + size_t(bb[lane]) * stride + max(i0, min(st[lane], i0 + 2 * kChunk)));
            }
#pragma unroll
            for (int j = 0; j < kBlocksPerWarp; ++j)
#pragma unroll
                for (int t = 0; t < kChunk / 32; ++t) qi[j * kRowPitch + lane + 32 * t] = sq(r[j][t]);
            __syncwarp();
            if (chainLane)
            {
                const float* row = qi + chainBlock * kRowPitch;
                for (int k = 0; k < kChunk; k += 4)
                {
                    const float4 a4 = *reinterpret_cast<const float4*>(row + k);
                    sum = __fadd_rn(sum, a4.x);
                    sum = __fadd_rn(sum, a4.y);
                    sum = __fadd_rn(sum, a4.z);
                    sum = __fadd_rn(sum, a4.w);
                }
            }
            __syncwarp();
        }
        // software-pipelined: the next step's loads are issued before this step's chains run
        float ri[kBlocksPerWarp][kChunk / 32], ro[kBlocksPerWarp][kChunk / 32];
        auto load_step = [&](int c) {
#pragma unroll
            for (int j = 0; j < kBlocksPerWarp; ++j)
            {
                const float* x = src + size_t(bb[j]) * stride;
#pragma unroll
                for (int t = 0; t < kChunk / 32; ++t)
                {
                    const int i = st[j] + c + lane + 32 * t, o = i - windowLength + 1;
                    const bool live = i < en[j];
                    ri[j][t] = live ? __ldg(RPPB_RD(x + i)) : 0.0f;
                    ro[j][t] = live && o >= 0 ? __ldg(RPPB_RD(x + o)) : 0.0f;
                }
            }
            if (lane < kBlocksPerWarp)   // later steps' entering samples, from L2
            {
                const int i0 = st[lane] + c + 2 * kChunk;
                l2_prefetch(src + size_t(bb[lane]) * stride + i0,
                            src + size_t(bb[lane]) * stride + max(i0, min(en[lane], i0 + 2 * kChunk)));
            }
        };
        if (blkMax > 0) load_step(0);
        for (int c = 0; c < blkMax; c += kChunk)
        {
#pragma unroll
            for (int j = 0; j < kBlocksPerWarp; ++j)
#pragma unroll
                for (int t = 0; t < kChunk / 32; ++t)
                {
                    qi[j * kRowPitch + lane + 32 * t] = sq(ri[j][t]);
                    qo[j * kRowPitch + lane + 32 * t] = sq(ro[j][t]);
                }
            if (c + kChunk < blkMax) load_step(c + kChunk);
            __syncwarp();
            if (chainLane)
            {
                const float* ri = qi + chainBlock * kRowPitch;
                const float* ro = qo + chainBlock * kRowPitch;
                float* rv = vv + chainBlock * kRowPitch;
                for (int k = 0; k < kChunk; k += 4)
                {
                    const float4 a4 = *reinterpret_cast<const float4*>(ri + k);
                    const float4 o4 = *reinterpret_cast<const float4*>(ro + k);
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
                    bmax = fmaxf(fmaxf(bmax, fmaxf(v4.x, v4.y)), fmaxf(v4.z, v4.w));
                    *reinterpret_cast<float4*>(rv + k) = v4;
                }
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < kBlocksPerWarp; ++j)
            {
                float* m = mms + size_t(bb[j]) * stride;
#pragma unroll
                for (int k = lane; k < kChunk; k += 32)
                    if (st[j] + c + k < en[j]) *RPPB_WR(m + (st[j] + c + k)) = vv[j * kRowPitch + k];
            }
            __syncwarp();
        }
        // chain lane 8j holds block j's maximum (values past a shorter block's end are below its last)
#pragma unroll
        for (int j = 0; j < kBlocksPerWarp; ++j)
        {
            const float bm = __shfl_sync(0xffffffffu, bmax, kLaneGap * j);
            const long long w = g * kBlocksPerWarp + j;
            if (lane == 0 && w < total) *RPPB_WR(blockMax + w) = bm;
        }
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
    const int L = min(*RPPB_RD(len + b), int(stride));
    if (L <= 0)
    {
        if (lane == 0) { *RPPB_WR(outBegin + b) = 0; *RPPB_WR(outLength + b) = 0; }
        return;
    }
    const long long R = block_len(L, reset);
    const long long u0 = prefix[b], u1 = prefix[b + 1];
    const int nb = int(u1 - u0);
    float base = referencePower;
    if (referencePower == 0.0f)
    {
        float m = -FLT_MAX;
        for (int k = lane; k < nb; k += 32) m = fmaxf(m, *RPPB_RD(blockMax + (u0 + k)));
        base = warp_max(m);
    }
    const float cutOffMag = __fmul_rn(base, cutOff);
    const float* m = mms + size_t(b) * stride;

    // first block whose maximum reaches the cutoff, then the first index inside it
    int firstBlock = -1;
    for (int k0 = 0; k0 < nb && firstBlock < 0; k0 += 32)
    {
        const int k = k0 + lane;
        unsigned hit = __ballot_sync(0xffffffffu, k < nb && *RPPB_RD(blockMax + (u0 + k)) >= cutOffMag);
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
            unsigned hit = __ballot_sync(0xffffffffu, i < s1 && *RPPB_RD(m + i) >= cutOffMag);
            if (hit) beginIdx = i0 + __ffs(hit) - 1;
        }
        int lastBlock = -1;
        for (int k1 = nb - 1; k1 >= 0 && lastBlock < 0; k1 -= 32)
        {
            const int k = k1 - lane;
            unsigned hit = __ballot_sync(0xffffffffu, k >= 0 && *RPPB_RD(blockMax + (u0 + k)) >= cutOffMag);
            if (hit) lastBlock = k1 - (__ffs(hit) - 1);
        }
        int endIdx = -1;
        const int e0 = int(lastBlock * R), e1 = int(min((long long)L, e0 + R));
        for (int i1 = e1 - 1; i1 >= e0 && endIdx < 0; i1 -= 32)
        {
            const int i = i1 - lane;
            unsigned hit = __ballot_sync(0xffffffffu, i >= e0 && *RPPB_RD(m + i) >= cutOffMag);
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
        *RPPB_WR(outBegin + b) = detectBegin;
        *RPPB_WR(outLength + b) = detectLength;
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
    const size_t smem = size_t(kMmsWarps) * kWarpFloats * sizeof(float);
    int grid = persistent_grid(h, reinterpret_cast<const void*>(mms_kernel), kMmsThreads, smem);
    mms_kernel<<<grid, kMmsThreads, smem, h.stream()>>>(a.src, a.srcStride, a.len, a.windowLength, a.resetInterval, mms,
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
