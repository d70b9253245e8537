// normalize (2-D, F32): (x - mean) * invStdDev + shift over each sample's roi, per row (axisMask 2),
// per column (axisMask 1) or per sample (axisMask 3), with the statistics computed here or given.
//
// Reference: src/modules/tensor/cpu/kernel/normalize.cpp:29-120 and :417-600 (the 2-D branch that
// "is called for the audio testcase").  Per sample:
//   - the whole destination sample [0, dstStride0) is zeroed, then the roi [length0 x length1] is
//     written (the roi begins are not read);
//   - a parameter reduces R elements: mean = sum * (1/R) and invStdDev = rsqrt(sumsq * (1/R)) *
//     scale (0 where the variance is 0), the sums being the reference's recursive halving tree
//     (runs of at most 32 elements summed in order, halves added pairwise), replayed exactly;
//   - computeMeanStddev bit 0 / bit 1: mean / std dev computed here, written to the caller's
//     meanTensor / stdDevTensor (n x maxSize); otherwise read from them.  With both bits clear
//     the caller's std-dev values become scale / stdDev (1 where 0), shared by all samples.
// The sums are bit-identical to the host path; the inverse square root is CUDA's correctly rounded
// one, where the reference uses the SSE reciprocal-square-root estimate refined by one Newton step
// (about 1e-7 relative apart).
//
// Kernels: stats_kernel (only when something is computed) -- one thread per parameter for short
// reductions, one warp per parameter for long ones (the parameter's elements staged once in shared
// memory when contiguous; the 32 lanes take the 32 subtrees five levels down the same halving tree
// and combine them pairwise in tree order); normalize_kernel -- one destination row per CTA step,
// four columns per thread.  HBM-bound.
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
// warp-parallel tree from kNormalizeWarpMinElems (544) elements on: every node of the top five
// levels then holds at least floor(n / 16) >= 34 > 32 elements, so it splits as the lanes assume
static_assert(kNormalizeWarpMinElems / 16 > 32, "the warp tree's top five levels must all split");
constexpr int kStageElems = 1024;   // per warp: 4 KB of shared memory

// The reference's compute_sum / compute_diff_square_sum value (the "+= into 0" steps are exact:
// the partial sums are never -0).
template <bool kSq>
__device__ float tree_sum(const float* in, int stride, int n, float mean)
{
    if (n > 32)
    {
        const int h = n >> 1;
        const float a = tree_sum<kSq>(in, stride, h, mean);
        const float b = tree_sum<kSq>(in + (long long)h * stride, stride, n - h, mean);
        return __fadd_rn(a, b);
    }
    float t = 0.f;
    for (int i = 0; i < n; ++i)
    {
        const float x = *RPPB_RD(in + (long long)i * stride);
        if (kSq)
        {
            const float c = __fsub_rn(x, mean);
            t = __fadd_rn(t, __fmul_rn(c, c));
        }
        else
            t = __fadd_rn(t, x);
    }
    return t;
}

// Same value, the 32 subtrees five levels down summed by the 32 lanes (n >= kNormalizeWarpMinElems).
template <bool kSq>
__device__ float warp_tree_sum(const float* in, int stride, int n, float mean)
{
    const int lane = threadIdx.x & 31;
    int start = 0, len = n;
    for (int d = 4; d >= 0; --d)
    {
        const int h = len >> 1;
        if ((lane >> d) & 1)
        {
            start += h;
            len -= h;
        }
        else
            len = h;
    }
    float v = tree_sum<kSq>(in + (long long)start * stride, stride, len, mean);
    for (int k = 0; k < 5; ++k)
    {
        const float o = __shfl_xor_sync(0xffffffffu, v, 1 << k);
        const bool left = ((lane >> k) & 1) == 0;
        v = left ? __fadd_rn(v, o) : __fadd_rn(o, v);
    }
    return v;
}

__global__ void __launch_bounds__(kThreads) stats_kernel(NormalizeArgs a, const int4* __restrict__ tasks, int numTasks)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * kThreads) >> 5;
    // warp mode: a parameter's contiguous elements are read once, coalesced, into this warp's
    // buffer, and both tree sums run from there
    __shared__ float s_stage[kThreads / 32][kStageElems];
    float* stage = s_stage[threadIdx.x >> 5];
    for (int t = (blockIdx.x * kThreads + threadIdx.x) >> 5; t < numTasks; t += warps)
    {
        const int4 task = *RPPB_RD(tasks + t);   // sample, first parameter, parameters, warp mode
        const int b = task.x;
        const NormalizeSample s = *RPPB_RD(a.samples + b);
        const float* base = a.src + size_t(b) * a.srcStride0;
        auto one = [&](int p, bool warp) {
            const float* in = base + (long long)p * s.paramStride;
            int es = s.elemStride;
            if (warp && es == 1 && s.count <= kStageElems)
            {
                __syncwarp();   // the previous task's reads of the buffer are done
                for (int k = lane; k < s.count; k += 32) stage[k] = __ldg(RPPB_RD(in + k));
                __syncwarp();
                in = stage;
            }
            float mean;
            if (a.compute & 1)
            {
                const float sum = warp ? warp_tree_sum<false>(in, es, s.count, 0.f)
                                       : tree_sum<false>(in, es, s.count, 0.f);
                mean = __fmul_rn(sum, s.normFactor);
            }
            else
                mean = *RPPB_RD(a.meanIn + (size_t(b) * a.maxSize + p));
            float inv = 0.f;
            if (a.compute & 2)
            {
                const float sq = warp ? warp_tree_sum<true>(in, es, s.count, mean)
                                      : tree_sum<true>(in, es, s.count, mean);
                const float x = __fmul_rn(sq, s.normFactor);
                inv = x != 0.f ? __fmul_rn(__frsqrt_rn(x), a.scale) : 0.f;
            }
            if (!warp || lane == 0)
            {
                if (a.compute & 1) *RPPB_WR(a.meanOut + (size_t(b) * a.maxSize + p)) = mean;
                if (a.compute & 2) *RPPB_WR(a.invOut + (size_t(b) * a.maxSize + p)) = inv;
            }
        };
        if (task.w) one(task.y, true);
        else if (lane < task.z) one(task.y + lane, false);
    }
}

__global__ void __launch_bounds__(kThreads) invert_kernel(const float* __restrict__ std, float* __restrict__ inv,
                                                         int count, float scale)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < count; i += gridDim.x * kThreads)
    {
        const float v = *RPPB_RD(std + i);
        *RPPB_WR(inv + i) = v == 0.f ? 1.0f : __fdiv_rn(scale, v);
    }
}

// One destination row (dstStride1 elements of a sample) per CTA step, 4 consecutive columns per
// thread: roi elements get (x - mean) * inv + shift, the rest of the sample's stride zeros.
// 16-byte loads and stores where the strides and addresses allow.
__global__ void __launch_bounds__(kThreads) normalize_kernel(NormalizeArgs a, const float* __restrict__ mean,
                                                             const float* __restrict__ inv, int paramOffsetPerSample,
                                                             int rowsPerSample, bool vecSrc, bool vecDst)
{
    const long long units = (long long)a.n * rowsPerSample;
    for (long long u = blockIdx.x; u < units; u += gridDim.x)
    {
        const int b = int(u / rowsPerSample);
        const uint32_t r = uint32_t(u - (long long)b * rowsPerSample);
        const NormalizeSample s = *RPPB_RD(a.samples + b);
        const uint32_t rowBegin = r * a.dstStride1;
        const uint32_t rowLen = min(a.dstStride1, a.dstStride0 - rowBegin);
        float* d = a.dst + size_t(b) * a.dstStride0 + rowBegin;
        const bool rowIn = r < uint32_t(s.len0);
        const float* x = a.src + size_t(b) * a.srcStride0 + size_t(r) * a.srcStride1;
        const size_t q0 = size_t(b) * paramOffsetPerSample;
        float rowMean = 0.f, rowInv = 0.f;
        if (rowIn && a.axisMask != 1)
        {
            const size_t q = q0 + (a.axisMask == 2 ? r : 0);
            rowMean = *RPPB_RD(mean + q);
            rowInv = *RPPB_RD(inv + q);
        }
        const uint32_t len1 = rowIn ? uint32_t(s.len1) : 0u;
        for (uint32_t c = 4 * threadIdx.x; c < rowLen; c += 4 * kThreads)
        {
            float xv[4] = {0.f, 0.f, 0.f, 0.f};
            if (c + 4 <= len1 && vecSrc)
            {
                const float4 v = __ldg(RPPB_RD(reinterpret_cast<const float4*>(x + c)));
                xv[0] = v.x; xv[1] = v.y; xv[2] = v.z; xv[3] = v.w;
            }
            else
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (c + t < len1) xv[t] = __ldg(RPPB_RD(x + size_t(c + t) * a.srcStride2));
            float ov[4];
#pragma unroll
            for (int t = 0; t < 4; ++t)
            {
                float m = rowMean, iv = rowInv;
                if (a.axisMask == 1 && c + t < len1)
                {
                    m = *RPPB_RD(mean + (q0 + c + t));
                    iv = *RPPB_RD(inv + (q0 + c + t));
                }
                ov[t] = c + t < len1 ? __fadd_rn(__fmul_rn(__fsub_rn(xv[t], m), iv), a.shift) : 0.f;
            }
            if (c + 4 <= rowLen && vecDst)
                *RPPB_WR(reinterpret_cast<float4*>(d + c)) = make_float4(ov[0], ov[1], ov[2], ov[3]);
            else
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (c + t < rowLen) *RPPB_WR(d + (c + t)) = ov[t];
        }
    }
}

}  // namespace

void launch_normalize(Handle& h, const NormalizeArgs& a, const int4* tasks, int numTasks, const float* meanEff,
                      const float* invEff, int paramOffsetPerSample, const float* stdToInvert, float* invertOut,
                      int invertCount)
{
    if (a.n <= 0) return;
    if (invertCount > 0)
    {
        invert_kernel<<<std::min((invertCount + kThreads - 1) / kThreads, 1024), kThreads, 0, h.stream()>>>(
            stdToInvert, invertOut, invertCount, a.scale);
        count_launch(1);
    }
    if (numTasks > 0)
    {
        const int grid = std::min((numTasks * 32 + kThreads - 1) / kThreads,
                                  persistent_grid(h, reinterpret_cast<const void*>(stats_kernel), kThreads, 0));
        stats_kernel<<<std::max(grid, 1), kThreads, 0, h.stream()>>>(a, tasks, numTasks);
        count_launch(1);
    }
    if (a.dstStride0 > 0)
    {
        const int rowsPerSample = int((a.dstStride0 + a.dstStride1 - 1) / a.dstStride1);
        const long long units = (long long)a.n * rowsPerSample;
        const bool vecSrc = a.srcStride2 == 1 && (a.srcStride0 & 3) == 0 && (a.srcStride1 & 3) == 0 &&
                            (reinterpret_cast<uintptr_t>(a.src) & 15) == 0;
        const bool vecDst = (a.dstStride0 & 3) == 0 && (a.dstStride1 & 3) == 0 &&
                            (reinterpret_cast<uintptr_t>(a.dst) & 15) == 0;
        const int grid = int(std::min<long long>(
            units, persistent_grid(h, reinterpret_cast<const void*>(normalize_kernel), kThreads, 0)));
        normalize_kernel<<<grid, kThreads, 0, h.stream()>>>(a, meanEff, invEff, paramOffsetPerSample, rowsPerSample,
                                                            vecSrc, vecDst);
        count_launch(1);
    }
    check_cuda(cudaGetLastError(), "normalize");
}

}  // namespace rppb
