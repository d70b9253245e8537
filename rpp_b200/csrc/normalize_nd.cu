// normalize for every element type and rank other than the 2-D F32 case (normalize.cu): U8, F16
// and I8 at ranks 1-4, F32 at ranks 1, 3 and 4.
//
// Reference: src/modules/tensor/cpu/kernel/normalize.cpp (the host path the oracle restates):
//   - F32 3-D (:122-198, :244-352, :592-730): per axis mask the statistics reduce "lines" of the
//     roi (the srcReductionDims / srcStride table), from a start offset by the first two roi
//     begins; the result is written NHWC -> NHWC, NHWC -> NCHW (mask 3), or not at all for other
//     layout pairs (the destination is only cleared);
//   - every other case (:200-242, :354-415, :472-505, :731-868): consecutive normalized axes are
//     collapsed as collapse_axis does (only the first run merges), the roi is addressed densely
//     from its begin offset (source) and from the sample start (destination), and the sums are
//     ADDED to the values already in the caller's mean / std-dev arrays.
// The host (dispatch.cu) turns each sample into a plan:
//   statistics: parameter p = row-major index over up to four parameter levels (count, source
//     stride), its lines = row-major over up to four outer levels, each line (stride, count)
//     summed by the reference's recursive halving tree and added to the running sum in order;
//   output: up to four levels (count, source stride, destination stride, parameter multiplier),
//     out = (x - mean[p]) * multiplier[p] + shift, stored as the destination type (integers
//     clamped to their range, then truncated; half rounded to nearest even).
// Kernels: zero_kernel (the sample's destination elements the output does not cover), stats_kernel
// (one thread per parameter, or one warp per parameter for lines of >= 544 elements),
// normalize_kernel (samples over the grid's rows, elements strided over its CTAs).
#include <cuda_fp16.h>

#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;

template <int TYPE>
__device__ __forceinline__ float load_elem(const void* p, size_t i)
{
    if constexpr (TYPE == kNormF32) return *RPPB_RD(static_cast<const float*>(p) + i);
    else if constexpr (TYPE == kNormF16) return __half2float(*RPPB_RD(static_cast<const __half*>(p) + i));
    else if constexpr (TYPE == kNormU8) return float(*RPPB_RD(static_cast<const unsigned char*>(p) + i));
    else return float(*RPPB_RD(static_cast<const signed char*>(p) + i));
}

template <int TYPE>
__device__ __forceinline__ void store_elem(void* p, size_t i, float v)
{
    if constexpr (TYPE == kNormF32) *RPPB_WR(static_cast<float*>(p) + i) = v;
    else if constexpr (TYPE == kNormF16) *RPPB_WR(static_cast<__half*>(p) + i) = __float2half_rn(v);
    else if constexpr (TYPE == kNormU8)
        *RPPB_WR(static_cast<unsigned char*>(p) + i) =
            static_cast<unsigned char>(__float2uint_rz(fmaxf(fminf(v, 255.f), 0.f)));
    else
        *RPPB_WR(static_cast<signed char*>(p) + i) =
            static_cast<signed char>(__float2int_rz(fmaxf(fminf(v, 127.f), -128.f)));
}

// The reference's compute_sum / compute_diff_square_sum of one line (the value the "+=" adds).
template <int TYPE, bool kSq>
__device__ float line_sum(const void* base, size_t start, long long stride, long long n, float mean)
{
    if (n > 32)
    {
        const long long h = n >> 1;
        const float a = line_sum<TYPE, kSq>(base, start, stride, h, mean);
        const float b = line_sum<TYPE, kSq>(base, start + size_t(h * stride), stride, n - h, mean);
        return __fadd_rn(a, b);
    }
    float t = 0.f;
    for (long long i = 0; i < n; ++i)
    {
        const float x = load_elem<TYPE>(base, start + size_t(i * stride));
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

// The same value with the 32 subtrees five levels down taken by the 32 lanes (n >= 544: every node
// of those levels then still splits).
template <int TYPE, bool kSq>
__device__ float warp_line_sum(const void* base, size_t start, long long stride, long long n, float mean)
{
    const int lane = threadIdx.x & 31;
    long long s0 = 0, len = n;
    for (int d = 4; d >= 0; --d)
    {
        const long long h = len >> 1;
        if ((lane >> d) & 1)
        {
            s0 += h;
            len -= h;
        }
        else
            len = h;
    }
    float v = line_sum<TYPE, kSq>(base, start + size_t(s0 * stride), stride, len, mean);
    for (int k = 0; k < 5; ++k)
    {
        const float o = __shfl_xor_sync(0xffffffffu, v, 1 << k);
        v = ((lane >> k) & 1) == 0 ? __fadd_rn(v, o) : __fadd_rn(o, v);
    }
    return v;
}

// Sum of parameter p over its lines in order, onto `init`.
template <int TYPE, bool kSq>
__device__ float param_sum(const NormNdArgs& a, const NormNdSample& s, const void* src, uint32_t p, float init,
                           float mean, bool warp)
{
    size_t base = s.srcBase;
    uint32_t rem = p;
    for (int l = s.pLevels - 1; l >= 0; --l)
    {
        const uint32_t c = rem % s.pCount[l];
        rem /= s.pCount[l];
        base += size_t(c) * s.pStride[l];
    }
    uint32_t lines = 1;
    for (int l = 0; l < s.oLevels; ++l) lines *= s.oCount[l];
    float acc = init;
    for (uint32_t q = 0; q < lines; ++q)
    {
        size_t off = base;
        uint32_t r = q;
        for (int l = s.oLevels - 1; l >= 0; --l)
        {
            const uint32_t c = r % s.oCount[l];
            r /= s.oCount[l];
            off += size_t(c) * s.oStride[l];
        }
        const float t = warp ? warp_line_sum<TYPE, kSq>(src, off, s.lineStride, s.lineCount, mean)
                             : line_sum<TYPE, kSq>(src, off, s.lineStride, s.lineCount, mean);
        acc = __fadd_rn(acc, t);
    }
    return acc;
}

// tasks: (sample, first parameter, parameters, warp mode)
template <int TYPE>
__global__ void __launch_bounds__(kThreads) stats_kernel(NormNdArgs a, const int4* __restrict__ tasks, int numTasks)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * kThreads) >> 5;
    for (int t = (blockIdx.x * kThreads + threadIdx.x) >> 5; t < numTasks; t += warps)
    {
        const int4 task = *RPPB_RD(tasks + t);
        const int b = task.x;
        const NormNdSample s = *RPPB_RD(a.samples + b);
        const void* src = static_cast<const char*>(a.src) + size_t(b) * a.srcStride0 * a.srcElem;
        auto one = [&](uint32_t p, bool warp) {
            const size_t q = size_t(b) * a.maxSize + p;
            float mean;
            if (a.compute & 1)
            {
                const float init = s.accumulate ? *RPPB_RD(a.meanOut + q) : 0.f;
                mean = __fmul_rn(param_sum<TYPE, false>(a, s, src, p, init, 0.f, warp), s.normFactor);
            }
            else
                mean = *RPPB_RD(a.meanIn + q);
            float inv = 0.f;
            if (a.compute & 2)
            {
                const float init = s.accumulate ? *RPPB_RD(a.invOut + q) : 0.f;
                const float x = __fmul_rn(param_sum<TYPE, true>(a, s, src, p, init, mean, warp), s.normFactor);
                inv = x != 0.f ? __fmul_rn(__frsqrt_rn(x), a.scale) : 0.f;
            }
            if (!warp || lane == 0)
            {
                if (a.compute & 1) *RPPB_WR(a.meanOut + q) = mean;
                if (a.compute & 2) *RPPB_WR(a.invOut + q) = inv;
            }
        };
        if (task.w) one(uint32_t(task.y), true);
        else if (lane < task.z) one(uint32_t(task.y + lane), false);
    }
}

// Clears destination elements [zeroFrom, dstStride0) of every sample.
template <int TYPE>
__global__ void __launch_bounds__(kThreads) zero_kernel(NormNdArgs a)
{
    for (int b = blockIdx.y; b < a.n; b += gridDim.y)
    {
        const size_t zeroFrom = RPPB_RD(a.samples + b)->zeroFrom;
        void* dst = static_cast<char*>(a.dst) + size_t(b) * a.dstStride0 * a.dstElem;
        for (size_t i = zeroFrom + size_t(blockIdx.x) * kThreads + threadIdx.x; i < a.dstStride0;
             i += size_t(gridDim.x) * kThreads)
            store_elem<TYPE>(dst, i, 0.f);
    }
}

template <int TYPE>
__global__ void __launch_bounds__(kThreads) normalize_kernel(NormNdArgs a, const float* __restrict__ mean,
                                                             const float* __restrict__ inv, int paramOffsetPerSample)
{
    for (int b = blockIdx.y; b < a.n; b += gridDim.y)
    {
        const NormNdSample s = *RPPB_RD(a.samples + b);
        const void* src = static_cast<const char*>(a.src) + size_t(b) * a.srcStride0 * a.srcElem;
        void* dst = static_cast<char*>(a.dst) + size_t(b) * a.dstStride0 * a.dstElem;
        const float* m = mean + size_t(b) * paramOffsetPerSample;
        const float* iv = inv + size_t(b) * paramOffsetPerSample;
        for (size_t e = size_t(blockIdx.x) * kThreads + threadIdx.x; e < s.elems; e += size_t(gridDim.x) * kThreads)
        {
            size_t so = s.srcBase, dof = 0, rem = e;
            uint32_t p = 0;
            for (int l = s.levels - 1; l >= 0; --l)
            {
                const size_t c = rem % s.lv[l].count;
                rem /= s.lv[l].count;
                so += c * s.lv[l].srcStride;
                dof += c * s.lv[l].dstStride;
                p += uint32_t(c) * s.lv[l].paramMult;
            }
            const float x = load_elem<TYPE>(src, so);
            store_elem<TYPE>(dst, dof, __fadd_rn(__fmul_rn(__fsub_rn(x, *RPPB_RD(m + p)), *RPPB_RD(iv + p)), a.shift));
        }
    }
}

// Given std devs (nothing computed): scale / stdDev, 1 where it is 0, shared by every sample.
__global__ void __launch_bounds__(kThreads) invert_kernel(const float* __restrict__ std, float* __restrict__ inv,
                                                         int count, float scale)
{
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < count; i += gridDim.x * kThreads)
    {
        const float v = *RPPB_RD(std + i);
        *RPPB_WR(inv + i) = v == 0.f ? 1.0f : __fdiv_rn(scale, v);
    }
}

template <int TYPE>
void launch_type(Handle& h, const NormNdArgs& a, const int4* tasks, int numTasks, const float* meanEff,
                 const float* invEff, int paramOffsetPerSample, size_t maxElems, size_t maxZero)
{
    const dim3 block(kThreads);
    if (maxZero > 0)
    {
        const dim3 grid(unsigned(std::min<size_t>((maxZero + kThreads - 1) / kThreads, 1024)), unsigned(std::min(a.n, 65535)));
        zero_kernel<TYPE><<<grid, block, 0, h.stream()>>>(a);
        count_launch(1);
    }
    if (numTasks > 0)
    {
        const int grid = std::min((numTasks * 32 + kThreads - 1) / kThreads,
                                  persistent_grid(h, reinterpret_cast<const void*>(stats_kernel<TYPE>), kThreads, 0));
        stats_kernel<TYPE><<<std::max(grid, 1), block, 0, h.stream()>>>(a, tasks, numTasks);
        count_launch(1);
    }
    if (maxElems > 0)
    {
        const dim3 grid(unsigned(std::min<size_t>((maxElems + kThreads - 1) / kThreads, 1024)), unsigned(std::min(a.n, 65535)));
        normalize_kernel<TYPE><<<grid, block, 0, h.stream()>>>(a, meanEff, invEff, paramOffsetPerSample);
        count_launch(1);
    }
}

}  // namespace

void launch_normalize_nd(Handle& h, const NormNdArgs& a, const int4* tasks, int numTasks, const float* meanEff,
                         const float* invEff, int paramOffsetPerSample, size_t maxElems, size_t maxZero,
                         const float* stdToInvert, float* invertOut, int invertCount)
{
    if (a.n <= 0) return;
    if (invertCount > 0)
    {
        invert_kernel<<<std::min((invertCount + kThreads - 1) / kThreads, 1024), kThreads, 0, h.stream()>>>(
            stdToInvert, invertOut, invertCount, a.scale);
        count_launch(1);
    }
    switch (a.type)
    {
    case kNormF32: launch_type<kNormF32>(h, a, tasks, numTasks, meanEff, invEff, paramOffsetPerSample, maxElems, maxZero); break;
    case kNormF16: launch_type<kNormF16>(h, a, tasks, numTasks, meanEff, invEff, paramOffsetPerSample, maxElems, maxZero); break;
    case kNormU8: launch_type<kNormU8>(h, a, tasks, numTasks, meanEff, invEff, paramOffsetPerSample, maxElems, maxZero); break;
    default: launch_type<kNormI8>(h, a, tasks, numTasks, meanEff, invEff, paramOffsetPerSample, maxElems, maxZero); break;
    }
    check_cuda(cudaGetLastError(), "normalize (N-D)");
}

}  // namespace rppb
