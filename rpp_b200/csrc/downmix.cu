// down_mixing: mono = sum over interleaved channels of x[t][c] * w[c], w = 1/channels
// (normalized to sum 1 when requested).
//
// Follows src/modules/tensor/cpu/kernel/down_mixing.cpp:42-117 including its summation order,
// so results are bit-identical: channels are taken in SIMD groups (4 lanes below 8 channels,
// 8 lanes from 8 up) whose lane sums are reduced in the order of rpp_hsum_ps
// (src/include/common/cpu/rpp_cpu_simd_math.hpp:846-867), then the leftover channels are added
// one by one; a single channel is a plain copy.  All products and sums use explicit
// round-to-nearest intrinsics so no FMA contraction changes a result.
//
// Streaming kernel: persistent CTAs over 1024-output chunks of the ragged batch; consecutive
// threads take consecutive outputs, so each warp reads one contiguous span of interleaved input.
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 1024;
constexpr int kMaxChannels = 64;

struct DownmixCount
{
    const int* dims;
    __device__ long long operator()(int b) const
    {
        int l = dims[2 * b];
        return l <= 0 ? 0 : (l + kChunk - 1) / kChunk;
    }
};

__device__ __forceinline__ float hsum4(const float* p)
{
    return __fadd_rn(__fadd_rn(p[0], p[1]), __fadd_rn(p[2], p[3]));
}
__device__ __forceinline__ float hsum8(const float* p)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(p[0], p[4]), __fadd_rn(p[2], p[6])),
                     __fadd_rn(__fadd_rn(p[1], p[5]), __fadd_rn(p[3], p[7])));
}

__global__ void __launch_bounds__(kThreads) down_mixing_kernel(const float* __restrict__ src, uint32_t srcStride,
                                                               float* __restrict__ dst, uint32_t dstStride,
                                                               const int* __restrict__ dims, bool normalize,
                                                               const long long* __restrict__ prefix, int n)
{
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const int chunk = int(w - prefix[b]);
        const int L = min(dims[2 * b], int(dstStride));   // stay inside dst
        const int C = dims[2 * b + 1];
        const float* x = src + size_t(b) * srcStride;
        float* y = dst + size_t(b) * dstStride;
        if (C <= 1)
        {
            for (int t = chunk * kChunk + threadIdx.x; t < min(L, (chunk + 1) * kChunk); t += kThreads) y[t] = x[t];
            continue;
        }
        if (C > kMaxChannels) continue;   // rejected by the dispatch layer when it can see the dims
        const float w0 = 1.f / float(C);
        float inv = 1.f;
        if (normalize)
        {
            float sum = 0.0f;
            for (int c = 0; c < C; ++c) sum = __fadd_rn(sum, w0);
            inv = __double2float_rn(__ddiv_rn(1.0, double(sum)));
        }
        const float wc = normalize ? __fmul_rn(w0, inv) : w0;   // every channel has the same weight
        const int lanes = C > 7 ? 8 : 4;
        const int aligned = (C / lanes) * lanes;
        for (int t = chunk * kChunk + threadIdx.x; t < min(L, (chunk + 1) * kChunk); t += kThreads)
        {
            const float* xs = x + size_t(t) * C;
            float acc;
            if (C == 2)
            {
                // fewer than 4 channels: the SIMD part sums nothing, both channels go through the tail
                acc = __fadd_rn(__fadd_rn(0.f, __fmul_rn(xs[0], wc)), __fmul_rn(xs[1], wc));
            }
            else
            {
                float p[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                for (int g = 0; g < aligned; g += lanes)
                    for (int l = 0; l < lanes; ++l) p[l] = __fadd_rn(p[l], __fmul_rn(xs[g + l], wc));
                acc = lanes == 8 ? hsum8(p) : hsum4(p);
                for (int c = aligned; c < C; ++c) acc = __fadd_rn(acc, __fmul_rn(xs[c], wc));
            }
            y[t] = acc;
        }
    }
}

}  // namespace

void launch_down_mixing(Handle& h, void* scratch, const float* src, uint32_t srcStride, float* dst, uint32_t dstStride, int n,
                        const int* dims, bool normalize)
{
    if (n <= 0) return;
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(DownmixCount{dims}, n, prefix, h.stream());
    int grid = persistent_grid(h, reinterpret_cast<const void*>(down_mixing_kernel), kThreads, 0);
    down_mixing_kernel<<<grid, kThreads, 0, h.stream()>>>(src, srcStride, dst, dstStride, dims, normalize, prefix, n);
    count_launch();
    check_cuda(cudaGetLastError(), "down_mixing_kernel");
}

}  // namespace rppb
