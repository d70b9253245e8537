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
#include "downmix.cuh"
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
        int l = *RPPB_RD(dims + 2 * b);
        return l <= 0 ? 0 : (l + kChunk - 1) / kChunk;
    }
};

__global__ void __launch_bounds__(kThreads) down_mixing_kernel(const float* __restrict__ src, uint32_t srcStride,
                                                               float* __restrict__ dst, uint32_t dstStride,
                                                               const int* __restrict__ dims, bool normalize,
                                                               const long long* __restrict__ prefix, int n)
{
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const int chunk = int(w - prefix[b]);
        const int L = min(*RPPB_RD(dims + 2 * b), int(dstStride));   // stay inside dst
        const int C = *RPPB_RD(dims + (2 * b + 1));
        const float* x = src + size_t(b) * srcStride;
        float* y = dst + size_t(b) * dstStride;
        if (C <= 1)
        {
            for (int t = chunk * kChunk + threadIdx.x; t < min(L, (chunk + 1) * kChunk); t += kThreads)
                *RPPB_WR(y + t) = *RPPB_RD(x + t);
            continue;
        }
        if (C > kMaxChannels) continue;   // rejected by the dispatch layer when it can see the dims
        const MonoMix mix{x, C, MonoMix::weight(C, normalize)};
        for (int t = chunk * kChunk + threadIdx.x; t < min(L, (chunk + 1) * kChunk); t += kThreads)
        {
            const float acc = mix(t);
            *RPPB_WR(y + t) = acc;
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
