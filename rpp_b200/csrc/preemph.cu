// pre_emphasis_filter: y[0] = x[0] - c * border, y[i] = x[i] - c * x[i-1] for 0 < i < length.
//
// Follows the reference host kernel (src/modules/tensor/cpu/kernel/pre_emphasis_filter.cpp:39-71),
// whose AVX body computes x[i] - (x[i-1] * c) as a rounded product then a rounded difference
// (no FMA: the reference build passes -mno-fma); the explicit __fmul_rn/__fsub_rn keep that
// rounding, so outputs are bit-identical to the host path.  Like the host path, y[0] is written
// even for an empty sample.
//
// HBM-bound streaming kernel: persistent CTAs walk a flat list of 2048-sample chunks over the
// ragged batch; each thread moves float4s (when both tensors are 16-byte aligned per sample)
// and takes the one sample before its vector from the neighbouring lane with a shuffle.
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 2048;   // samples per work unit: 256 threads x 2 float4

struct PreemphCount
{
    const int* len;
    __device__ long long operator()(int b) const
    {
        int l = *RPPB_RD(len + b);
        return l <= 0 ? 1 : (l + kChunk - 1) / kChunk;
    }
};

template <bool kVec>
__global__ void __launch_bounds__(kThreads) pre_emphasis_kernel(const float* __restrict__ src, uint32_t srcStride,
                                                                float* __restrict__ dst, uint32_t dstStride,
                                                                const int* __restrict__ len,
                                                                const float* __restrict__ coeff, int border,
                                                                size_t srcElems, const long long* __restrict__ prefix,
                                                                int n)
{
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    const int lane = threadIdx.x & 31;
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const int chunk = int(w - prefix[b]);
        const float* x = src + size_t(b) * srcStride;
        float* y = dst + size_t(b) * dstStride;
        const int L = *RPPB_RD(len + b);
        const float c = *RPPB_RD(coeff + b);
#pragma unroll
        for (int k = 0; k < kChunk / (kThreads * 4); ++k)
        {
            const int i = chunk * kChunk + (k * kThreads + threadIdx.x) * 4;
            float v[4], prev;
            bool full = kVec && (i + 3 < L);
            if (full)
            {
                float4 q = *RPPB_RD(reinterpret_cast<const float4*>(x + i));
                v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
            }
            else
            {
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = (i + j < L) ? *RPPB_RD(x + (i + j)) : 0.f;
            }
            // x[i-1] is the previous lane's last sample, except at lane 0 of each warp.
            float up = __shfl_up_sync(0xffffffffu, v[3], 1);
            if (i == 0)
            {
                size_t base = size_t(b) * srcStride;
                prev = border == 1 ? *RPPB_RD(x) : border == 2 ? (base + 1 < srcElems ? *RPPB_RD(x + 1) : 0.f) : 0.f;
                if (L <= 0) v[0] = base < srcElems ? *RPPB_RD(x) : 0.f;
            }
            else
            {
                prev = (lane == 0 && i - 1 < L) ? *RPPB_RD(x + (i - 1)) : up;
            }
            float out[4];
            out[0] = __fsub_rn(v[0], __fmul_rn(c, prev));
#pragma unroll
            for (int j = 1; j < 4; ++j) out[j] = __fsub_rn(v[j], __fmul_rn(c, v[j - 1]));
            if (full)
            {
                *RPPB_WR(reinterpret_cast<float4*>(y + i)) = make_float4(out[0], out[1], out[2], out[3]);
            }
            else
            {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (i + j < L || i + j == 0) *RPPB_WR(y + (i + j)) = out[j];
            }
        }
    }
}

}  // namespace

void launch_pre_emphasis(Handle& h, void* scratch, const float* src, uint32_t srcStride, float* dst, uint32_t dstStride, int n,
                         const int* len, const float* coeff, int border, size_t srcElems)
{
    if (n <= 0) return;
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(PreemphCount{len}, n, prefix, h.stream());
    const bool vec = (reinterpret_cast<uintptr_t>(src) % 16 == 0) && (reinterpret_cast<uintptr_t>(dst) % 16 == 0) &&
                     (srcStride % 4 == 0) && (dstStride % 4 == 0);
    if (vec)
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(pre_emphasis_kernel<true>), kThreads, 0);
        pre_emphasis_kernel<true><<<grid, kThreads, 0, h.stream()>>>(src, srcStride, dst, dstStride, len, coeff,
                                                                     border, srcElems, prefix, n);
        count_launch();
    }
    else
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(pre_emphasis_kernel<false>), kThreads, 0);
        pre_emphasis_kernel<false><<<grid, kThreads, 0, h.stream()>>>(src, srcStride, dst, dstStride, len, coeff,
                                                                      border, srcElems, prefix, n);
        count_launch();
    }
    check_cuda(cudaGetLastError(), "pre_emphasis_kernel");
}

}  // namespace rppb
