// resample: band-limited interpolation with the caller's windowed-sinc lookup table.
//
// Reference: src/modules/tensor/cpu/kernel/resample.cpp:46-141 and RpptResamplingWindow
// (api/rppdefs.h:751-790).  Output length ceil(length * outRate / inRate) (float arithmetic);
// equal rates copy.  Outputs go in blocks of 256: a block's origin in the input is FP64
// (outBlock * inRate/outRate), split into an integer sample and a float phase, and the phase
// advances by the float ratio once per output — a sequential float sum the GPU replays in the
// same order.  Output j sums input samples [ceil(phase) - lobes, ceil(phase) + lobes) clipped to
// the signal, each weighted by linear interpolation in the table at x * scale + center.  For
// mono input the reference sums 4 lanes (SSE; truncating table index) and folds them as
// (l0 + l2) + (l1 + l3) before a scalar tail (flooring, clamped index); multi-channel input is
// summed per channel in order.  Every product and sum is explicitly rounded, so outputs are
// bit-identical to the host path.
//
// One CTA per 256-output block: thread 0 replays the phase sum into shared memory; when down-mixing,
// the CTA then stages the block's input span (down-mixed once per input sample) in shared memory;
// every thread computes one output.  Compute-bound: 2 * lobes taps of ~10 float
// operations per output.
#include "common.cuh"
#include "downmix.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kBlock = 256;        // outputs per block (the reference's block size)
constexpr int kCopyChunk = 4096;   // floats per unit of an equal-rate copy
constexpr int kSpan = 4096;        // input samples of one block staged in shared memory (mono paths)

__host__ __device__ __forceinline__ size_t resample_smem_floats(int lutSize) { return ((lutSize + 3) & ~3) + kSpan; }

__device__ __forceinline__ int out_length(int L, float inRate, float outRate)
{
    return int(ceilf(__fdiv_rn(__fmul_rn(float(L), outRate), inRate)));
}

struct ResampleCount
{
    const float* inRate;
    const float* outRate;
    const int* dims;
    bool mix;
    const RppbClip* clips;   // table mode when set (mono, outRate = outRateAll)
    float outRateAll;
    __device__ long long operator()(int b) const
    {
        int L, C, Cs;
        float ir, orr;
        if (clips)
        {
            L = clips[b].length, C = 1, Cs = 1, ir = clips[b].inRate, orr = outRateAll;
        }
        else
        {
            L = dims[2 * b], Cs = dims[2 * b + 1], C = mix ? 1 : Cs, ir = inRate[b], orr = outRate[b];
        }
        if (L <= 0 || Cs <= 0) return 0;
        if (ir == orr) return ((long long)L * C + kCopyChunk - 1) / kCopyChunk;
        const int outEnd = out_length(L, ir, orr);
        return outEnd <= 0 ? 0 : (outEnd + kBlock - 1) / kBlock;
    }
};

struct Win
{
    const float* lut;   // shared memory
    int lutSize;
    float scale, center;

    // rppdefs.h:771-782: truncating index (the SSE lanes)
    __device__ __forceinline__ float lane(float x) const
    {
        const float locRaw = __fadd_rn(__fmul_rn(x, scale), center);
        int idx = int(locRaw);
        const float weight = __fsub_rn(locRaw, float(idx));
        idx = min(max(idx, 0), lutSize - 2);
        const float cur = lut[idx], nxt = lut[idx + 1];
        return __fadd_rn(cur, __fmul_rn(weight, __fsub_rn(nxt, cur)));
    }
    // rppdefs.h:760-769: floor, clamped index (the scalar tail and the multi-channel path)
    __device__ __forceinline__ float scalar(float x) const
    {
        const float locRaw = __fadd_rn(__fmul_rn(x, scale), center);
        int idx = int(floorf(locRaw));
        const float weight = __fsub_rn(locRaw, float(idx));
        idx = min(max(idx, 0), lutSize - 2);
        const float cur = lut[idx], nxt = lut[idx + 1];
        return __fadd_rn(cur, __fmul_rn(weight, __fsub_rn(nxt, cur)));
    }
};

// kMix: the input is interleaved multi-channel and is down-mixed to mono on the fly (MonoMix), so
// the launch equals rppt_down_mixing_gpu followed by a mono rppt_resample_gpu.
template <bool kMix, bool kTable>
__global__ void __launch_bounds__(kBlock) resample_kernel(const float* __restrict__ src, uint32_t srcStride,
                                                          float* __restrict__ dst, uint32_t dstStride,
                                                          const float* __restrict__ inRateT,
                                                          const float* __restrict__ outRateT,
                                                          const int* __restrict__ dims, ResampleWindowDev wd,
                                                          bool normalize, const long long* __restrict__ prefix, int n,
                                                          const RppbClip* __restrict__ clips, float outRateAll)
{
    extern __shared__ float s_lut[];   // the table, then the staged input span
    float* s_in = s_lut + ((wd.lutSize + 3) & ~3);
    __shared__ float s_phase[kBlock];
    for (int i = threadIdx.x; i < wd.lutSize; i += blockDim.x) s_lut[i] = wd.lut[i];
    __syncthreads();
    const Win win{s_lut, wd.lutSize, wd.scale, wd.center};
    const int lobes = wd.lobes;
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);
    const long long total = prefix[n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, n, w);
        const int unit = int(w - prefix[b]);
        const int L = kTable ? clips[b].length : dims[2 * b];
        const int Csrc = kTable ? 1 : dims[2 * b + 1];
        const int C = kMix ? 1 : Csrc;   // channels of the resampled signal
        const float inRate = kTable ? clips[b].inRate : inRateT[b];
        const float outRate = kTable ? outRateAll : outRateT[b];
        const float* x = kTable ? clips[b].src : src + size_t(b) * srcStride;
        float* y = kTable ? clips[b].work : dst + size_t(b) * dstStride;
        if (kTable) dstStride = 0x7fffffffu;   // work holds the whole resampled clip
        const MonoMix mix{x, kMix ? Csrc : 1, kMix ? MonoMix::weight(max(Csrc, 1), normalize) : 1.f};
        if (kMix && Csrc > 64) continue;
        if (inRate == outRate)
        {
            if (kMix)
            {
                const long long count = min((long long)L, (long long)dstStride);
                for (long long i = (long long)unit * kCopyChunk + threadIdx.x;
                     i < min(count, (long long)(unit + 1) * kCopyChunk); i += blockDim.x)
                    y[i] = mix(i);
                continue;
            }
            const long long count = kTable ? (long long)L : min((long long)L * C, (long long)min(srcStride, dstStride));
            for (long long i = (long long)unit * kCopyChunk + threadIdx.x; i < min(count, (long long)(unit + 1) * kCopyChunk);
                 i += blockDim.x)
                y[i] = x[i];
            continue;
        }
        const int outEnd = min(out_length(L, inRate, outRate), int(dstStride / uint32_t(C)));   // stay inside dst
        const double scale = __ddiv_rn(double(inRate), double(outRate));
        const float fscale = __double2float_rn(scale);
        const int outBlock = unit * kBlock;
        const double inBlockRaw = __dmul_rn(double(outBlock), scale);
        const int inBlockRounded = int(inBlockRaw);
        if (threadIdx.x == 0)
        {
            float p = __double2float_rn(__dsub_rn(inBlockRaw, double(inBlockRounded)));
            for (int k = 0; k < kBlock; ++k)
            {
                s_phase[k] = p;
                p = __fadd_rn(p, fscale);
            }
        }
        __syncthreads();
        const float* in = x + (long long)inBlockRounded * C;
        // down-mixing path: the block's input span [lo, hi), down-mixed once per sample, goes to
        // shared memory (every tap of the block lies inside it because the phases increase); plain
        // mono input is read through L1 directly, which measured faster than staging it
        int lo = 0;
        bool staged = false;
        if (kMix)
        {
            const int cnt = min(kBlock, outEnd - outBlock);
            if (cnt > 0)
            {
                lo = max(int(ceilf(s_phase[0])) - lobes, -inBlockRounded);
                const int hi = min(int(ceilf(s_phase[cnt - 1])) + lobes, L - inBlockRounded);
                staged = hi - lo <= kSpan;
                if (staged)
                    for (int i = threadIdx.x; i < hi - lo; i += kBlock)
                        s_in[i] = kMix ? mix((long long)inBlockRounded + lo + i) : __ldg(in + lo + i);
            }
            __syncthreads();
        }
        const int outPos = outBlock + threadIdx.x;
        if (outPos < outEnd)
        {
            const float inPos = s_phase[threadIdx.x];
            const int xc = int(ceilf(inPos));
            int loc0 = xc - lobes, loc1 = xc + lobes;
            if (loc0 + inBlockRounded < 0) loc0 = -inBlockRounded;
            if (loc1 + inBlockRounded > L) loc1 = L - inBlockRounded;
            if (kMix || C == 1)
            {
                // mono input: sample l of the block, down-mixed when kMix
                auto at = [&](int l) -> float {
                    if (staged) return s_in[l - lo];
                    return kMix ? mix((long long)inBlockRounded + l) : __ldg(in + l);
                };
                int l = loc0;
                const float locBegin = __fsub_rn(float(l), inPos);
                float lane[4] = {__fadd_rn(locBegin, 0.f), __fadd_rn(locBegin, 1.f), __fadd_rn(locBegin, 2.f),
                                 __fadd_rn(locBegin, 3.f)};
                float acc4[4] = {0.f, 0.f, 0.f, 0.f};
                for (; l + 3 < loc1; l += 4)
                {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                    {
                        acc4[j] = __fadd_rn(acc4[j], __fmul_rn(at(l + j), win.lane(lane[j])));
                        lane[j] = __fadd_rn(lane[j], 4.f);
                    }
                }
                float accum = __fadd_rn(__fadd_rn(acc4[0], acc4[2]), __fadd_rn(acc4[1], acc4[3]));
                float xx = __fsub_rn(float(l), inPos);
                for (; l < loc1; ++l, xx = __fadd_rn(xx, 1.f))
                    accum = __fadd_rn(accum, __fmul_rn(at(l), win.scalar(xx)));
                y[outPos] = accum;
            }
            else
            {
                constexpr int kMaxC = 16;
                float acc[kMaxC];
#pragma unroll
                for (int c = 0; c < kMaxC; ++c) acc[c] = 0.f;
                float xx = __fsub_rn(float(loc0), inPos);
                for (int l = loc0; l < loc1; ++l, xx = __fadd_rn(xx, 1.f))
                {
                    const float wv = win.scalar(xx);
#pragma unroll
                    for (int c = 0; c < kMaxC; ++c)
                        if (c < C) acc[c] = __fadd_rn(acc[c], __fmul_rn(__ldg(in + (long long)l * C + c), wv));
                }
#pragma unroll
                for (int c = 0; c < kMaxC; ++c)
                    if (c < C) y[(long long)outPos * C + c] = acc[c];
            }
        }
        __syncthreads();   // s_phase is rewritten by the next unit
    }
}

}  // namespace

void launch_resample(Handle& h, void* scratch, const float* src, uint32_t srcStride, float* dst, uint32_t dstStride,
                     int n, const float* inRate, const float* outRate, const int* dims, const ResampleWindowDev& win,
                     bool downmix, bool normalize)
{
    if (n <= 0) return;
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(ResampleCount{inRate, outRate, dims, downmix, nullptr, 0.f}, n, prefix, h.stream());
    const size_t smem = resample_smem_floats(win.lutSize) * sizeof(float);
    if (downmix)
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(resample_kernel<true, false>), kBlock, smem);
        resample_kernel<true, false><<<grid, kBlock, smem, h.stream()>>>(src, srcStride, dst, dstStride, inRate,
                                                                         outRate, dims, win, normalize, prefix, n,
                                                                         nullptr, 0.f);
    }
    else
    {
        int grid = persistent_grid(h, reinterpret_cast<const void*>(resample_kernel<false, false>), kBlock, smem);
        resample_kernel<false, false><<<grid, kBlock, smem, h.stream()>>>(src, srcStride, dst, dstStride, inRate,
                                                                          outRate, dims, win, normalize, prefix, n,
                                                                          nullptr, 0.f);
    }
    count_launch();
    check_cuda(cudaGetLastError(), "resample_kernel");
}

void launch_resample_clips(Handle& h, void* scratch, const RppbClip* clips, int n, float outRate,
                           const ResampleWindowDev& win)
{
    if (n <= 0) return;
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(ResampleCount{nullptr, nullptr, nullptr, false, clips, outRate}, n, prefix, h.stream());
    const size_t smem = resample_smem_floats(win.lutSize) * sizeof(float);
    int grid = persistent_grid(h, reinterpret_cast<const void*>(resample_kernel<false, true>), kBlock, smem);
    resample_kernel<false, true><<<grid, kBlock, smem, h.stream()>>>(nullptr, 0, nullptr, 0, nullptr, nullptr, nullptr,
                                                                     win, false, prefix, n, clips, outRate);
    count_launch();
    check_cuda(cudaGetLastError(), "resample_kernel(clips)");
}

}  // namespace rppb
