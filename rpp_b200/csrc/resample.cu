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
// One CTA of 8 + 1 warps walks the 256-output blocks: the ninth warp replays the next block's phase
// sum into shared memory (double-buffered) while the eight compute this block, one output per
// thread; when down-mixing, the block's input span is staged (down-mixed once per input sample) in
// shared memory first.  The lookup table sits in shared memory as (value, next - value) pairs when
// they fit, so a tap reads one 8-byte entry.  Compute-bound: 2 * lobes taps of ~10 float
// operations per output.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "downmix.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kBlock = 256;        // outputs per block (the reference's block size)
constexpr int kCopyChunk = 4096;   // floats per unit of an equal-rate copy
constexpr int kSpan = 4096;        // input samples of one block staged in shared memory (mono paths)

constexpr int kThreads = kBlock + 32;   // 8 warps compute outputs, the ninth replays the next unit's phases

// Shared memory (floats): the table -- as padded (value, next - value) pairs when kPairs, else
// plain -- then the staged input span.
__host__ __device__ __forceinline__ size_t resample_pair_entries(int lutSize, int padLeft, int padRight)
{
    return size_t(padLeft) + size_t(lutSize - 1) + size_t(padRight);
}
__host__ __device__ __forceinline__ size_t resample_smem_floats(const ResampleWindowDev& w, bool pairs)
{
    return (pairs ? 2 * resample_pair_entries(w.lutSize, w.padLeft, w.padRight)
                  : ((size_t(w.lutSize) + 3) & ~size_t(3))) +
           kSpan;
}
constexpr size_t kPairTableLimit = 200 * 1024;   // bytes of shared memory for the pair layout

// Pair-table padding: a tap's x lies in (-(lobes + 1), lobes + 1), so its index, trunc or floor of
// x * scale + center, lies within [center - (lobes + 1)|scale| - 2, center + (lobes + 1)|scale| + 2].
// Whether every table position a tap can produce lies in [0, 2^22): the bound the magic-number index of
// Win<kPairs, true> needs (with the pair table, whose padding covers the indices; the clamp of the plain
// table is not applied on that path).  A tap's offset x = l - phase lies in [-lobes, lobes + 1): the
// first tap is ceil(phase) - lobes (or later, at the signal's start), and float rounding keeps x >= -lobes
// because -lobes is representable; x * scale + center is then bounded by its values at the two ends.
inline bool resample_magic_ok(const ResampleWindowDev& w, bool pairs)
{
    const double a = -double(w.lobes) * double(w.scale), b = (double(w.lobes) + 1.0) * double(w.scale);
    const double lo = double(w.center) + std::min(a, b), hi = double(w.center) + std::max(a, b);
    return pairs && lo >= 0.0 && hi < 4194304.0;
}

// A power-of-two table scale (x * scale exact for every finite tap position).
inline bool resample_scale_pow2(const ResampleWindowDev& w)
{
    int e = 0;
    return w.scale > 0.f && std::isfinite(w.scale) && std::frexp(double(w.scale), &e) == 0.5;
}

inline void resample_pads(ResampleWindowDev& w)
{
    const double reach = (double(w.lobes) + 1.0) * std::fabs(double(w.scale));
    const double lo = std::floor(double(w.center) - reach) - 2.0, hi = std::ceil(double(w.center) + reach) + 2.0;
    const double padL = lo < 0.0 ? -lo : 0.0, padR = hi > double(w.lutSize - 2) ? hi - double(w.lutSize - 2) : 0.0;
    const bool ok = padL < 65536.0 && padR < 65536.0;
    w.padLeft = ok ? int(padL) : -1;
    w.padRight = ok ? int(padR) : -1;
}

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

// kMagic: the table index comes from adding 1.5 * 2^23 with rounding toward minus infinity, which leaves
// floor(locRaw) in the low mantissa bits and float(floor(locRaw)) one subtraction away, instead of two
// float <-> int conversions per tap (low-throughput instructions).  Used when the host has shown that
// every locRaw a tap can produce lies in [0, 2^22): then trunc == floor, and both are exact this way.
// The pair entry is then addressed as bias + 8 * bits(m): the shared address of entry 0 less 8 * bits of
// 1.5 * 2^23 (mod 2^32), one shift-add per tap.
// kFma: the table scale is a power of two, so x * scale is exact and x * scale + center rounds once
// either way: one fused multiply-add gives the reference's value.
template <bool kPairs, bool kMagic = false, bool kFma = false>
struct Win
{
    const float* lut;     // shared memory: the table (plain layout)
    const float2* pairs;  // shared memory: (value, next - value) at index 0 of the padded pair layout
    int lutSize;
    float scale, center;
    uint32_t bias;        // kMagic with kPairs: shared address of pairs[0] - 8 * bits(1.5 * 2^23)

    __device__ __forceinline__ float interp(int idx, float weight) const
    {
        if constexpr (kPairs)
        {
            // pairs[i] for i in [-padLeft, lutSize - 2 + padRight] holds the entry the clamped index
            // [0, lutSize - 2] selects: no clamp for the indices a tap can produce
            const float2 e = pairs[idx];
            return __fadd_rn(e.x, __fmul_rn(weight, e.y));
        }
        else
        {
            idx = min(max(idx, 0), lutSize - 2);
            const float cur = lut[idx], nxt = lut[idx + 1];
            return __fadd_rn(cur, __fmul_rn(weight, __fsub_rn(nxt, cur)));
        }
    }
    __device__ __forceinline__ float magic_floor(float locRaw) const
    {
        constexpr float kM = 12582912.0f;   // 1.5 * 2^23
        const float m = __fadd_rd(locRaw, kM);
        const float w = __fsub_rn(locRaw, __fsub_rn(m, kM));
        if constexpr (kPairs)
        {
            const uint32_t a = bias + (uint32_t(__float_as_int(m)) << 3);
            float ex, ey;
            asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(ex), "=f"(ey) : "r"(a));
            return __fadd_rn(ex, __fmul_rn(w, ey));
        }
        return interp(__float_as_int(m) - __float_as_int(kM), w);
    }
    // rppdefs.h:771-782: truncating index (the SSE lanes)
    __device__ __forceinline__ float lane(float x) const
    {
        const float locRaw = kFma ? __fmaf_rn(x, scale, center) : __fadd_rn(__fmul_rn(x, scale), center);
        if constexpr (kMagic) return magic_floor(locRaw);
        const int idx = int(locRaw);
        return interp(idx, __fsub_rn(locRaw, float(idx)));
    }
    // rppdefs.h:760-769: floor, clamped index (the scalar tail and the multi-channel path)
    __device__ __forceinline__ float scalar(float x) const
    {
        const float locRaw = kFma ? __fmaf_rn(x, scale, center) : __fadd_rn(__fmul_rn(x, scale), center);
        if constexpr (kMagic) return magic_floor(locRaw);
        const int idx = int(floorf(locRaw));
        return interp(idx, __fsub_rn(locRaw, float(idx)));
    }
};

// Where unit w of the flat work list lives and, for a resampling unit, its phases.
struct UnitInfo
{
    int b, unit, L, Csrc, C;
    float inRate, outRate;
    const float* x;
    float* y;
    uint32_t dstStride;
};

// kMix: the input is interleaved multi-channel and is down-mixed to mono on the fly (MonoMix), so
// the launch equals rppt_down_mixing_gpu followed by a mono rppt_resample_gpu.
template <bool kMix, bool kTable, bool kPairs, bool kMagic = false, bool kFma = false>
__global__ void __launch_bounds__(kThreads) resample_kernel(const float* __restrict__ src, uint32_t srcStride,
                                                            float* __restrict__ dst, uint32_t dstStride,
                                                            const float* __restrict__ inRateT,
                                                            const float* __restrict__ outRateT,
                                                            const int* __restrict__ dims, ResampleWindowDev wd,
                                                            bool normalize, const long long* __restrict__ prefix,
                                                            int n, const RppbClip* __restrict__ clips,
                                                            float outRateAll)
{
    extern __shared__ float s_lut[];   // the table, then the staged input span
    const int pairCount = kPairs ? int(resample_pair_entries(wd.lutSize, wd.padLeft, wd.padRight)) : 0;
    float* s_in = s_lut + (kPairs ? 2 * pairCount : ((wd.lutSize + 3) & ~3));
    __shared__ float s_phase[2][kBlock];
    if (kPairs)
        for (int i = threadIdx.x; i < pairCount; i += kThreads)
        {
            const int e = min(max(i - wd.padLeft, 0), wd.lutSize - 2);   // the clamped entry
            reinterpret_cast<float2*>(s_lut)[i] = make_float2(wd.lut[e], __fsub_rn(wd.lut[e + 1], wd.lut[e]));
        }
    else
        for (int i = threadIdx.x; i < wd.lutSize; i += kThreads) s_lut[i] = wd.lut[i];
    const Win<kPairs, kMagic, kFma> win{s_lut, reinterpret_cast<const float2*>(s_lut) + (kPairs ? wd.padLeft : 0),
                                        wd.lutSize, wd.scale, wd.center,
                                        uint32_t(__cvta_generic_to_shared(reinterpret_cast<const float2*>(s_lut) +
                                                                          (kPairs ? wd.padLeft : 0))) -
                                            0x5A000000u};   // 8 * 0x4B400000 mod 2^32
    const int lobes = wd.lobes;
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);   // ends with __syncthreads
    const long long total = prefix[n];

    auto info = [&](long long w) {
        UnitInfo u;
        u.b = ragged_find(prefix, n, w);
        u.unit = int(w - prefix[u.b]);
        u.L = kTable ? clips[u.b].length : dims[2 * u.b];
        u.Csrc = kTable ? 1 : dims[2 * u.b + 1];
        u.C = kMix ? 1 : u.Csrc;   // channels of the resampled signal
        u.inRate = kTable ? clips[u.b].inRate : inRateT[u.b];
        u.outRate = kTable ? outRateAll : outRateT[u.b];
        u.x = kTable ? clips[u.b].src : src + size_t(u.b) * srcStride;
        u.y = kTable ? clips[u.b].work : dst + size_t(u.b) * dstStride;
        u.dstStride = kTable ? 0x7fffffffu : dstStride;   // a clip's work buffer holds the whole resampled clip
        return u;
    };
    // the reference's phase sum of a resampling unit (one thread; replayed in its float order)
    auto phases = [&](long long w, float* out) {
        if (w >= total) return;
        const UnitInfo u = info(w);
        if (u.inRate == u.outRate || (kMix && u.Csrc > 64)) return;
        const double scale = __ddiv_rn(double(u.inRate), double(u.outRate));
        const float fscale = __double2float_rn(scale);
        const double inBlockRaw = __dmul_rn(double(u.unit * kBlock), scale);
        float p = __double2float_rn(__dsub_rn(inBlockRaw, double(int(inBlockRaw))));
        for (int k = 0; k < kBlock; ++k)
        {
            out[k] = p;
            p = __fadd_rn(p, fscale);
        }
    };

    if (threadIdx.x == kBlock) phases(blockIdx.x, s_phase[0]);
    __syncthreads();
    int cur = 0;
    for (long long w = blockIdx.x; w < total; w += gridDim.x, cur ^= 1)
    {
        if (threadIdx.x >= kBlock)
        {
            // the ninth warp: the next unit's phases while the others compute this one
            if (threadIdx.x == kBlock) phases(w + gridDim.x, s_phase[cur ^ 1]);
        }
        else
        {
            const UnitInfo u = info(w);
            const float* x = u.x;
            float* y = u.y;
            const int L = u.L, Csrc = u.Csrc, C = u.C;
            const MonoMix mix{x, kMix ? Csrc : 1, kMix ? MonoMix::weight(max(Csrc, 1), normalize) : 1.f};
            if (kMix && Csrc > 64)
            {
                // not handled here (rejected by the caller)
            }
            else if (u.inRate == u.outRate)
            {
                if (kMix)
                {
                    const long long count = min((long long)L, (long long)u.dstStride);
                    for (long long i = (long long)u.unit * kCopyChunk + threadIdx.x;
                         i < min(count, (long long)(u.unit + 1) * kCopyChunk); i += kBlock)
                        y[i] = mix(i);
                }
                else
                {
                    const long long count =
                        kTable ? (long long)L : min((long long)L * C, (long long)min(srcStride, u.dstStride));
                    for (long long i = (long long)u.unit * kCopyChunk + threadIdx.x;
                         i < min(count, (long long)(u.unit + 1) * kCopyChunk); i += kBlock)
                        y[i] = x[i];
                }
            }
            else
            {
                const float* ph = s_phase[cur];
                const int outEnd = min(out_length(L, u.inRate, u.outRate), int(u.dstStride / uint32_t(C)));
                const double scale = __ddiv_rn(double(u.inRate), double(u.outRate));
                const int outBlock = u.unit * kBlock;
                const int inBlockRounded = int(__dmul_rn(double(outBlock), scale));
                const float* in = x + (long long)inBlockRounded * C;
                // down-mixing path: the unit's input span [lo, hi), down-mixed once per sample, goes to
                // shared memory (every tap of the unit lies inside it because the phases increase);
                // plain mono input is read through L1 directly, which measured faster than staging it
                int lo = 0;
                bool staged = false;
                if (kMix)
                {
                    const int cnt = min(kBlock, outEnd - outBlock);
                    if (cnt > 0)
                    {
                        lo = max(int(ceilf(ph[0])) - lobes, -inBlockRounded);
                        const int hi = min(int(ceilf(ph[cnt - 1])) + lobes, L - inBlockRounded);
                        staged = hi - lo <= kSpan;
                        if (staged)
                            for (int i = threadIdx.x; i < hi - lo; i += kBlock)
                                s_in[i] = mix((long long)inBlockRounded + lo + i);
                    }
                    asm volatile("bar.sync 1, %0;" ::"n"(kBlock) : "memory");   // the compute warps only
                }
                const int outPos = outBlock + threadIdx.x;
                if (outPos < outEnd)
                {
                    const float inPos = ph[threadIdx.x];
                    const int xc = int(ceilf(inPos));
                    int loc0 = xc - lobes, loc1 = xc + lobes;
                    if (loc0 + inBlockRounded < 0) loc0 = -inBlockRounded;
                    if (loc1 + inBlockRounded > L) loc1 = L - inBlockRounded;
                    if (kMix || C == 1)
                    {
                        // mono input: 4 lanes, folded as (l0 + l2) + (l1 + l3), then a scalar tail
                        auto taps = [&](auto at) {
                            int l = loc0;
                            const float locBegin = __fsub_rn(float(l), inPos);
                            float lane[4] = {__fadd_rn(locBegin, 0.f), __fadd_rn(locBegin, 1.f),
                                             __fadd_rn(locBegin, 2.f), __fadd_rn(locBegin, 3.f)};
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
                            return accum;
                        };
                        float r;
                        if (kMix && staged) r = taps([&](int l) { return s_in[l - lo]; });
                        else if (kMix) r = taps([&](int l) { return mix((long long)inBlockRounded + l); });
                        else r = taps([&](int l) { return __ldg(in + l); });
                        y[outPos] = r;
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
            }
        }
        __syncthreads();   // s_phase[cur] is rewritten two units on; s_phase[cur ^ 1] is ready
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
    ResampleWindowDev w = win;
    resample_pads(w);
    const bool pairs = w.padLeft >= 0 && resample_smem_floats(w, true) * sizeof(float) <= kPairTableLimit;
    const size_t smem = resample_smem_floats(w, pairs) * sizeof(float);
    auto go = [&](auto kernel) {
        const int grid = persistent_grid(h, reinterpret_cast<const void*>(kernel), kThreads, smem);
        kernel<<<grid, kThreads, smem, h.stream()>>>(src, srcStride, dst, dstStride, inRate, outRate, dims, w,
                                                     normalize, prefix, n, nullptr, 0.f);
    };
    const bool magic = resample_magic_ok(w, pairs);
    const bool fma = resample_scale_pow2(w);
    if (downmix && magic && fma) go(resample_kernel<true, false, true, true, true>);
    else if (downmix && magic) go(resample_kernel<true, false, true, true>);
    else if (downmix && pairs) go(resample_kernel<true, false, true>);
    else if (downmix) go(resample_kernel<true, false, false>);
    else if (magic && fma) go(resample_kernel<false, false, true, true, true>);
    else if (magic) go(resample_kernel<false, false, true, true>);
    else if (pairs) go(resample_kernel<false, false, true>);
    else go(resample_kernel<false, false, false>);
    count_launch();
    check_cuda(cudaGetLastError(), "resample_kernel");
}

void launch_resample_clips(Handle& h, void* scratch, const RppbClip* clips, int n, float outRate,
                           const ResampleWindowDev& win)
{
    if (n <= 0) return;
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(ResampleCount{nullptr, nullptr, nullptr, false, clips, outRate}, n, prefix, h.stream());
    ResampleWindowDev w = win;
    resample_pads(w);
    const bool pairs = w.padLeft >= 0 && resample_smem_floats(w, true) * sizeof(float) <= kPairTableLimit;
    const size_t smem = resample_smem_floats(w, pairs) * sizeof(float);
    auto go = [&](auto kernel) {
        const int grid = persistent_grid(h, reinterpret_cast<const void*>(kernel), kThreads, smem);
        kernel<<<grid, kThreads, smem, h.stream()>>>(nullptr, 0, nullptr, 0, nullptr, nullptr, nullptr, w, false,
                                                     prefix, n, clips, outRate);
    };
    if (resample_magic_ok(w, pairs) && resample_scale_pow2(w)) go(resample_kernel<false, true, true, true, true>);
    else if (resample_magic_ok(w, pairs)) go(resample_kernel<false, true, true, true>);
    else if (pairs) go(resample_kernel<false, true, true>);
    else go(resample_kernel<false, true, false>);
    count_launch();
    check_cuda(cudaGetLastError(), "resample_kernel(clips)");
}

}  // namespace rppb
