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
// One CTA of 8 + 1 warps takes its 256-output blocks in groups of eight.  The ninth warp decodes the
// next group into shared memory: where each block lives, its output count and its phase sum, the
// eight sums side by side, one per lane.  Meanwhile the eight compute warps work through the current
// group, each taking one 32-output slice of every block of the group.  A block's first slice, the one
// with the smallest phases, falls to a different warp for each block.  When down-mixing, each warp
// stages its slice's input span (down-mixed once per input sample) in shared memory.  The lookup table
// sits in shared memory as (value, next - value) pairs when they fit, so a tap reads one 8-byte entry.
// Where a slice's phases allow it, the taps take the exact walk (resample_exact_range): each tap reads
// the entry 32 positions past the previous one and uses the same weight.  That is 4 float operations
// and 2 loads per tap, in place of ~10 operations.  Compute-bound.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "downmix.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kBlock = 256;        // outputs per block (the reference's block size)
constexpr int kCopyChunk = 4096;   // floats per unit of an equal-rate copy

constexpr int kThreads = kBlock + 32;   // 8 warps compute outputs, the ninth decodes the next group of blocks

// Shared memory (floats): the table -- as padded (value, next - value) pairs when kPairs, else
// plain -- then, when down-mixing, the staged input span.
__host__ __device__ __forceinline__ size_t resample_pair_entries(int lutSize, int padLeft, int padRight)
{
    return size_t(padLeft) + size_t(lutSize - 1) + size_t(padRight);
}
__host__ __device__ __forceinline__ size_t resample_smem_floats(const ResampleWindowDev& w, bool pairs, bool span)
{
    return (pairs ? 2 * resample_pair_entries(w.lutSize, w.padLeft, w.padRight)
                  : ((size_t(w.lutSize) + 3) & ~size_t(3))) +
           (span ? size_t(kBlock / 32) * 256 : 0);   // down-mixing: each compute warp's slice span
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

// The exact walk.  With table scale 32 and an integer center, take an output whose phase p has binary
// exponent E (p in [2^E, 2^(E+1))).  A tap at input sample l has offset l - p, a multiple of 2^(E-23)
// (l is an integer, E <= 23) with |l - p| <= lobes.  When lobes < 2^(E+1) that offset is a float, so the
// reference's float subtraction and its lane increments by 1 and 4 are exact.  The tap's table position
// 32 (l - p) + center is a multiple of 2^(E-18) (E <= 18) below center + 32 lobes; when that is below
// 2^(E+6) the position is a float too, so the fused multiply-add is exact.  The positions of consecutive
// taps then differ by exactly 32: their table indices are 32 apart and their interpolation weights equal.
// The range is empty unless the kernel takes the round-down-add index (kMagic) and the FMA position
// (kFma), whose values these are.
inline void resample_exact_range(ResampleWindowDev& w, bool magic, bool fma)
{
    w.exactMinE = 1 << 30;
    w.exactMaxE = -(1 << 30);
    if (!magic || !fma || w.scale != 32.f || w.center != std::floor(w.center) || w.lobes < 1) return;
    for (int e = -126; e <= 18; ++e)
        if (double(w.lobes) < std::ldexp(1.0, e + 1) &&
            double(w.center) + 32.0 * double(w.lobes) < std::ldexp(1.0, e + 6))
        {
            w.exactMinE = e;
            w.exactMaxE = 18;
            return;
        }
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
            const RppbClip* c = RPPB_RD(clips + b);
            L = c->length, C = 1, Cs = 1, ir = c->inRate, orr = outRateAll;
        }
        else
        {
            L = *RPPB_RD(dims + 2 * b), Cs = *RPPB_RD(dims + (2 * b + 1)), C = mix ? 1 : Cs, ir = *RPPB_RD(inRate + b),
            orr = *RPPB_RD(outRate + b);
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

// The exact walk (resample_exact_range): the pair entry at byte offset kOff from shared address a.
template <int kOff>
__device__ __forceinline__ float2 pair_at(uint32_t a)
{
    float2 v;
    asm("ld.shared.v2.f32 {%0, %1}, [%2+%3];" : "=f"(v.x), "=f"(v.y) : "r"(a), "n"(kOff));
    return v;
}

// A unit of the flat work list, decoded by the phase warp for the compute warps.
constexpr int kUnitSkip = 0, kUnitCopy = 1, kUnitResample = 2;
struct UnitInfo
{
    const float* x;        // the sample's input
    float* y;              // the sample's output
    int L, Csrc, C;        // input length, input channels, channels of the resampled signal
    int unit;              // the unit's index within its sample
    uint32_t dstStride;
    int mode;              // kUnitSkip, kUnitCopy or kUnitResample
    int outEnd;            // resampling: outputs of the sample that the destination takes
    int inBlockRounded;    // resampling: the input sample the unit's phases count from
    float wc;              // down-mixing: the weight of every channel
};

// A CTA takes its units (blockIdx.x + i * gridDim.x, i = 0, 1, ...) in groups of kGroup.  Lane j of the
// phase warp decodes unit j of the next group (the eight phase sums run side by side) while the compute
// warps work through the current group in kGroup steps: at step s, warp w takes outputs [32 s, 32 s + 32)
// of unit (w + s) mod kGroup.  A unit's first outputs have the smallest phases and are the ones the exact
// walk may not cover, so every warp takes one such slice per group and the group barrier waits for no
// single slow warp.
constexpr int kWarps = kBlock / 32;   // compute warps
constexpr int kGroup = kWarps;
constexpr int kSliceSpan = 256;       // down-mixing: input samples of one slice staged by its warp
static_assert(kGroup == kWarps && kBlock == kWarps * 32, "one 32-output slice per compute warp and step");

// kMix: the input is interleaved multi-channel and is down-mixed to mono on the fly (MonoMix), so
// the launch equals rppt_down_mixing_gpu followed by a mono rppt_resample_gpu.
template <bool kMix, bool kTable, bool kPairs, bool kMagic = false, bool kFma = false>
__global__ void __launch_bounds__(kThreads, 4)
    resample_kernel(const float* __restrict__ src, uint32_t srcStride, float* __restrict__ dst, uint32_t dstStride,
                    const float* __restrict__ inRateT, const float* __restrict__ outRateT,
                    const int* __restrict__ dims, ResampleWindowDev wd, bool normalize,
                    const long long* __restrict__ prefix, int n, const RppbClip* __restrict__ clips,
                    float outRateAll)
{
    extern __shared__ float s_lut[];   // the table, then (down-mixing) each compute warp's staged slice span
    const int pairCount = kPairs ? int(resample_pair_entries(wd.lutSize, wd.padLeft, wd.padRight)) : 0;
    float* s_spans = s_lut + (kPairs ? 2 * pairCount : ((wd.lutSize + 3) & ~3));
    __shared__ __align__(16) float s_phase[2][kGroup][kBlock];
    __shared__ UnitInfo s_unit[2][kGroup];
    if (kPairs)
        for (int i = threadIdx.x; i < pairCount; i += kThreads)
        {
            const int e = min(max(i - wd.padLeft, 0), wd.lutSize - 2);   // the clamped entry
            const float v0 = *RPPB_RD(wd.lut + e), v1 = *RPPB_RD(wd.lut + (e + 1));
            reinterpret_cast<float2*>(s_lut)[i] = make_float2(v0, __fsub_rn(v1, v0));
        }
    else
        for (int i = threadIdx.x; i < wd.lutSize; i += kThreads) s_lut[i] = *RPPB_RD(wd.lut + i);
    const Win<kPairs, kMagic, kFma> win{s_lut, reinterpret_cast<const float2*>(s_lut) + (kPairs ? wd.padLeft : 0),
                                        wd.lutSize, wd.scale, wd.center,
                                        uint32_t(__cvta_generic_to_shared(reinterpret_cast<const float2*>(s_lut) +
                                                                          (kPairs ? wd.padLeft : 0))) -
                                            0x5A000000u};   // 8 * 0x4B400000 mod 2^32
    const int lobes = wd.lobes;
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, n, s_prefix);   // ends with __syncthreads
    const long long total = prefix[n];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // the CTA's unit j of group g
    auto unit_of = [&](long long g, int j) {
        return (long long)blockIdx.x + (g * kGroup + j) * (long long)gridDim.x;
    };
    // decodes unit w into s_unit[slot][j]: where it lives, what it does and, for a resampling unit, the
    // reference's phase sum into s_phase[slot][j] (replayed in its float order)
    auto decode = [&](long long w, int slot, int j) {
        UnitInfo u;
        u.mode = kUnitSkip;
        if (w < total)
        {
            const int b = ragged_find(prefix, n, w);
            u.unit = int(w - prefix[b]);
            const RppbClip* clip = kTable ? RPPB_RD(clips + b) : nullptr;
            u.L = kTable ? clip->length : *RPPB_RD(dims + 2 * b);
            u.Csrc = kTable ? 1 : *RPPB_RD(dims + (2 * b + 1));
            u.C = kMix ? 1 : u.Csrc;
            const float inRate = kTable ? clip->inRate : *RPPB_RD(inRateT + b);
            const float outRate = kTable ? outRateAll : *RPPB_RD(outRateT + b);
            u.x = kTable ? clip->src : src + size_t(b) * srcStride;
            u.y = kTable ? clip->work : dst + size_t(b) * dstStride;
            u.dstStride = kTable ? 0x7fffffffu : dstStride;   // a clip's work buffer holds the whole resampled clip
            u.wc = kMix ? MonoMix::weight(max(u.Csrc, 1), normalize) : 1.f;
            u.mode = inRate == outRate ? kUnitCopy : (kMix && u.Csrc > 64) ? kUnitSkip : kUnitResample;
            u.outEnd = 0;
            u.inBlockRounded = 0;
            if (u.mode == kUnitResample)
            {
                u.outEnd = min(out_length(u.L, inRate, outRate), int(u.dstStride / uint32_t(u.C)));
                const double scale = __ddiv_rn(double(inRate), double(outRate));
                const float fscale = __double2float_rn(scale);
                const double inBlockRaw = __dmul_rn(double(u.unit * kBlock), scale);
                u.inBlockRounded = int(inBlockRaw);
                float p = __double2float_rn(__dsub_rn(inBlockRaw, double(int(inBlockRaw))));
                float4* out = reinterpret_cast<float4*>(s_phase[slot][j]);
#pragma unroll 8
                for (int k = 0; k < kBlock / 4; ++k)
                {
                    float4 q;
                    q.x = p;
                    q.y = p = __fadd_rn(p, fscale);
                    q.z = p = __fadd_rn(p, fscale);
                    q.w = p = __fadd_rn(p, fscale);
                    p = __fadd_rn(p, fscale);
                    out[k] = q;
                }
                // ask L2 for the unit's input span (a group ahead of its use): the taps of its outputs
                // read samples [ceil(first phase) - lobes, ceil(last phase) + lobes) from inBlockRounded on
                const int cnt = min(kBlock, u.outEnd - u.unit * kBlock);
                if (cnt > 0)
                {
                    const float* ph = s_phase[slot][j];
                    const long long lo = max((long long)u.inBlockRounded + int(ceilf(ph[0])) - lobes, 0ll);
                    const long long hi =
                        min((long long)u.inBlockRounded + int(ceilf(ph[cnt - 1])) + lobes, (long long)u.L);
                    if (hi > lo) l2_prefetch(u.x + lo * u.Csrc, u.x + hi * u.Csrc);
                }
            }
        }
        s_unit[slot][j] = u;
    };

    if (warp == kWarps && lane < kGroup) decode(unit_of(0, lane), 0, lane);
    __syncthreads();
    int cur = 0;
    for (long long g = 0; unit_of(g, 0) < total; ++g, cur ^= 1)
    {
        if (warp == kWarps)
        {
            // the phase warp: the next group while the others compute this one
            if (lane < kGroup) decode(unit_of(g + 1, lane), cur ^ 1, lane);
        }
        else
        {
            float* s_span = s_spans + warp * kSliceSpan;
            for (int step = 0; step < kGroup; ++step)
            {
                const int j = (warp + step) % kGroup;
                const UnitInfo u = s_unit[cur][j];
                const float* x = u.x;
                float* y = u.y;
                const int L = u.L, C = u.C;
                const MonoMix mix{x, kMix ? u.Csrc : 1, u.wc};
                if (u.mode == kUnitCopy)
                {
                    constexpr int kPart = kCopyChunk / kGroup;
                    const long long count =
                        kMix ? min((long long)L, (long long)u.dstStride)
                             : (kTable ? (long long)L : min((long long)L * C, (long long)min(srcStride, u.dstStride)));
                    const long long i0 = (long long)u.unit * kCopyChunk + step * kPart;
                    for (long long i = i0 + lane; i < min(count, i0 + kPart); i += 32)
                        *RPPB_WR(y + i) = kMix ? mix(i) : *RPPB_RD(x + i);
                }
                else if (u.mode == kUnitResample)
                {
                    const float* ph = s_phase[cur][j];
                    const int outBlock = u.unit * kBlock;
                    const int cnt = min(kBlock, u.outEnd - outBlock);   // outputs of the unit
                    const int k0 = step * 32;                           // the slice's first output
                    if (k0 < cnt)
                    {
                        const int inBlockRounded = u.inBlockRounded;
                        const float* in = x + (long long)inBlockRounded * C;
                        // down-mixing: the slice's input span [lo, hi), down-mixed once per sample, staged by
                        // this warp (every tap of the slice lies inside it because the phases increase)
                        int lo = 0;
                        bool staged = false;
                        if (kMix)
                        {
                            lo = max(int(ceilf(ph[k0])) - lobes, -inBlockRounded);
                            const int hi = min(int(ceilf(ph[min(k0 + 31, cnt - 1)])) + lobes, L - inBlockRounded);
                            staged = hi - lo <= kSliceSpan;
                            if (staged)
                                for (int i = lane; i < hi - lo; i += 32)
                                    s_span[i] = mix((long long)inBlockRounded + lo + i);
                            __syncwarp();
                        }
                        const int k = k0 + lane;
                        const int outPos = outBlock + k;
                        const float inPos = ph[k];
                        // the exact walk (resample_exact_range) where every output of the slice allows it,
                        // so a warp runs one of the two tap loops
                        bool exact = false;
                        if constexpr (kPairs && kMagic && kFma)
                        {
                            const int e = int((__float_as_uint(inPos) >> 23) & 0xffu) - 127;
                            exact = __all_sync(0xffffffffu, k >= cnt || (e >= wd.exactMinE && e <= wd.exactMaxE));
                        }
                        if (k < cnt)
                        {
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
                                    float lane4[4] = {__fadd_rn(locBegin, 0.f), __fadd_rn(locBegin, 1.f),
                                                      __fadd_rn(locBegin, 2.f), __fadd_rn(locBegin, 3.f)};
                                    float acc4[4] = {0.f, 0.f, 0.f, 0.f};
                                    for (; l + 3 < loc1; l += 4)
                                    {
#pragma unroll
                                        for (int q = 0; q < 4; ++q)
                                        {
                                            acc4[q] = __fadd_rn(acc4[q], __fmul_rn(at(l + q), win.lane(lane4[q])));
                                            lane4[q] = __fadd_rn(lane4[q], 4.f);
                                        }
                                    }
                                    float accum = __fadd_rn(__fadd_rn(acc4[0], acc4[2]), __fadd_rn(acc4[1], acc4[3]));
                                    float xx = __fsub_rn(float(l), inPos);
                                    for (; l < loc1; ++l, xx = __fadd_rn(xx, 1.f))
                                        accum = __fadd_rn(accum, __fmul_rn(at(l), win.scalar(xx)));
                                    return accum;
                                };
                                // the exact walk: the first tap's pair entry and weight by the same operations
                                // as above, then each tap 32 entries (256 bytes) further on at that weight; the
                                // same products and sums in the same order
                                auto taps_exact = [&](auto at) {
                                    constexpr float kM = 12582912.0f;   // 1.5 * 2^23
                                    const float locRaw =
                                        __fmaf_rn(__fsub_rn(float(loc0), inPos), win.scale, win.center);
                                    const float m = __fadd_rd(locRaw, kM);
                                    const float w = __fsub_rn(locRaw, __fsub_rn(m, kM));
                                    uint32_t a = win.bias + (uint32_t(__float_as_int(m)) << 3);
                                    auto tap = [&](int l, float2 e) {
                                        return __fmul_rn(at(l), __fadd_rn(e.x, __fmul_rn(w, e.y)));
                                    };
                                    int l = loc0;
                                    float acc4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
                                    for (; l + 3 < loc1; l += 4, a += 4 * 256)
                                    {
                                        acc4[0] = __fadd_rn(acc4[0], tap(l, pair_at<0>(a)));
                                        acc4[1] = __fadd_rn(acc4[1], tap(l + 1, pair_at<256>(a)));
                                        acc4[2] = __fadd_rn(acc4[2], tap(l + 2, pair_at<512>(a)));
                                        acc4[3] = __fadd_rn(acc4[3], tap(l + 3, pair_at<768>(a)));
                                    }
                                    float accum = __fadd_rn(__fadd_rn(acc4[0], acc4[2]), __fadd_rn(acc4[1], acc4[3]));
                                    for (; l < loc1; ++l, a += 256) accum = __fadd_rn(accum, tap(l, pair_at<0>(a)));
                                    return accum;
                                };
                                auto run = [&](auto at) {
                                    if constexpr (kPairs && kMagic && kFma)
                                        if (exact) return taps_exact(at);
                                    return taps(at);
                                };
                                float r;
                                if (kMix && staged) r = run([&](int l) { return s_span[l - lo]; });
                                else if (kMix) r = run([&](int l) { return mix((long long)inBlockRounded + l); });
                                else r = run([&](int l) { return __ldg(RPPB_RD(in + l)); });
                                *RPPB_WR(y + outPos) = r;
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
                                        if (c < C)
                                            acc[c] = __fadd_rn(acc[c],
                                                               __fmul_rn(__ldg(RPPB_RD(in + (long long)l * C + c)), wv));
                                }
#pragma unroll
                                for (int c = 0; c < kMaxC; ++c)
                                    if (c < C) *RPPB_WR(y + ((long long)outPos * C + c)) = acc[c];
                            }
                        }
                        if (kMix) __syncwarp();   // the warp's span is restaged by its next slice
                    }
                }
                // kUnitSkip: no unit, or more than 64 channels to down-mix (rejected by the caller)
            }
        }
        __syncthreads();   // slot cur is rewritten by the next group's decode; slot cur ^ 1 is ready
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
    const bool pairs = w.padLeft >= 0 && resample_smem_floats(w, true, downmix) * sizeof(float) <= kPairTableLimit;
    const size_t smem = resample_smem_floats(w, pairs, downmix) * sizeof(float);
    const bool magic = resample_magic_ok(w, pairs);
    const bool fma = resample_scale_pow2(w);
    resample_exact_range(w, magic, fma);
    auto go = [&](auto kernel) {
        const int grid = persistent_grid(h, reinterpret_cast<const void*>(kernel), kThreads, smem);
        kernel<<<grid, kThreads, smem, h.stream()>>>(src, srcStride, dst, dstStride, inRate, outRate, dims, w,
                                                     normalize, prefix, n, nullptr, 0.f);
    };
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
    const bool pairs = w.padLeft >= 0 && resample_smem_floats(w, true, false) * sizeof(float) <= kPairTableLimit;
    const size_t smem = resample_smem_floats(w, pairs, false) * sizeof(float);
    const bool magic = resample_magic_ok(w, pairs);
    const bool fma = resample_scale_pow2(w);
    resample_exact_range(w, magic, fma);
    auto go = [&](auto kernel) {
        const int grid = persistent_grid(h, reinterpret_cast<const void*>(kernel), kThreads, smem);
        kernel<<<grid, kThreads, smem, h.stream()>>>(nullptr, 0, nullptr, 0, nullptr, nullptr, nullptr, w, false,
                                                     prefix, n, clips, outRate);
    };
    if (magic && fma) go(resample_kernel<false, true, true, true, true>);
    else if (magic) go(resample_kernel<false, true, true, true>);
    else if (pairs) go(resample_kernel<false, true, true>);
    else go(resample_kernel<false, true, false>);
    count_launch();
    check_cuda(cudaGetLastError(), "resample_kernel(clips)");
}

}  // namespace rppb
