// The fused front end's work queue and mel tables, shared by its two spectrum engines (fused.cu: the
// FP32 register FFT, bit-identical to the plain calls; fused_tc.cu: the factored DFT on tensor cores).
//
// Work items of two kinds walk one queue, claimed in order with an atomic counter: spectrum items
// (a clip's frames f0 .. f0 + tiles * TF) and decibel items (a clip's frames, converted in place once
// all of the clip's spectrum items are counted), interleaved per clip slot so that a clip's decibels
// run `lookahead` clips after its spectrum.  Included once per translation unit (internal linkage).
#pragma once

#include <cfloat>

#include <algorithm>
#include <cstring>
#include <string>

#include "common.cuh"
#include "handle.hpp"
#include "mel_tables.cuh"
#include "ops.hpp"
#include "stft.cuh"

namespace rppb {

constexpr int kFusedThreads = 256;
constexpr int kDbFramesDefault = 128;         // frames per decibel item unless tuned
constexpr int kSubTilesDefault = 2;           // spectrum tiles per spectrum item unless tuned
constexpr int kFusedPrefixCache = 320;        // slots cached in shared memory (n + lookahead + 1)
constexpr long long kWaitLimit = 1ll << 24;   // x ~128 ns sleeps: a few seconds
constexpr long long kInjectedWaitLimit = 1024; // wait fault injection: ~0.1 ms per decibel item

namespace {

// Where clip b lives: uniform-stride batch, or one entry of a clip table.
struct ClipView
{
    const float* x;
    int L;
    float* y;
    uint32_t hStride;
    int maxFrames;
    float coeff;
    bool hasSecond;   // x[1] may be read (REFLECT border of a 1-sample clip)
};

__device__ __forceinline__ ClipView clip_view(const FrontendArgs& a, int b)
{
    if (a.clips)
    {
        const RppbClip c = *RPPB_RD(a.clips + b);
        const int L = c.length <= 0 ? 0 : resampled_length(c.length, c.inRate, a.outRate);
        return {c.work, L, c.dst, uint32_t(c.dstStride), c.dstStride, a.coeffAll, L >= 2};
    }
    return {a.src + size_t(b) * a.srcStride, *RPPB_RD(a.len + b), a.dst + size_t(b) * a.dstNStride, a.dstHStride,
            a.maxFrames, *RPPB_RD(a.coeff + b), size_t(b) * a.srcStride + 1 < a.srcElems};
}

template <int TF>
struct SlotCount
{
    FrontendArgs a;
    int n, D;
    __device__ int frames(int b) const
    {
        const ClipView c = clip_view(a, b);
        return max(0, min(num_windows(c.L, a.W, a.hop, a.center), c.maxFrames));
    }
    // spectrum items of clip b: subTiles tiles of TF frames each
    __device__ int tiles(int b) const { return (frames(b) + TF * a.subTiles - 1) / (TF * a.subTiles); }
    __device__ int db_tiles(int b) const { return (frames(b) + a.dbFrames - 1) / a.dbFrames; }
    __device__ long long operator()(int s) const
    {
        long long c = 0;
        if (s < n) c += tiles(s);
        if (s - D >= 0 && s - D < n) c += db_tiles(s - D);
        return c;
    }
};

// One claimed work item, decoded by thread 0 and handed to the CTA through shared memory.
struct Item
{
    const float* x;
    float* y;          // clip output at the item's first frame
    uint32_t hs;
    int L, F, f0, Tv, b;
    int kind;          // 0 spectrum tile, 1 decibel tile, -1 queue exhausted
    float coeff, bval;
};

template <int TF>
__device__ Item decode_item(const FrontendArgs& a, const SlotCount<TF>& cnt, const long long* prefix, int nslots,
                            long long total, long long w)
{
    Item it{};
    if (w >= total)
    {
        it.kind = -1;
        return it;
    }
    const int s = ragged_find(prefix, nslots, w);
    const int local = int(w - prefix[s]);
    const int c1 = s < a.n ? cnt.tiles(s) : 0;
    const bool spectrumItem = local < c1;
    it.kind = spectrumItem ? 0 : 1;
    it.b = spectrumItem ? s : s - a.lookahead;
    const int tile = spectrumItem ? local : local - c1;
    const ClipView cv = clip_view(a, it.b);
    it.x = cv.x;
    it.L = cv.L;
    it.F = min(num_windows(cv.L, a.W, a.hop, a.center), cv.maxFrames);
    const int itemFrames = spectrumItem ? TF * a.subTiles : a.dbFrames;
    it.f0 = tile * itemFrames;
    it.Tv = min(itemFrames, it.F - it.f0);
    it.y = cv.y + it.f0;
    it.hs = cv.hStride;
    it.coeff = cv.coeff;
    it.bval = 0.f;
    if (spectrumItem && a.border == 1) it.bval = *RPPB_RD(cv.x);
    else if (spectrumItem && a.border == 2 && cv.hasSecond) it.bval = *RPPB_RD(cv.x + 1);
    return it;
}

// Shared memory plan (bytes), computed identically on host and device.
template <int NFFT, int TF>
struct FusedLayout
{
    using S = StftShape<NFFT, kFusedThreads, TF>;
    size_t tw, tw1, win, span, work, melW, melIv, melGrp, total;
    __host__ __device__ FusedLayout(int numFilter, int W, int hop)
    {
        const int bins = S::BINS;
        tw = 0;
        tw1 = tw + S::tw_bytes;
        win = tw1 + S::tw1_bytes;
        span = win + size_t(NFFT) * 4;
        work = span + S::span_bytes(W, hop);
        // the FFT slots + power tile, or (before the loop) the mel table build
        size_t fftOut = S::fft_bytes + S::out_bytes;
        size_t tables = 2 * size_t(numFilter + 2) * 4 + size_t(numFilter) * 4 + 2 * size_t(numFilter + 1) * 8 +
                        size_t(bins) * 4 + 64;
        size_t workBytes = (fftOut > tables ? fftOut : tables);
        melW = (work + workBytes + 15) & ~size_t(15);
        melIv = (melW + size_t(bins) * 8 + 15) & ~size_t(15);
        melGrp = (melIv + size_t(numFilter + 1) * 8 + 15) & ~size_t(15);
        total = (melGrp + size_t(2 * kFusedThreads / TF + 1) * 4 + 15) & ~size_t(15);
    }
};

// The fused kernel's mel tables in its shared-memory layout, built by the whole CTA in the work region
// (free until the first FFT); ends with __syncthreads.  Mel weights by bin: bin k of interval i (between
// mel points i and i + 1) weighs (1 - wd_k) * norm_i into filter i and wd_k * norm_(i-1) into filter
// i - 1, so filter m sums interval m's bins, then interval m + 1's, in ascending bin order -- the order
// and the weights of the mel_filter_bank kernel.
template <int NFFT, int TFX>
__device__ __forceinline__ void build_fused_mel(const FrontendArgs& a, unsigned char* smem,
                                                const FusedLayout<NFFT, TFX>& lay)
{
    using S = StftShape<NFFT, kFusedThreads, TFX>;
    constexpr int TF = S::TF, BINS = S::BINS;
    constexpr int kGroups = 2 * kFusedThreads / TF;   // mel thread groups: TF / 2 frame pairs each
    const int nmel = a.mel.numFilter;
    float* s_out = reinterpret_cast<float*>(smem + lay.work + S::fft_bytes);
    float2* melW = reinterpret_cast<float2*>(smem + lay.melW);   // bin k: (weight into filter i, into filter i - 1)
    int2* melIv = reinterpret_cast<int2*>(smem + lay.melIv);     // interval i: bins [x, y)
    int* melGrp = reinterpret_cast<int*>(smem + lay.melGrp);     // thread group g: filters [g], [g + 1])
    unsigned char* t = smem + lay.work;
    MelTableView v;
    v.first = reinterpret_cast<int*>(t);
    v.last = v.first + (nmel + 2);
    v.norm = reinterpret_cast<float*>(v.last + (nmel + 2));
    size_t o = (size_t(reinterpret_cast<unsigned char*>(v.norm + nmel) - t) + 7) & ~size_t(7);
    v.f0 = reinterpret_cast<double*>(t + o);
    v.f1 = v.f0 + (nmel + 1);
    v.weightsDown = reinterpret_cast<float*>(v.f1 + (nmel + 1));
    v.range = reinterpret_cast<int*>(v.weightsDown + BINS);
    build_mel_tables(v, a.mel, NFFT);   // ends with __syncthreads
    for (int i = threadIdx.x; i <= nmel; i += kFusedThreads)
    {
        const int k0 = v.first[i], k1 = v.last[i];
        melIv[i] = k1 > k0 ? make_int2(k0, k1) : make_int2(0, 0);
        for (int k = k0; k < k1; ++k)
        {
            const float wd = v.weightsDown[k];
            float rise = 0.f, fall = 0.f;
            if (i < nmel)
            {
                rise = __fsub_rn(1.0f, wd);
                if (a.mel.normalize) rise = __fmul_rn(rise, v.norm[i]);
            }
            if (i > 0) fall = a.mel.normalize ? __fmul_rn(wd, v.norm[i - 1]) : wd;
            melW[k] = make_float2(rise, fall);
        }
    }
    // group g emits filters [melGrp[g], melGrp[g + 1]) and sweeps their intervals; the groups'
    // shares of (bins + 2) per interval are balanced.  cum[i] = cost of intervals 0..i (an
    // inclusive scan by warp 0, in the power tile's space, which is free until the first FFT);
    // boundary g is 1 + the first filter m whose intervals 0..m+1 reach g / kGroups of the total.
    int* cum = reinterpret_cast<int*>(s_out);
    for (int i = threadIdx.x; i <= nmel; i += kFusedThreads)
        cum[i] = (v.last[i] > v.first[i] ? v.last[i] - v.first[i] : 0) + 2;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        const int lane = threadIdx.x, chunk = (nmel + 1 + 31) / 32;
        const int i0 = min(lane * chunk, nmel + 1), i1 = min(i0 + chunk, nmel + 1);
        int sum = 0;
        for (int i = i0; i < i1; ++i) sum += cum[i];
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        int run = incl - sum;
        for (int i = i0; i < i1; ++i)
        {
            run += cum[i];
            cum[i] = run;
        }
    }
    __syncthreads();
    const int totalCost = cum[nmel];
    for (int grp = threadIdx.x; grp <= kGroups; grp += kFusedThreads)
    {
        int lo = 0, hi = nmel;   // first m in [0, nmel) with cum[m + 1] * kGroups >= grp * total, else nmel
        if (grp == 0) hi = -1;
        else
            while (lo < hi)
            {
                const int mid = (lo + hi) >> 1;
                if (cum[mid + 1] * kGroups >= grp * totalCost) hi = mid;
                else lo = mid + 1;
            }
        melGrp[grp] = grp == 0 ? 0 : grp == kGroups ? nmel : min(lo + 1, nmel);
    }
    __syncthreads();
}

// Builds the fused kernel's mel tables once, with one CTA, into `out`: the bytes [melW, total) of its
// shared-memory layout (melW, melIv, melGrp), which every launch with the same mel parameters and tile
// copies instead of building them in each CTA.
template <int NFFT, int TFX>
__global__ void __launch_bounds__(kFusedThreads) fused_mel_tables_kernel(FrontendArgs a, uint4* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const FusedLayout<NFFT, TFX> lay(a.mel.numFilter, a.W, a.hop);
    build_fused_mel<NFFT, TFX>(a, smem, lay);
    const uint4* src = reinterpret_cast<const uint4*>(smem + lay.melW);
    for (int i = threadIdx.x; i < int((lay.total - lay.melW) / 16); i += kFusedThreads) *RPPB_WR(out + i) = src[i];
}

// The fused kernels' mel tables (the bytes [melW, total) of FusedLayout<NFFT, TFX>), built once per
// handle, mel parameters and tile by a one-CTA kernel on the handle stream and cached; nullptr while
// the stream is being captured with parameters the handle has not cached (nothing is allocated during
// capture).  Launched before the prefix kernel: the fused kernels read the tables before their
// grid-dependency wait, which orders them only after the kernel just before them.
template <int NFFT, int TFX>
uint4* fused_mel_table_cache(Handle& h, const FrontendArgs& a)
{
    const FusedLayout<NFFT, TFX> lay(a.mel.numFilter, a.W, a.hop);
    auto bits = [](float v) {
        uint32_t u;
        std::memcpy(&u, &v, sizeof u);
        return std::to_string(u);
    };
    const std::string key = "fusedmel:" + std::to_string(NFFT) + ":" + std::to_string(TFX) + ":" +
                            std::to_string(a.mel.numFilter) + ":" + bits(a.mel.minFreq) + ":" + bits(a.mel.maxFreq) +
                            ":" + bits(a.mel.sampleRate) + ":" + std::to_string(a.mel.htk) + ":" +
                            std::to_string(int(a.mel.normalize));
    bool fresh = false;
    uint4* melTables = static_cast<uint4*>(h.device_table(key, lay.total - lay.melW, &fresh));
    if (fresh)
    {
        const void* tk = reinterpret_cast<const void*>(fused_mel_tables_kernel<NFFT, TFX>);
        persistent_grid(h, tk, kFusedThreads, lay.total);   // sets the kernel's shared-memory opt-in
        fused_mel_tables_kernel<NFFT, TFX><<<1, kFusedThreads, lay.total, h.stream()>>>(a, melTables);
        count_launch();
        check_cuda(cudaGetLastError(), "fused_mel_tables_kernel");
    }
    return melTables;
}

// Bytes of the mel table block for numFilter filters at nfft 512 with 16-frame tiles (the tensor-core
// engine builds it into the call's scratch when it cannot use the cache).
inline size_t fused_mel_table_bytes_512(int numFilter, int W, int hop)
{
    const FusedLayout<512, 16> lay(numFilter, W, hop);
    return lay.total - lay.melW;
}

}  // namespace
}  // namespace rppb
