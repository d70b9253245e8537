// mel_filter_bank over NFT spectra.
//
// Reference: src/modules/tensor/cpu/kernel/mel_filter_bank.cpp:40-193 and the scales of
// api/rppdefs.h:795-851 (table construction: mel_tables.cuh).  Filter m sums the bins of interval m
// with weight (1 - weightsDown) * norm[m] and the bins of interval m+1 with weight
// weightsDown * norm[m], in ascending bin order, in float, starting from 0 — the reference's
// accumulation order, so with the same tables the outputs are bit-identical.  Columns
// [frames, min(frames + 8, hStride)) of each filter row are zeroed, as the reference does.
//
// Work list: (sample, 32-frame tile) units.  A CTA stages the tile's spectrum rows
// [binStart, binEnd) x 32 frames in shared memory (one coalesced 128-byte row segment per bin), then
// thread (group g, frame pair t) sweeps the bins of group g's contiguous filter range once for two
// frames (each power pair read once, feeding its two filters) and a warp stores 32 consecutive
// frames of two filter rows.  Tables are built by the CTA (rebuilt only when
// the sample's bin count changes), sized for this call's numFilter and bins.
#include <cfloat>

#include "common.cuh"
#include "mel_tables.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kTile = 32;            // frames per unit
constexpr int kLd = kTile + 2;       // spectrum tile leading dimension: even, so frame pairs load as float2
constexpr int kPairs = kTile / 2;    // frame pairs per tile
constexpr int kGroups = kThreads / kPairs;   // filter groups

struct MelCount
{
    const int* dims;
    uint32_t dstHStride;
    __device__ long long operator()(int b) const
    {
        long long frames = max(*RPPB_RD(dims + (2 * b + 1)), 0);
        long long cols = min(frames + 8, (long long)dstHStride);
        return (cols + kTile - 1) / kTile;
    }
};

// Shared memory plan for numFilter filters and at most maxBins bins (host and device agree).
// weights: bin k -> (weight into filter i, weight into filter i - 1) for k in interval i;
// intervals: interval i -> its bins [x, y); groups: thread group g emits filters
// [groups[g], groups[g + 1]).
struct MelLayout
{
    size_t range, first, last, norm, f0, f1, wd, weights, intervals, groups, cum, spec, total;
    __host__ __device__ MelLayout(int numFilter, int maxBins)
    {
        range = 0;
        first = 16;
        last = first + size_t(numFilter + 2) * 4;
        norm = last + size_t(numFilter + 2) * 4;
        f0 = (norm + size_t(numFilter) * 4 + 7) & ~size_t(7);
        f1 = f0 + size_t(numFilter + 1) * 8;
        wd = f1 + size_t(numFilter + 1) * 8;
        weights = (wd + size_t(maxBins) * 4 + 15) & ~size_t(15);
        intervals = (weights + size_t(maxBins) * 8 + 15) & ~size_t(15);
        groups = (intervals + size_t(numFilter + 1) * 8 + 15) & ~size_t(15);
        cum = (groups + size_t(kGroups + 1) * 4 + 15) & ~size_t(15);
        spec = (cum + size_t(numFilter + 1) * 4 + 15) & ~size_t(15);
        total = spec + size_t(maxBins) * kLd * 4;
    }
};

// Bin-major form of the tables: bin k of interval i (between mel points i and i + 1) weighs
// (1 - weightsDown) * norm[i] into filter i and weightsDown * norm[i - 1] into filter i - 1 (norm
// only when normalizing), so filter m sums interval m's bins, then interval m + 1's, in ascending
// bin order -- the reference's accumulation.  The filter ranges of the kGroups thread groups are
// balanced by (bins + 2) per interval: cum[i] = cost of intervals 0..i by a warp scan, boundary g
// at 1 + the first filter m whose intervals 0..m+1
// reach g / kGroups of the total (cum: numFilter + 1 ints of scratch).  Ends with __syncthreads.
__device__ void build_sweep(const MelTableView& T, int numFilter, bool normalize, float2* weights, int2* intervals,
                            int* groups, int* cum)
{
    for (int i = threadIdx.x; i <= numFilter; i += blockDim.x)
    {
        const int k0 = T.first[i], k1 = T.last[i];
        intervals[i] = k1 > k0 ? make_int2(k0, k1) : make_int2(0, 0);
        for (int k = k0; k < k1; ++k)
        {
            const float wd = T.weightsDown[k];
            float rise = 0.f, fall = 0.f;
            if (i < numFilter)
            {
                rise = __fsub_rn(1.0f, wd);
                if (normalize) rise = __fmul_rn(rise, T.norm[i]);
            }
            if (i > 0) fall = normalize ? __fmul_rn(wd, T.norm[i - 1]) : wd;
            weights[k] = make_float2(rise, fall);
        }
        cum[i] = (k1 > k0 ? k1 - k0 : 0) + 2;
    }
    __syncthreads();
    if (threadIdx.x < 32)
    {
        const int lane = threadIdx.x, chunk = (numFilter + 1 + 31) / 32;
        const int i0 = min(lane * chunk, numFilter + 1), i1 = min(i0 + chunk, numFilter + 1);
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
    const int total = cum[numFilter];
    for (int g = threadIdx.x; g <= kGroups; g += blockDim.x)
    {
        int lo = 0, hi = numFilter;
        if (g > 0)
            while (lo < hi)
            {
                const int mid = (lo + hi) >> 1;
                if (cum[mid + 1] * kGroups >= g * total) hi = mid;
                else lo = mid + 1;
            }
        groups[g] = g == 0 ? 0 : g == kGroups ? numFilter : min(lo + 1, numFilter);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) mel_kernel(MelArgs a, float maxFreq, int maxBins,
                                                       const long long* __restrict__ prefix)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const MelLayout lay(a.numFilter, maxBins);
    int* range = reinterpret_cast<int*>(smem + lay.range);
    const MelTableView T{reinterpret_cast<int*>(smem + lay.first), reinterpret_cast<int*>(smem + lay.last),
                         reinterpret_cast<float*>(smem + lay.norm), reinterpret_cast<double*>(smem + lay.f0),
                         reinterpret_cast<double*>(smem + lay.f1), reinterpret_cast<float*>(smem + lay.wd), range};
    float* s_spec = reinterpret_cast<float*>(smem + lay.spec);
    float2* weights = reinterpret_cast<float2*>(smem + lay.weights);
    int2* intervals = reinterpret_cast<int2*>(smem + lay.intervals);
    int* groups = reinterpret_cast<int*>(smem + lay.groups);
    const MelParams mp{a.minFreq, maxFreq, a.sampleRate, a.htk, a.numFilter, a.normalize};
    if (threadIdx.x == 0) range[2] = -1;
    __syncthreads();
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, a.n, s_prefix);
    const long long total = prefix[a.n];
    const int t = 2 * (threadIdx.x % kPairs);   // first of this thread's two frames
    const int g = threadIdx.x / kPairs;
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int tile = int(w - prefix[b]);
        const int bins = *RPPB_RD(a.dims + 2 * b);
        const int frames = min(max(*RPPB_RD(a.dims + (2 * b + 1)), 0), int(min(a.srcHStride, a.dstHStride)));
        const int nfft = (bins - 1) * 2;
        const bool ok = nfft >= 2 && bins <= maxBins && uint32_t(bins) <= a.srcRows;
        const int held = range[2];
        __syncthreads();   // every thread has read the key before a rebuild may change it
        if (ok && held != nfft)
        {
            build_mel_tables(T, mp, nfft);
            build_sweep(T, a.numFilter, a.normalize, weights, intervals, groups, reinterpret_cast<int*>(smem + lay.cum));
        }
        const int t0 = tile * kTile;
        const int zc = int(min((long long)frames + 8, (long long)a.dstHStride));
        const int tv = min(kTile, frames - t0);   // valid frames of this tile (may be <= 0)
        const int k0 = range[0], k1 = range[1];
        if (ok && tv > 0)
        {
            // stage spectrum rows [k0, k1) x frames [t0, t0 + tv) (zeros past tv): lane = frame
            // column, warp w takes rows w, w + kWarps, ...; both pointers advance by a fixed row step
            // and kBatch loads per thread are in flight before their stores
            static_assert(kTile == 32, "one warp per staged row");
            constexpr int kWarps = kThreads / 32, kBatch = 8;
            const int lane = threadIdx.x & 31, rows = k1 - k0;
            const bool colOk = lane < tv;
            const size_t rowStep = size_t(kWarps) * a.srcHStride;
            int r = threadIdx.x >> 5;
            const float* xs = a.src + size_t(b) * a.srcNStride + t0 + size_t(k0 + r) * a.srcHStride + lane;
            float* ss = s_spec + r * kLd + lane;
            for (; r + (kBatch - 1) * kWarps < rows; r += kBatch * kWarps)
            {
                float v[kBatch];
#pragma unroll
                for (int j = 0; j < kBatch; ++j, xs += rowStep) v[j] = colOk ? __ldg(RPPB_RD(xs)) : 0.0f;
#pragma unroll
                for (int j = 0; j < kBatch; ++j, ss += kWarps * kLd) *ss = v[j];
            }
            for (; r < rows; r += kWarps, xs += rowStep, ss += kWarps * kLd) *ss = colOk ? __ldg(RPPB_RD(xs)) : 0.0f;
        }
        __syncthreads();
        // one sweep over the group's intervals for frames t0 + t and t0 + t + 1; each power pair is
        // read once.  Columns at or past `frames` (below zc) get zeros.
        const int col = t0 + t;
        if (col < zc)
        {
            const bool live0 = ok && col < frames, live1 = ok && col + 1 < frames, has1 = col + 1 < zc;
            const int m0 = ok ? groups[g] : 0, m1 = ok ? groups[g + 1] : 0;
            float* yp = a.dst + size_t(b) * a.dstNStride + size_t(m0) * a.dstHStride + col;
            float2 fall = make_float2(0.f, 0.f);   // filter i - 1: rising sum, then falling terms
            for (int i = m0; i <= m1 && ok; ++i)
            {
                const int2 iv = intervals[i];
                const float* sp = s_spec + (iv.x - k0) * kLd + t;
                float2 rise = make_float2(0.f, 0.f);   // filter i
#pragma unroll 1
                for (int k = iv.x; k < iv.y; ++k, sp += kLd)
                {
                    const float2 pw = *reinterpret_cast<const float2*>(sp);
                    const float2 w = weights[k];
                    fall.x = __fadd_rn(fall.x, __fmul_rn(pw.x, w.y));
                    fall.y = __fadd_rn(fall.y, __fmul_rn(pw.y, w.y));
                    rise.x = __fadd_rn(rise.x, __fmul_rn(pw.x, w.x));
                    rise.y = __fadd_rn(rise.y, __fmul_rn(pw.y, w.x));
                }
                if (i > m0)
                {
                    *RPPB_WR(yp) = live0 ? fall.x : 0.0f;
                    if (has1) *RPPB_WR(yp + 1) = live1 ? fall.y : 0.0f;
                    yp += a.dstHStride;
                }
                fall = rise;
            }
            if (!ok)   // no tables for this sample: zeros, as the reference leaves its output
                for (int m = g; m < a.numFilter; m += kGroups)
                {
                    float* z = a.dst + size_t(b) * a.dstNStride + size_t(m) * a.dstHStride + col;
                    *RPPB_WR(z) = 0.0f;
                    if (has1) *RPPB_WR(z + 1) = 0.0f;
                }
        }
        __syncthreads();   // the next unit restages the tile and may rebuild the tables
    }
}

}  // namespace

void launch_mel_filter_bank(Handle& h, void* scratch, const MelArgs& a)
{
    if (a.n <= 0) return;
    const int maxBins = int(a.srcRows);
    const size_t smem = MelLayout(a.numFilter, maxBins).total;
    if (smem > 227 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "too many bins or filters for the mel tile");
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(MelCount{a.dims, a.dstHStride}, a.n, prefix, h.stream());
    const float maxFreq = (a.maxFreq == 0) ? a.sampleRate / 2 : a.maxFreq;
    int grid = persistent_grid(h, reinterpret_cast<const void*>(mel_kernel), kThreads, smem);
    mel_kernel<<<grid, kThreads, smem, h.stream()>>>(a, maxFreq, maxBins, prefix);
    count_launch();
    check_cuda(cudaGetLastError(), "mel_kernel");
}

}  // namespace rppb
