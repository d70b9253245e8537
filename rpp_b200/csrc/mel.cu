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
// thread (group g, frame t) computes filters g, g+8, ... for frame t from shared memory and a warp
// stores 32 consecutive frames of one filter row.  Tables are built by the CTA (rebuilt only when
// the sample's bin count changes), sized for this call's numFilter and bins.
#include <cfloat>

#include "common.cuh"
#include "mel_tables.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kTile = 32;            // frames per unit
constexpr int kLd = kTile + 1;       // spectrum tile leading dimension (conflict-free columns)
constexpr int kGroups = kThreads / kTile;

struct MelCount
{
    const int* dims;
    uint32_t dstHStride;
    __device__ long long operator()(int b) const
    {
        long long frames = max(dims[2 * b + 1], 0);
        long long cols = min(frames + 8, (long long)dstHStride);
        return (cols + kTile - 1) / kTile;
    }
};

// Shared memory plan for numFilter filters and at most maxBins bins (host and device agree).
// rowStart/entries: filter m's weights as (tile offset of the bin's row, weight) pairs
// entries[rowStart[m] .. rowStart[m + 1]), in the reference's accumulation order.
struct MelLayout
{
    size_t range, first, last, norm, f0, f1, wd, rowStart, entries, spec, total;
    __host__ __device__ MelLayout(int numFilter, int maxBins)
    {
        range = 0;
        first = 16;
        last = first + size_t(numFilter + 2) * 4;
        norm = last + size_t(numFilter + 2) * 4;
        f0 = (norm + size_t(numFilter) * 4 + 7) & ~size_t(7);
        f1 = f0 + size_t(numFilter + 1) * 8;
        wd = f1 + size_t(numFilter + 1) * 8;
        rowStart = (wd + size_t(maxBins) * 4 + 15) & ~size_t(15);
        entries = (rowStart + size_t(numFilter + 1) * 4 + 15) & ~size_t(15);
        spec = (entries + size_t(2 * maxBins + 2) * 8 + 15) & ~size_t(15);
        total = spec + size_t(maxBins) * kLd * 4;
    }
};

// Flattens the tables into (offset, weight) entries: bins of interval m with (1 - weightsDown) *
// norm[m], then bins of interval m + 1 with weightsDown * norm[m] (norm only when normalizing);
// offset = (bin - k0) * kLd in the staged tile.  Ends with __syncthreads.
__device__ void build_entries(const MelTableView& T, int numFilter, bool normalize, int* rowStart, int2* ent)
{
    const int k0 = T.range[0];
    if (threadIdx.x == 0)
    {
        int acc = 0;
        for (int m = 0; m < numFilter; ++m)
        {
            rowStart[m] = acc;
            acc += max(T.last[m] - T.first[m], 0) + max(T.last[m + 1] - T.first[m + 1], 0);
        }
        rowStart[numFilter] = acc;
    }
    __syncthreads();
    for (int m = threadIdx.x; m < numFilter; m += blockDim.x)
    {
        int e = rowStart[m];
        for (int k = T.first[m]; k < T.last[m]; ++k, ++e)
        {
            float w = __fsub_rn(1.0f, T.weightsDown[k]);
            if (normalize) w = __fmul_rn(w, T.norm[m]);
            ent[e] = make_int2((k - k0) * kLd, __float_as_int(w));
        }
        for (int k = T.first[m + 1]; k < T.last[m + 1]; ++k, ++e)
        {
            float w = T.weightsDown[k];
            if (normalize) w = __fmul_rn(w, T.norm[m]);
            ent[e] = make_int2((k - k0) * kLd, __float_as_int(w));
        }
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
    int* rowStart = reinterpret_cast<int*>(smem + lay.rowStart);
    int2* ent = reinterpret_cast<int2*>(smem + lay.entries);
    const MelParams mp{a.minFreq, maxFreq, a.sampleRate, a.htk, a.numFilter, a.normalize};
    if (threadIdx.x == 0) range[2] = -1;
    __syncthreads();
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, a.n, s_prefix);
    const long long total = prefix[a.n];
    const int t = threadIdx.x % kTile;
    const int g = threadIdx.x / kTile;
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int tile = int(w - prefix[b]);
        const int bins = a.dims[2 * b];
        const int frames = min(max(a.dims[2 * b + 1], 0), int(min(a.srcHStride, a.dstHStride)));
        const int nfft = (bins - 1) * 2;
        const bool ok = nfft >= 2 && bins <= maxBins && uint32_t(bins) <= a.srcRows;
        const int held = range[2];
        __syncthreads();   // every thread has read the key before a rebuild may change it
        if (ok && held != nfft)
        {
            build_mel_tables(T, mp, nfft);
            build_entries(T, a.numFilter, a.normalize, rowStart, ent);
        }
        const int t0 = tile * kTile;
        const int zc = int(min((long long)frames + 8, (long long)a.dstHStride));
        const int tv = min(kTile, frames - t0);   // valid frames of this tile (may be <= 0)
        const int k0 = range[0], k1 = range[1];
        if (ok && tv > 0)
        {
            // stage spectrum rows [k0, k1) x frames [t0, t0 + tv)
            const float* x = a.src + size_t(b) * a.srcNStride + t0;
            for (int idx = threadIdx.x; idx < (k1 - k0) * kTile; idx += kThreads)
            {
                const int r = idx / kTile, c = idx % kTile;
                if (c < tv) s_spec[r * kLd + c] = __ldg(x + size_t(k0 + r) * a.srcHStride + c);
            }
        }
        __syncthreads();
        const int col = t0 + t;
        if (col < zc)
        {
            const bool live = ok && col < frames;
            const float* sp = s_spec + t;
            float* yp = a.dst + size_t(b) * a.dstNStride + size_t(g) * a.dstHStride + col;
            const size_t ystep = size_t(kGroups) * a.dstHStride;
            for (int m = g; m < a.numFilter; m += kGroups, yp += ystep)
            {
                float acc = 0.0f;
                if (live)
                {
                    const int e1 = rowStart[m + 1];
#pragma unroll 4
                    for (int e = rowStart[m]; e < e1; ++e)
                    {
                        const int2 en = ent[e];
                        acc = __fadd_rn(acc, __fmul_rn(sp[en.x], __int_as_float(en.y)));
                    }
                }
                *yp = acc;
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
