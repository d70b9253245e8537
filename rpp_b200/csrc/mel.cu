// mel_filter_bank over NFT spectra.
//
// Reference: src/modules/tensor/cpu/kernel/mel_filter_bank.cpp:40-193 and the scales of
// api/rppdefs.h:795-851.  Per sample, nfft = (bins - 1) * 2 and hzStep = sampleRate / nfft.
// numFilter + 1 intervals are laid out evenly in mel between hz_to_mel(minFreq) and
// hz_to_mel(maxFreq) (mel edges accumulate an FP64 step; the scale functions are float
// functions); bin k belongs to the first interval whose upper edge f1 exceeds k * hzStep and
// has weightsDown = (f1 - f) / (f1 - f0) (rounded to float); with normalize, filter m is
// scaled by 2 / (f_{m+2} - f_m).  Filter m sums the bins of interval m with weight
// (1 - weightsDown) and the bins of interval m+1 with weight weightsDown, in ascending bin
// order, in float, starting from 0 — exactly the reference's accumulation order, so with the
// same tables the outputs are bit-identical.  Columns [frames, min(frames + 8, hStride)) of
// each filter row are zeroed, as the reference does.
//
// The tables are built on the GPU by the CTA that needs them (rebuilt only when the sample's
// bin count differs from the last one it built): the float scale functions use logf/expf
// evaluated as correctly rounded double log/exp, the edges and weights are FP64 like the
// reference's.  Work list: (sample, 64-frame tile) units; thread (group g, frame t) computes
// filters g, g+4, ... for frame t, reading the spectrum column through L1 (each bin feeds two
// filters), and the warp's 32 consecutive frames make every load and store one 128-byte line.
#include <cfloat>

#include "common.cuh"
#include "mel_tables.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kTile = 64;            // frames per unit
constexpr int kGroups = kThreads / kTile;
constexpr int kMaxBins = 4097;       // nfft up to 8192
constexpr int kMaxFilters = 1024;

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

struct MelSmem
{
    int range[3];
    int first[kMaxFilters + 2];
    int last[kMaxFilters + 2];
    float norm[kMaxFilters];
    double f1[kMaxFilters + 1];
    double f0[kMaxFilters + 1];
    float weightsDown[kMaxBins];
};

__global__ void __launch_bounds__(kThreads) mel_kernel(MelArgs a, float maxFreq, const long long* __restrict__ prefix)
{
    extern __shared__ __align__(16) unsigned char smem[];
    MelSmem& T = *reinterpret_cast<MelSmem*>(smem);
    const MelTableView view{T.first, T.last, T.norm, T.f0, T.f1, T.weightsDown, T.range};
    const MelParams mp{a.minFreq, maxFreq, a.sampleRate, a.htk, a.numFilter, a.normalize};
    if (threadIdx.x == 0) T.range[2] = -1;
    __syncthreads();
    const long long total = prefix[a.n];
    const int t = threadIdx.x % kTile;
    const int g = threadIdx.x / kTile;
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int tile = int(w - prefix[b]);
        const int bins = a.dims[2 * b];
        const int frames = max(a.dims[2 * b + 1], 0);
        const int nfft = (bins - 1) * 2;
        const bool ok = nfft >= 2 && nfft / 2 + 1 <= kMaxBins && uint32_t(bins) <= a.srcRows;
        const int held = T.range[2];
        __syncthreads();   // every thread has read the key before a rebuild may change it
        if (ok && held != nfft) build_mel_tables(view, mp, nfft);
        const int col = tile * kTile + t;
        const int zc = int(min((long long)frames + 8, (long long)a.dstHStride));
        float* y = a.dst + size_t(b) * a.dstNStride;
        if (col < zc)
        {
            const float* x = a.src + size_t(b) * a.srcNStride + col;
            for (int m = g; m < a.numFilter; m += kGroups)
            {
                float acc = 0.0f;
                if (ok && col < frames)
                {
                    // bins of interval m: weight (1 - weightsDown) * norm[m]
                    for (int k = T.first[m]; k < T.last[m]; ++k)
                    {
                        float wgt = __fsub_rn(1.0f, T.weightsDown[k]);
                        if (a.normalize) wgt = __fmul_rn(wgt, T.norm[m]);
                        acc = __fadd_rn(acc, __fmul_rn(__ldg(x + size_t(k) * a.srcHStride), wgt));
                    }
                    // bins of interval m + 1: weight weightsDown * norm[m]
                    for (int k = T.first[m + 1]; k < T.last[m + 1]; ++k)
                    {
                        float wgt = T.weightsDown[k];
                        if (a.normalize) wgt = __fmul_rn(wgt, T.norm[m]);
                        acc = __fadd_rn(acc, __fmul_rn(__ldg(x + size_t(k) * a.srcHStride), wgt));
                    }
                }
                y[size_t(m) * a.dstHStride + col] = acc;
            }
        }
        __syncthreads();   // the next unit may rebuild the tables
    }
}

}  // namespace

void launch_mel_filter_bank(Handle& h, void* scratch, const MelArgs& a)
{
    if (a.n <= 0) return;
    if (a.numFilter > kMaxFilters) fail(RPP_ERROR_INVALID_ARGUMENTS, "numFilter above 1024");
    long long* prefix = static_cast<long long*>(scratch);
    launch_ragged_prefix(MelCount{a.dims, a.dstHStride}, a.n, prefix, h.stream());
    const float maxFreq = (a.maxFreq == 0) ? a.sampleRate / 2 : a.maxFreq;
    const size_t smem = sizeof(MelSmem);
    int grid = persistent_grid(h, reinterpret_cast<const void*>(mel_kernel), kThreads, smem);
    mel_kernel<<<grid, kThreads, smem, h.stream()>>>(a, maxFreq, prefix);
    count_launch();
    check_cuda(cudaGetLastError(), "mel_kernel");
}

}  // namespace rppb
