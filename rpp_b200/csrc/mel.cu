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

__device__ __forceinline__ float logf_cr(float x) { return __double2float_rn(log(double(x))); }
__device__ __forceinline__ float expf_cr(float x) { return __double2float_rn(exp(double(x))); }

// Float scale functions of api/rppdefs.h:806-851, operation by operation.
__device__ float hz_to_mel(int htk, float hz)
{
    if (htk) return __fmul_rn(1127.0f, logf_cr(__fadd_rn(1.0f, __fdiv_rn(hz, 700.0f))));
    const float fsp = 66.666667f, minLogHz = 1000.0f;
    const float minLogMel = __fdiv_rn(__fsub_rn(minLogHz, 0.0f), fsp);
    const float stepLog = 0.068751777f;
    const float invMinLogHz = 0.001f, invStepLog = __fdiv_rn(1.0f, stepLog), invFsp = __fdiv_rn(1.0f, fsp);
    if (hz >= minLogHz) return __fadd_rn(minLogMel, __fmul_rn(logf_cr(__fmul_rn(hz, invMinLogHz)), invStepLog));
    return __fmul_rn(__fsub_rn(hz, 0.0f), invFsp);
}

__device__ float mel_to_hz(int htk, float mel)
{
    if (htk) return __fmul_rn(700.0f, __fsub_rn(expf_cr(__fdiv_rn(mel, 1127.0f)), 1.0f));
    const float fsp = 66.666667f, minLogHz = 1000.0f;
    const float minLogMel = __fdiv_rn(__fsub_rn(minLogHz, 0.0f), fsp);
    const float stepLog = 0.068751777f;
    if (mel >= minLogMel) return __fmul_rn(minLogHz, expf_cr(__fmul_rn(stepLog, __fsub_rn(mel, minLogMel))));
    return __fadd_rn(0.0f, __fmul_rn(mel, fsp));
}

struct MelTables
{
    int nfft;                 // key of the tables currently held
    int binStart, binEnd;
    int first[kMaxFilters + 2];   // first bin of interval i (binEnd when empty)
    int last[kMaxFilters + 2];    // last bin + 1
    float norm[kMaxFilters];
    double f1[kMaxFilters + 1];
    double f0[kMaxFilters + 1];
    float weightsDown[kMaxBins];
};

// Builds the tables for `nfft` with the whole CTA.
__device__ void build_tables(MelTables& T, const MelArgs& a, float maxFreq, int nfft)
{
    const int numFilter = a.numFilter;
    const int numBins = nfft / 2 + 1;
    const double melLow = hz_to_mel(a.htk, a.minFreq), melHigh = hz_to_mel(a.htk, maxFreq);
    const double melStep = __ddiv_rn(__dsub_rn(melHigh, melLow), double(numFilter + 1));
    const double hzStep = __ddiv_rn(double(a.sampleRate), double(nfft));
    const double invHzStep = __ddiv_rn(1.0, hzStep);
    // interval edges: mel1_i = melLow + melStep (+ melStep) * i, accumulated in order (:87-92)
    for (int i = threadIdx.x; i <= numFilter; i += blockDim.x)
    {
        double mel0 = melLow, mel1 = __dadd_rn(melLow, melStep);
        for (int k = 0; k < i; ++k)
        {
            mel0 = mel1;
            mel1 = __dadd_rn(mel1, melStep);
        }
        const double f0 = mel_to_hz(a.htk, __double2float_rn(mel0));
        const double f1 = mel_to_hz(a.htk, __double2float_rn(i == numFilter ? melHigh : mel1));
        T.f0[i] = f0;
        T.f1[i] = f1;
        if (i < numFilter)
        {
            float nf = 1.f;
            if (a.normalize)
            {
                const double f2 = mel_to_hz(a.htk, __double2float_rn(__dadd_rn(mel1, melStep)));
                nf = __double2float_rn(__ddiv_rn(2.0, __dsub_rn(f2, f0)));
            }
            T.norm[i] = nf;
        }
    }
    if (threadIdx.x == 0)
    {
        T.binStart = int(ceil(__dmul_rn(double(a.minFreq), invHzStep)));
        T.binEnd = min(int(ceil(__dmul_rn(double(maxFreq), invHzStep))), numBins);
        T.nfft = nfft;
    }
    for (int i = threadIdx.x; i < numFilter + 2; i += blockDim.x)
    {
        T.first[i] = INT_MAX;
        T.last[i] = -1;
    }
    __syncthreads();
    // bin k -> first interval with fIter < f1 (the reference's sequential sweep, :94-110)
    for (int k = T.binStart + threadIdx.x; k < T.binEnd; k += blockDim.x)
    {
        const double fIter = __dmul_rn(double(k), hzStep);
        int lo = 0, hi = numFilter + 1;   // search in [0, numFilter], numFilter+1 = none
        while (lo < hi)
        {
            int mid = (lo + hi) >> 1;
            if (fIter < T.f1[mid]) hi = mid;
            else lo = mid + 1;
        }
        if (lo <= numFilter)
        {
            const double slope = __ddiv_rn(1.0, __dsub_rn(T.f1[lo], T.f0[lo]));
            T.weightsDown[k] = __double2float_rn(__dmul_rn(__dsub_rn(T.f1[lo], fIter), slope));
            atomicMin(&T.first[lo], k);
            atomicMax(&T.last[lo], k + 1);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) mel_kernel(MelArgs a, float maxFreq, const long long* __restrict__ prefix)
{
    extern __shared__ __align__(16) unsigned char smem[];
    MelTables& T = *reinterpret_cast<MelTables*>(smem);
    if (threadIdx.x == 0) T.nfft = -1;
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
        const int held = T.nfft;
        __syncthreads();   // every thread has read the key before a rebuild may change it
        if (ok && held != nfft) build_tables(T, a, maxFreq, nfft);
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
    const size_t smem = sizeof(MelTables);
    check_cuda(cudaFuncSetAttribute(mel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "smem attr");
    int grid = persistent_grid(h, reinterpret_cast<const void*>(mel_kernel), kThreads, smem);
    mel_kernel<<<grid, kThreads, smem, h.stream()>>>(a, maxFreq, prefix);
    check_cuda(cudaGetLastError(), "mel_kernel");
}

}  // namespace rppb
