// Mel filter placement built on the GPU (shared by the plain mel_filter_bank kernel and the
// fused front end).
//
// Reference: src/modules/tensor/cpu/kernel/mel_filter_bank.cpp:55-112 and the scales of
// api/rppdefs.h:795-851.  numFilter + 1 intervals evenly spaced in mel between
// hz_to_mel(minFreq) and hz_to_mel(maxFreq); the mel edges accumulate an FP64 step in order, the
// scale functions are float functions (logf/expf evaluated as correctly rounded double log/exp),
// and bin k goes to the first interval whose upper edge f1 exceeds k * sampleRate / nfft, with
// weightsDown = (f1 - f) / (f1 - f0) rounded to float and, with normalize, filter m scaled by
// 2 / (f_{m+2} - f_m).
#pragma once

#include <climits>

#include "common.cuh"
#include "ops.hpp"

namespace rppb {

// Where the tables live (shared memory chosen by the caller).
struct MelTableView
{
    int* first;          // [numFilter + 2] first bin of interval i (INT_MAX when empty)
    int* last;           // [numFilter + 2] last bin + 1 (-1 when empty)
    float* norm;         // [numFilter]
    double* f0;          // [numFilter + 1]
    double* f1;          // [numFilter + 1]
    float* weightsDown;  // [nfft/2 + 1]
    int* range;          // [3]: binStart, binEnd, nfft of the tables held
};

static __device__ __forceinline__ float logf_cr(float x) { return __double2float_rn(log(double(x))); }
static __device__ __forceinline__ float expf_cr(float x) { return __double2float_rn(exp(double(x))); }

// Float scale functions of api/rppdefs.h:806-851, operation by operation.
static __device__ float hz_to_mel(int htk, float hz)
{
    if (htk) return __fmul_rn(1127.0f, logf_cr(__fadd_rn(1.0f, __fdiv_rn(hz, 700.0f))));
    const float fsp = 66.666667f, minLogHz = 1000.0f;
    const float minLogMel = __fdiv_rn(__fsub_rn(minLogHz, 0.0f), fsp);
    const float stepLog = 0.068751777f;
    const float invMinLogHz = 0.001f, invStepLog = __fdiv_rn(1.0f, stepLog), invFsp = __fdiv_rn(1.0f, fsp);
    if (hz >= minLogHz) return __fadd_rn(minLogMel, __fmul_rn(logf_cr(__fmul_rn(hz, invMinLogHz)), invStepLog));
    return __fmul_rn(__fsub_rn(hz, 0.0f), invFsp);
}

static __device__ float mel_to_hz(int htk, float mel)
{
    if (htk) return __fmul_rn(700.0f, __fsub_rn(expf_cr(__fdiv_rn(mel, 1127.0f)), 1.0f));
    const float fsp = 66.666667f, minLogHz = 1000.0f;
    const float minLogMel = __fdiv_rn(__fsub_rn(minLogHz, 0.0f), fsp);
    const float stepLog = 0.068751777f;
    if (mel >= minLogMel) return __fmul_rn(minLogHz, expf_cr(__fmul_rn(stepLog, __fsub_rn(mel, minLogMel))));
    return __fadd_rn(0.0f, __fmul_rn(mel, fsp));
}

// Builds the tables for `nfft` with the whole CTA.
static __device__ void build_mel_tables(const MelTableView& T, const MelParams& a, int nfft)
{
    const int numFilter = a.numFilter;
    const int numBins = nfft / 2 + 1;
    const double melLow = hz_to_mel(a.htk, a.minFreq), melHigh = hz_to_mel(a.htk, a.maxFreq);
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
        T.range[0] = int(ceil(__dmul_rn(double(a.minFreq), invHzStep)));
        T.range[1] = min(int(ceil(__dmul_rn(double(a.maxFreq), invHzStep))), numBins);
        T.range[2] = nfft;
    }
    for (int i = threadIdx.x; i < numFilter + 2; i += blockDim.x)
    {
        T.first[i] = INT_MAX;
        T.last[i] = -1;
    }
    __syncthreads();
    // bin k -> first interval with fIter < f1 (the reference's sequential sweep, :94-110)
    for (int k = T.range[0] + threadIdx.x; k < T.range[1]; k += blockDim.x)
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

}  // namespace rppb
