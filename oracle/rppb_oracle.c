/*
 * ORACLE — test infrastructure only.  This file is a CPU restatement of the reference's host
 * audio path (ROCm/rpp src/modules/tensor/cpu/kernel/*.cpp), used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.  It is never
 * linked into the product library and never runs on the product path.
 *
 * Two kinds of functions:
 *  - float restatements that repeat the reference's float operations in the reference's order
 *    (compiled with -ffp-contract=off, no fast-math, like the reference's -mno-fma build), so
 *    they agree bit for bit with the reference where the reference is deterministic float
 *    arithmetic (pre-emphasis, down-mixing, resampling, mel filter bank, decibels, NSR);
 *  - FP64 forms (spectrogram, mel, decibels, the whole front-end chain) that evaluate the same
 *    definitions in double precision: the "FP64 oracle" against which errors are reported.
 *    The reference's FP32 spectrogram runs ffts (a prebuilt third-party binary), whose
 *    operation order is not restated; its FP32 results are checked against the reference
 *    library itself and the shipped goldens, within a per-frame relative tolerance.
 *
 * Parity is pinned by tests/test_oracle_golden.py: against the shipped golden outputs
 * (utilities/test_suite/REFERENCE_OUTPUTS_AUDIO/*.bin, captured under tests/golden/) and
 * against the reference host library built by oracle/build_ref.sh.
 *
 * Strides are in elements, as in RpptDesc.strides.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- pre-emphasis
 * cpu/kernel/pre_emphasis_filter.cpp:39-71: y[0] = x[0] - c*border, y[i] = x[i] - c*x[i-1]. */
EXPORT void oracle_pre_emphasis(const float *src, long srcStride, float *dst, long dstStride, int n,
                                const int *len, const float *coeff, int border)
{
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        const float *x = src + (long)b * srcStride;
        float *y = dst + (long)b * dstStride;
        float c = coeff[b];
        float bv = (border == 1) ? x[0] : (border == 2) ? x[1] : 0.f;   /* CLAMP=1, REFLECT=2 */
        y[0] = x[0] - c * bv;
        for (int i = 1; i < len[b]; i++)
            y[i] = x[i] - c * x[i - 1];
    }
}

/* ---------------------------------------------------------------- down-mixing
 * cpu/kernel/down_mixing.cpp:42-117.  Lane sums and horizontal sums in the SSE/AVX order of
 * rpp_hsum_ps (src/include/common/cpu/rpp_cpu_simd_math.hpp:846-867). */
static float hsum4(const float p[4]) { return (p[0] + p[1]) + (p[2] + p[3]); }
static float hsum8(const float p[8]) { return ((p[0] + p[4]) + (p[2] + p[6])) + ((p[1] + p[5]) + (p[3] + p[7])); }

EXPORT void oracle_down_mixing(const float *src, long srcStride, float *dst, long dstStride, int n,
                               const int *dims, int normalize)
{
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        const float *x = src + (long)b * srcStride;
        float *y = dst + (long)b * dstStride;
        int samples = dims[2 * b], ch = dims[2 * b + 1];
        if (ch == 1)
        {
            memcpy(y, x, (size_t)samples * sizeof(float));
            continue;
        }
        float w[64];
        for (int c = 0; c < ch; c++) w[c] = 1.f / ch;
        if (normalize)
        {
            float sum = 0.0f;
            for (int c = 0; c < ch; c++) sum += w[c];
            float inv = (float)(1.0 / sum);
            for (int c = 0; c < ch; c++) w[c] *= inv;
        }
        int lanes = ch > 7 ? 8 : 4;
        int aligned = (ch / lanes) * lanes;
        for (long t = 0; t < samples; t++)
        {
            const float *xs = x + t * ch;
            float p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int g = 0; g < aligned; g += lanes)
                for (int l = 0; l < lanes; l++) p[l] = p[l] + xs[g + l] * w[g + l];
            float acc = (lanes == 8) ? hsum8(p) : hsum4(p);
            for (int c = aligned; c < ch; c++) acc += xs[c] * w[c];
            y[t] = acc;
        }
    }
}

/* ---------------------------------------------------------------- resample
 * cpu/kernel/resample.cpp:46-141 with the window of api/rppdefs.h:751-790: LUT interpolation,
 * 256-output blocks with an FP64 block origin and an FP32 running phase, 4-lane partial sums
 * for mono input, per-channel sequential sums for multi-channel input. */
typedef struct
{
    const float *lut;
    int lutSize;
    float scale, center;
    int lobes;
} oracle_window;

static float win_scalar(const oracle_window *w, float x)        /* rppdefs.h:760-769 */
{
    float locRaw = x * w->scale + w->center;
    int locFloor = (int)floorf(locRaw);
    float weight = locRaw - locFloor;
    if (locFloor > w->lutSize - 2) locFloor = w->lutSize - 2;
    if (locFloor < 0) locFloor = 0;
    float cur = w->lut[locFloor], nxt = w->lut[locFloor + 1];
    return cur + weight * (nxt - cur);
}

static float win_lane(const oracle_window *w, float x)          /* rppdefs.h:771-782 (truncating) */
{
    float locRaw = x * w->scale + w->center;
    int idx = (int)locRaw;
    float weight = locRaw - (float)idx;
    float cur = w->lut[idx], nxt = w->lut[idx + 1];
    return cur + weight * (nxt - cur);
}

EXPORT void oracle_resample(const float *src, long srcStride, float *dst, long dstStride, int n,
                            const float *inRate, const float *outRate, const int *dims,
                            const float *lut, int lutSize, float wscale, float wcenter, int lobes)
{
    oracle_window W = {lut, lutSize, wscale, wcenter, lobes};
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        const float *x = src + (long)b * srcStride;
        float *y = dst + (long)b * dstStride;
        float ir = inRate[b], orate = outRate[b];
        int len = dims[2 * b], ch = dims[2 * b + 1];
        if (orate == ir)
        {
            memcpy(y, x, (size_t)len * ch * sizeof(float));
            continue;
        }
        int outEnd = (int)ceilf((float)len * orate / ir);
        double scale = (double)ir / orate;
        float fscale = (float)scale;
        float tmp[64];
        for (int outBlock = 0; outBlock < outEnd; outBlock += 256)
        {
            int blockEnd = outBlock + 256 < outEnd ? outBlock + 256 : outEnd;
            double inBlockRaw = outBlock * scale;
            int inBlockRounded = (int)inBlockRaw;
            float inPos = (float)(inBlockRaw - inBlockRounded);
            const float *in = x + (long)inBlockRounded * ch;
            for (int outPos = outBlock; outPos < blockEnd; outPos++, inPos += fscale)
            {
                int xc = (int)ceilf(inPos);
                int loc0 = xc - lobes, loc1 = xc + lobes;
                if (loc0 + inBlockRounded < 0) loc0 = -inBlockRounded;
                if (loc1 + inBlockRounded > len) loc1 = len - inBlockRounded;
                if (ch == 1)
                {
                    int l = loc0;
                    float locBegin = l - inPos;
                    float lane[4] = {locBegin + 0.f, locBegin + 1.f, locBegin + 2.f, locBegin + 3.f};
                    float acc4[4] = {0, 0, 0, 0};
                    for (; l + 3 < loc1; l += 4)
                        for (int j = 0; j < 4; j++)
                        {
                            acc4[j] = acc4[j] + in[l + j] * win_lane(&W, lane[j]);
                            lane[j] = lane[j] + 4.f;
                        }
                    float accum = (acc4[0] + acc4[2]) + (acc4[1] + acc4[3]);
                    float xx = l - inPos;
                    for (; l < loc1; l++, xx++)
                        accum += in[l] * win_scalar(&W, xx);
                    y[outPos] = accum;
                }
                else
                {
                    for (int c = 0; c < ch; c++) tmp[c] = 0.f;
                    float xx = loc0 - inPos;
                    for (int l = loc0; l < loc1; l++, xx++)
                    {
                        float wv = win_scalar(&W, xx);
                        for (int c = 0; c < ch; c++) tmp[c] += in[(long)l * ch + c] * wv;
                    }
                    for (int c = 0; c < ch; c++) y[(long)outPos * ch + c] = tmp[c];
                }
            }
        }
    }
}

/* ---------------------------------------------------------------- spectrogram (FP64)
 * cpu/kernel/spectrogram.cpp:36-69 (Hann with the t+0.5 phase, frame count, reflect rule) and
 * :116-242 (frames, window centred in the nfft buffer, power 2 -> re^2+im^2, else |X|),
 * evaluated in double with an exact-twiddle FFT (radix-2 for powers of two, direct DFT
 * otherwise). */
static int reflect_idx(int loc, int minLoc, int maxLoc)          /* spectrogram.cpp:55-69 */
{
    if (maxLoc - minLoc < 2) return maxLoc - 1;
    for (;;)
    {
        if (loc < minLoc) loc = 2 * minLoc - loc;
        else if (loc >= maxLoc) loc = 2 * maxLoc - 2 - loc;
        else break;
    }
    return loc;
}

EXPORT int oracle_num_windows(int len, int windowLength, int windowStep, int center)   /* :47-52 */
{
    if (!center) len -= windowLength;
    return len / windowStep + 1;
}

static void fft_d(double *re, double *im, int N)    /* in-place, forward, natural order */
{
    for (int i = 1, j = 0; i < N; i++)
    {
        int bit = N >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j)
        {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int len = 2; len <= N; len <<= 1)
    {
        int half = len >> 1;
        for (int k = 0; k < half; k++)
        {
            double ang = -2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (int i = 0; i < N; i += len)
            {
                double ur = re[i + k], ui = im[i + k];
                double vr = re[i + k + half] * wr - im[i + k + half] * wi;
                double vi = re[i + k + half] * wi + im[i + k + half] * wr;
                re[i + k] = ur + vr; im[i + k] = ui + vi;
                re[i + k + half] = ur - vr; im[i + k + half] = ui - vi;
            }
        }
    }
}

/* Power spectrum of one prepared nfft buffer v (double) into out[bin] (bins = nfft/2+1). */
static void spectrum_d(const double *v, int nfft, int power, double *out, double *re, double *im)
{
    int bins = nfft / 2 + 1;
    int pow2 = (nfft & (nfft - 1)) == 0;
    if (pow2)
    {
        for (int i = 0; i < nfft; i++) { re[i] = v[i]; im[i] = 0.0; }
        fft_d(re, im, nfft);
    }
    else
    {
        for (int k = 0; k < bins; k++)
        {
            double sr = 0, si = 0;
            for (int t = 0; t < nfft; t++)
            {
                long e = ((long)t * k) % nfft;
                double ang = -2.0 * M_PI * (double)e / (double)nfft;
                sr += v[t] * cos(ang);
                si += v[t] * sin(ang);
            }
            re[k] = sr; im[k] = si;
        }
    }
    for (int k = 0; k < bins; k++)
        out[k] = (power == 1) ? sqrt(re[k] * re[k] + im[k] * im[k]) : re[k] * re[k] + im[k] * im[k];
}

/* Hann window as the reference builds it: FP64 then rounded to float (spectrogram.cpp:36-44). */
EXPORT void oracle_hann_window(float *w, int W)
{
    double a = (2.0 * M_PI) / W;
    for (int t = 0; t < W; t++) w[t] = (float)(0.5 * (1.0 - cos(a * (t + 0.5))));
}

/* dst (double) gets NFT [bins][hStride] (layoutNFT=1) or NTF [frames][hStride] per sample.
 * `preemph` != 0 applies pre-emphasis (coefficient coeff[b], border ZERO/CLAMP/REFLECT) in
 * double before framing, so the same function is the FP64 front of the fused chain. */
EXPORT void oracle_spectrogram_f64(const float *src, long srcStride, double *dst, long dstNStride, long dstHStride,
                                   int n, const int *len, int center, int reflect, const float *window, int nfft,
                                   int power, int W, int hop, int layoutNFT, int preemph, const float *coeff,
                                   int border)
{
    if (nfft == 0) nfft = W;
    int bins = nfft / 2 + 1;
    int off = center ? W / 2 : 0;
    float *wf = (float *)malloc(sizeof(float) * W);
    if (window) memcpy(wf, window, sizeof(float) * W);
    else oracle_hann_window(wf, W);
    int start0 = W < nfft ? (nfft - W) / 2 : 0;
#pragma omp parallel
    {
        double *v = (double *)malloc(sizeof(double) * nfft);
        double *re = (double *)malloc(sizeof(double) * nfft);
        double *im = (double *)malloc(sizeof(double) * nfft);
        double *pw = (double *)malloc(sizeof(double) * bins);
#pragma omp for schedule(dynamic)
        for (int b = 0; b < n; b++)
        {
            const float *x = src + (long)b * srcStride;
            int L = len[b];
            int F = oracle_num_windows(L, W, hop, center);
            double c = preemph ? (double)coeff[b] : 0.0;
            for (int f = 0; f < F; f++)
            {
                int ws = f * hop - off;
                for (int i = 0; i < nfft; i++) v[i] = 0.0;
                for (int t = 0; t < W; t++)
                {
                    int idx = ws + t;
                    double xv = 0.0;
                    int valid = 1;
                    if (idx < 0 || idx >= L)
                    {
                        if (reflect) idx = reflect_idx(idx, 0, L);
                        else valid = 0;
                    }
                    if (!valid || idx < 0 || idx >= L) xv = 0.0;
                    else if (preemph)
                    {
                        double prev = idx > 0 ? (double)x[idx - 1]
                                              : (border == 1 ? (double)x[0] : border == 2 ? (double)x[1] : 0.0);
                        xv = (double)x[idx] - c * prev;
                    }
                    else xv = (double)x[idx];
                    v[start0 + t] = (double)wf[t] * xv;
                }
                spectrum_d(v, nfft, power, pw, re, im);
                double *o = dst + (long)b * dstNStride;
                for (int k = 0; k < bins; k++)
                {
                    if (layoutNFT) o[(long)k * dstHStride + f] = pw[k];
                    else o[(long)f * dstHStride + k] = pw[k];
                }
            }
        }
        free(v); free(re); free(im); free(pw);
    }
    free(wf);
}

/* ---------------------------------------------------------------- mel filter bank
 * cpu/kernel/mel_filter_bank.cpp:40-193 with the scales of api/rppdefs.h:806-851.  The scale
 * functions are float functions (float log/exp), the filter edges FP64, the per-bin weights
 * rounded to float, and the output accumulated in float bin by bin. */
static float hz_to_mel_f(int htk, float hz)
{
    if (htk) return 1127.0f * logf(1.0f + (hz / 700.0f));
    const float fsp = 66.666667f, minLogHz = 1000.0f, minLogMel = (1000.0f - 0.0f) / fsp;
    const float stepLog = 0.068751777f, invMinLogHz = 0.001f, invStepLog = 1.0f / stepLog, invFsp = 1.0f / fsp;
    if (hz >= minLogHz) return minLogMel + logf(hz * invMinLogHz) * invStepLog;
    return (hz - 0.0f) * invFsp;
}

static float mel_to_hz_f(int htk, float mel)
{
    if (htk) return 700.0f * (expf(mel / 1127.0f) - 1.0f);
    const float fsp = 66.666667f, minLogHz = 1000.0f, minLogMel = (1000.0f - 0.0f) / fsp;
    const float stepLog = 0.068751777f;
    if (mel >= minLogMel) return minLogHz * expf(stepLog * (mel - minLogMel));
    return 0.0f + mel * fsp;
}

/* Table of one sample: interval[bin] (-1 = none), weightsDown[bin] (float), norm[filter]. */
typedef struct
{
    int start, end;     /* fftBinStart, fftBinEnd */
} mel_range;

static mel_range mel_tables(int htk, float minFreq, float maxFreq, int numFilter, float sampleRate, int normalize,
                            int nfft, int *interval, float *weightsDown, float *norm, double *weightsDownD,
                            double *normD)
{
    int numBins = nfft / 2 + 1;
    double melLow = hz_to_mel_f(htk, minFreq), melHigh = hz_to_mel_f(htk, maxFreq);
    double melStep = (melHigh - melLow) / (numFilter + 1);
    double hzStep = (double)sampleRate / nfft, invHzStep = 1.0 / hzStep;
    int binStart = (int)ceil(minFreq * invHzStep);
    int binEnd = (int)ceil(maxFreq * invHzStep);
    if (binEnd > numBins) binEnd = numBins;
    for (int i = 0; i < numFilter; i++) { norm[i] = 1.f; if (normD) normD[i] = 1.0; }
    for (int k = 0; k < numBins; k++) { interval[k] = -1; weightsDown[k] = 0.f; if (weightsDownD) weightsDownD[k] = 0.0; }
    int bin = binStart;
    double mel0 = melLow, mel1 = melLow + melStep;
    double fIter = bin * hzStep;
    for (int it = 0; it < numFilter + 1; it++, mel0 = mel1, mel1 += melStep)
    {
        double f0 = mel_to_hz_f(htk, (float)mel0);
        double f1 = mel_to_hz_f(htk, (float)(it == numFilter ? melHigh : mel1));
        double slope = 1. / (f1 - f0);
        if (normalize && it < numFilter)
        {
            double f2 = mel_to_hz_f(htk, (float)(mel1 + melStep));
            norm[it] = (float)(2.0 / (f2 - f0));
            if (normD) normD[it] = 2.0 / (f2 - f0);
        }
        for (; bin < binEnd && fIter < f1; bin++, fIter = bin * hzStep)
        {
            weightsDown[bin] = (float)((f1 - fIter) * slope);
            if (weightsDownD) weightsDownD[bin] = (f1 - fIter) * slope;
            interval[bin] = it;
        }
    }
    mel_range r = {binStart, binEnd};
    return r;
}

EXPORT void oracle_mel_filter_bank(const float *src, long srcNStride, long srcHStride, float *dst, long dstNStride,
                                   long dstHStride, int n, const int *dims, float maxFreqVal, float minFreq, int htk,
                                   int numFilter, float sampleRate, int normalize)
{
    float maxFreq = (maxFreqVal == 0) ? sampleRate / 2 : maxFreqVal;
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        int nfft = (dims[2 * b] - 1) * 2, numBins = nfft / 2 + 1, frames = dims[2 * b + 1];
        int *interval = (int *)malloc(sizeof(int) * (numBins + 1));
        float *wd = (float *)malloc(sizeof(float) * (numBins + 1));
        float *norm = (float *)malloc(sizeof(float) * (numFilter + 1));
        mel_range r = mel_tables(htk, minFreq, maxFreq, numFilter, sampleRate, normalize, nfft, interval, wd, norm,
                                 NULL, NULL);
        const float *x = src + (long)b * srcNStride;
        float *y = dst + (long)b * dstNStride;
        long zc = frames + 8 < dstHStride ? frames + 8 : dstHStride;
        for (int m = 0; m < numFilter; m++)
            for (long t = 0; t < zc; t++) y[m * dstHStride + t] = 0.f;
        for (int bin = r.start; bin < r.end; bin++)
        {
            const float *row = x + (long)bin * srcHStride;
            int up = interval[bin], down = up - 1;
            float wDown = wd[bin], wUp = 1.0f - wd[bin];
            if (down >= 0)
            {
                float w = normalize ? wDown * norm[down] : wDown;
                float *o = y + (long)down * dstHStride;
                for (int t = 0; t < frames; t++) o[t] = o[t] + row[t] * w;
            }
            if (up >= 0 && up < numFilter)
            {
                float w = normalize ? wUp * norm[up] : wUp;
                float *o = y + (long)up * dstHStride;
                for (int t = 0; t < frames; t++) o[t] = o[t] + row[t] * w;
            }
        }
        free(interval); free(wd); free(norm);
    }
}

/* FP64 mel of an FP64 spectrum: same filter placement, weights kept in double. */
EXPORT void oracle_mel_filter_bank_f64(const double *src, long srcNStride, long srcHStride, double *dst,
                                       long dstNStride, long dstHStride, int n, const int *dims, float maxFreqVal,
                                       float minFreq, int htk, int numFilter, float sampleRate, int normalize)
{
    float maxFreq = (maxFreqVal == 0) ? sampleRate / 2 : maxFreqVal;
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        int nfft = (dims[2 * b] - 1) * 2, numBins = nfft / 2 + 1, frames = dims[2 * b + 1];
        int *interval = (int *)malloc(sizeof(int) * (numBins + 1));
        float *wd = (float *)malloc(sizeof(float) * (numBins + 1));
        float *norm = (float *)malloc(sizeof(float) * (numFilter + 1));
        double *wdD = (double *)malloc(sizeof(double) * (numBins + 1));
        double *normD = (double *)malloc(sizeof(double) * (numFilter + 1));
        mel_range r = mel_tables(htk, minFreq, maxFreq, numFilter, sampleRate, normalize, nfft, interval, wd, norm,
                                 wdD, normD);
        const double *x = src + (long)b * srcNStride;
        double *y = dst + (long)b * dstNStride;
        for (int m = 0; m < numFilter; m++)
            for (long t = 0; t < frames; t++) y[m * dstHStride + t] = 0.0;
        for (int bin = r.start; bin < r.end; bin++)
        {
            const double *row = x + (long)bin * srcHStride;
            int up = interval[bin], down = up - 1;
            if (down >= 0)
            {
                double w = normalize ? wdD[bin] * normD[down] : wdD[bin];
                for (int t = 0; t < frames; t++) y[(long)down * dstHStride + t] += row[t] * w;
            }
            if (up >= 0 && up < numFilter)
            {
                double w = normalize ? (1.0 - wdD[bin]) * normD[up] : (1.0 - wdD[bin]);
                for (int t = 0; t < frames; t++) y[(long)up * dstHStride + t] += row[t] * w;
            }
        }
        free(interval); free(wd); free(norm); free(wdD); free(normD);
    }
}

/* Exposes the per-sample filter placement (tests compare the GPU-built tables with it). */
EXPORT void oracle_mel_tables(int htk, float minFreq, float maxFreqVal, int numFilter, float sampleRate,
                              int normalize, int nfft, int *interval, float *weightsDown, float *norm, int *range)
{
    float maxFreq = (maxFreqVal == 0) ? sampleRate / 2 : maxFreqVal;
    mel_range r = mel_tables(htk, minFreq, maxFreq, numFilter, sampleRate, normalize, nfft, interval, weightsDown,
                             norm, NULL, NULL);
    range[0] = r.start;
    range[1] = r.end;
}

/* ---------------------------------------------------------------- to_decibels
 * cpu/kernel/to_decibels.cpp:39-95: minRatio = pow(10, cutOff/mult) (denorm-min if 0),
 * mult *= log10(2), reference = per-sample max over the ROI when 0, y = mult*log2(max(minRatio,
 * x*inv)). */
EXPORT void oracle_to_decibels(const float *src, long srcNStride, long srcHStride, float *dst, long dstNStride,
                               long dstHStride, int n, const unsigned *dims /* {width,height} pairs */,
                               float cutOffDB, float multiplier, float referenceMagnitude)
{
    float minRatio = (float)pow(10, cutOffDB / multiplier);
    if (minRatio == 0.0f) minRatio = nextafterf(0.0f, 1.0f);
    const float log10Factor = 0.3010299956639812;
    multiplier *= log10Factor;
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        const float *x = src + (long)b * srcNStride;
        float *y = dst + (long)b * dstNStride;
        unsigned width = dims[2 * b], height = dims[2 * b + 1];
        float ref = referenceMagnitude;
        if (!referenceMagnitude)
        {
            ref = -FLT_MAX;
            if (width == 1)
            {
                for (unsigned i = 0; i < height; i++) if (x[i] > ref) ref = x[i];
            }
            else
                for (unsigned r = 0; r < height; r++)
                    for (unsigned c = 0; c < width; c++)
                        if (x[(long)r * srcHStride + c] > ref) ref = x[(long)r * srcHStride + c];
        }
        float inv = ref ? (1.f / ref) : 1.0f;
        if (width == 1)
        {
            for (unsigned i = 0; i < height; i++)
            {
                float v = x[i] * inv;
                y[i] = multiplier * log2f(minRatio < v ? v : minRatio);
            }
        }
        else
            for (unsigned r = 0; r < height; r++)
                for (unsigned c = 0; c < width; c++)
                {
                    float v = x[(long)r * srcHStride + c] * inv;
                    y[(long)r * dstHStride + c] = multiplier * log2f(minRatio < v ? v : minRatio);
                }
    }
}

/* FP64 decibels of a 2-D FP64 array per sample ([rows][hStride], rows x cols valid). */
EXPORT void oracle_to_decibels_f64(const double *src, long nStride, long hStride, double *dst, int n, const int *rows,
                                   const int *cols, double cutOffDB, double multiplier, double referenceMagnitude)
{
    double minRatio = pow(10.0, cutOffDB / multiplier);
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        const double *x = src + (long)b * nStride;
        double *y = dst + (long)b * nStride;
        double ref = referenceMagnitude;
        if (ref == 0.0)
        {
            ref = -DBL_MAX;
            for (int r = 0; r < rows[b]; r++)
                for (int c = 0; c < cols[b]; c++)
                    if (x[(long)r * hStride + c] > ref) ref = x[(long)r * hStride + c];
        }
        double inv = ref != 0.0 ? 1.0 / ref : 1.0;
        for (int r = 0; r < rows[b]; r++)
            for (int c = 0; c < cols[b]; c++)
            {
                double v = x[(long)r * hStride + c] * inv;
                y[(long)r * hStride + c] = multiplier * log10(v > minRatio ? v : minRatio);
            }
    }
}

/* ---------------------------------------------------------------- non-silent region
 * cpu/kernel/non_silent_region_detection.cpp:105-184: float moving sum of squares restarted
 * every resetInterval samples, cutoff, first/last index at or above it, begin moved back by
 * windowLength-1.  `mms` (optional, n x srcStride) receives the moving mean square. */
EXPORT void oracle_nsr(const float *src, long srcStride, int n, const int *len, int *begin, int *length,
                       float cutOffDB, int windowLength, float referencePower, int resetInterval, float *mms,
                       float *cutoffOut)
{
    const float cutOff = powf(10.0f, cutOffDB * 0.1f);
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < n; b++)
    {
        const float *x = src + (long)b * srcStride;
        int L = len[b];
        float *m = (float *)calloc(L > 0 ? L : 1, sizeof(float));
        int resetLength = (resetInterval == -1) ? L : resetInterval;
        float meanFactor = 1.0f / windowLength;
        int windowBegin = -windowLength + 1;
        for (int outPos = 0; outPos < L;)
        {
            float sum = 0.0f;
            for (int i = windowBegin > 0 ? windowBegin : 0; i < outPos; i++) sum += x[i] * x[i];
            int end = outPos + resetLength < L ? outPos + resetLength : L;
            for (; outPos < end; outPos++, windowBegin++)
            {
                sum += x[outPos] * x[outPos];
                m[outPos] = sum * meanFactor;
                if (windowBegin >= 0) sum -= x[windowBegin] * x[windowBegin];
            }
        }
        float base = referencePower;
        if (referencePower == 0.0f)
        {
            base = L > 0 ? m[0] : 0.f;
            for (int i = 1; i < L; i++) if (base < m[i]) base = m[i];
        }
        float cutOffMag = base * cutOff;
        int endIdx = L, beginIdx = L, db, de;
        for (int i = 0; i < endIdx; i++) if (m[i] >= cutOffMag) { beginIdx = i; break; }
        if (beginIdx == endIdx) { db = 0; de = 0; }
        else
        {
            for (int i = endIdx - 1; i >= beginIdx; i--) if (m[i] >= cutOffMag) { endIdx = i; break; }
            db = beginIdx;
            de = endIdx - beginIdx + 1;
        }
        if (db != 0 && de != 0)
        {
            int nb = db - (windowLength - 1);
            if (nb < 0) nb = 0;
            de += db - nb;
            db = nb;
        }
        begin[b] = db;
        length[b] = de;
        if (mms) memcpy(mms + (long)b * srcStride, m, sizeof(float) * (size_t)L);
        if (cutoffOut) cutoffOut[b] = cutOffMag;
        free(m);
    }
}

/* ---------------------------------------------------------------- resampling window
 * The test suite's caller-side LUT builder, utilities/test_suite/rpp_test_suite_audio.h:390-430
 * (Hann-windowed sinc, float arithmetic as written there).  lut must hold coeffs + 5 floats;
 * out[0..2] = scale, center, lobes of the resulting RpptResamplingWindow. */
static float ts_sinc(float x)
{
    x *= M_PI;
    return (fabsf(x) < 1e-5f) ? (1.f - (x * x * 0.16666667)) : sinf(x) / x;
}

static double ts_hann(double x) { return 0.5 * (1 + cos(x * M_PI)); }

EXPORT void oracle_windowed_sinc(int coeffs, int lobes, float *lut, float *out)
{
    float scale = 2.0f * lobes / (coeffs - 1);
    float scale_envelope = 2.0f / coeffs;
    int lookupSize = coeffs + 5;
    int center = (coeffs - 1) * 0.5f;
    for (int i = 0; i < lookupSize; i++) lut[i] = 0.f;
    for (int i = 0; i < coeffs; i++)
    {
        float x = (i - center) * scale;
        float y = (i - center) * scale_envelope;
        float w = ts_sinc(x) * ts_hann(y);
        lut[i + 1] = w;
    }
    out[0] = 1 / scale;
    out[1] = center + 1;
    out[2] = (float)lobes;
}

/* ---------------------------------------------------------------- slice (1-D and 2-D)
 * src/modules/tensor/cpu/kernel/slice.cpp:40-60 (per-sample anchor, shape, roi lengths) and
 * :197-228: maxLen_d = min(shape_d, length_d - anchor_d) with length_d = roi[numDims + d] (the roi
 * begin values are not read); when any anchor_d + shape_d > length_d and padding is enabled, the
 * first dstStride0 - 1 elements of the sample are filled with the fill value; then the box
 * [anchor, anchor + maxLen) is copied.  Negative box extents (anchor beyond the length) copy
 * nothing here; the reference converts them to huge unsigned sizes.  elemSize 4 (float) or 1 (u8). */
EXPORT void oracle_slice(const void *src, long srcStride0, long srcStride1, void *dst, long dstStride0,
                         long dstStride1, int n, int numDims, const int *anchor, const int *shape,
                         const unsigned *roi, const void *fill, int enablePadding, int elemSize)
{
    for (int b = 0; b < n; b++)
    {
        const int *a = anchor + b * numDims, *s = shape + b * numDims;
        const int *len = (const int *)(roi + b * numDims * 2 + numDims);
        const char *sp = (const char *)src + (size_t)b * srcStride0 * elemSize;
        char *dp = (char *)dst + (size_t)b * dstStride0 * elemSize;
        int need = 0;
        for (int d = 0; d < numDims; d++)
            if (a[d] + s[d] > len[d]) need = 1;
        if (need && enablePadding)
            for (long i = 0; i < dstStride0 - 1; i++) memcpy(dp + i * elemSize, fill, elemSize);
        if (numDims == 1)
        {
            int m = s[0] < len[0] - a[0] ? s[0] : len[0] - a[0];
            if (m > 0) memcpy(dp, sp + (size_t)a[0] * elemSize, (size_t)m * elemSize);
        }
        else
        {
            int mh = s[0] < len[0] - a[0] ? s[0] : len[0] - a[0];
            int mw = s[1] < len[1] - a[1] ? s[1] : len[1] - a[1];
            for (int r = 0; r < mh && mw > 0; r++)
                memcpy(dp + (size_t)r * dstStride1 * elemSize,
                       sp + ((size_t)(a[0] + r) * srcStride1 + a[1]) * elemSize, (size_t)mw * elemSize);
        }
    }
}

/* ---------------------------------------------------------------- slice (3-D and 4-D)
 * src/modules/tensor/cpu/kernel/slice.cpp:61-199, with the layout parameters of
 * rppt_tensor_geometric_augmentations.cpp:1074-1082 (src/include/common/rppi_validate.hpp:41-64).
 * strides: the descriptor's strides[0 .. numDims] (batch first); dims: its dims[1 .. numDims].
 * layout: 0 NCHW, 1 NHWC (3-D), 2 NCDHW, 3 NDHWC (4-D); any other layout copies nothing.
 * Channel-first: the spatial dims are 1.., every channel's box is copied (the channel anchor and
 * shape are not read), and the destination advances by the SOURCE's channel stride between
 * channels, as the reference does; channelParam is the channel count (the reference defines it
 * for 1 and 3 channels only).  Channel-last: the spatial dims are 0.., a row copies width x
 * channels elements.  Padding: when any spatial anchor + shape > length, the first dstStride0 - 1
 * elements are filled first.  Negative extents copy nothing (the reference turns them into huge
 * unsigned sizes). */
EXPORT void oracle_slice_nd(const void *src, const long *srcStrides, void *dst, const long *dstStrides,
                            const int *srcDims, int n, int numDims, int layout, const int *anchor, const int *shape,
                            const unsigned *roi, const void *fill, int enablePadding, int elemSize)
{
    const int chFirst = (numDims == 3 && layout == 0) || (numDims == 4 && layout == 2);
    const int chLast = (numDims == 3 && layout == 1) || (numDims == 4 && layout == 3);
    const int sp = numDims - 1;           /* spatial dims */
    const int o0 = chFirst ? 1 : 0;       /* first spatial dim */
    for (int b = 0; b < n; b++)
    {
        const int *a = anchor + b * numDims, *s = shape + b * numDims;
        const int *len = (const int *)(roi + b * numDims * 2 + numDims);
        const char *sb = (const char *)src + (size_t)b * srcStrides[0] * elemSize;
        char *db = (char *)dst + (size_t)b * dstStrides[0] * elemSize;
        int m[3] = {1, 1, 1}, need = 0, neg = 0;
        for (int k = 0; k < sp; k++)
        {
            const int d = o0 + k;
            if (a[d] + s[d] > len[d]) need = 1;
            m[k] = s[d] < len[d] - a[d] ? s[d] : len[d] - a[d];
            if (m[k] <= 0) neg = 1;
        }
        if (need && enablePadding)
            for (long i = 0; i < dstStrides[0] - 1; i++) memcpy(db + i * elemSize, fill, elemSize);
        if (neg || !(chFirst || chLast)) continue;
        if (chFirst)
        {
            const int C = srcDims[0];
            long sOff = 0;
            for (int k = 0; k < sp; k++) sOff += (long)a[o0 + k] * (k + 1 < sp ? srcStrides[o0 + k + 1] : 1);
            long dCh = 0;
            for (int c = 0; c < C; c++)
            {
                for (int i = 0; i < (sp == 3 ? m[0] : 1); i++)
                    for (int j = 0; j < m[sp - 2]; j++)
                    {
                        long so = sOff + (long)c * srcStrides[1], dof = dCh;
                        if (sp == 3)
                        {
                            so += (long)i * srcStrides[2] + (long)j * srcStrides[3];
                            dof += (long)i * dstStrides[2] + (long)j * dstStrides[3];
                        }
                        else
                        {
                            so += (long)j * srcStrides[2];
                            dof += (long)j * dstStrides[2];
                        }
                        memcpy(db + dof * elemSize, sb + so * elemSize, (size_t)m[sp - 1] * elemSize);
                    }
                dCh += srcStrides[1];   /* the source's channel stride (slice.cpp:111, :181) */
            }
        }
        else
        {
            const int C = srcDims[numDims - 1];
            long sOff = (long)a[0] * srcStrides[1] + (sp == 3 ? (long)a[1] * srcStrides[2] + (long)a[2] * C
                                                              : (long)a[1] * C);
            for (int i = 0; i < (sp == 3 ? m[0] : 1); i++)
                for (int j = 0; j < m[sp - 2]; j++)
                {
                    long so = sOff, dof = 0;
                    if (sp == 3)
                    {
                        so += (long)i * srcStrides[1] + (long)j * srcStrides[2];
                        dof += (long)i * dstStrides[1] + (long)j * dstStrides[2];
                    }
                    else
                    {
                        so += (long)j * srcStrides[1];
                        dof += (long)j * dstStrides[1];
                    }
                    memcpy(db + dof * elemSize, sb + so * elemSize, (size_t)m[sp - 1] * C * elemSize);
                }
        }
    }
}

/* ---------------------------------------------------------------- normalize (2-D, F32)
 * src/modules/tensor/cpu/kernel/normalize.cpp:29-120 (recursive sums, inverse std dev), :417-470
 * (normalize_2D_tensor) and :507-600 (the 2-D branch of normalize_f32_f32_host_tensor);
 * rpp_rsqrt_sse / rpp_rsqrt_ps of src/include/common/cpu/rpp_cpu_simd_math.hpp:870-930, restated
 * with the same SSE reciprocal-square-root instruction so that the restatement matches the
 * reference on the same CPU.  mean / stdDev are in-out arrays as in the reference: computed
 * values are written into them; with computeMeanStddev == 0 the caller's stdDev values are
 * replaced by scale / stdDev (1 where 0) for the first maxSize entries. */
#include <immintrin.h>

static void n_sum(float *out, const float *in, int stride, int n)
{
    if (n > 32)
    {
        int h = n >> 1;
        float t1 = 0, t2 = 0;
        n_sum(&t1, in, stride, h);
        n_sum(&t2, in + h * stride, stride, n - h);
        t1 += t2;
        *out += t1;
    }
    else
    {
        float t = 0;
        for (int i = 0; i < n; i++) t += in[i * stride];
        *out += t;
    }
}

static void n_dsq(float *out, const float *in, int stride, int n, float mean)
{
    if (n > 32)
    {
        int h = n >> 1;
        float t1 = 0, t2 = 0;
        n_dsq(&t1, in, stride, h, mean);
        n_dsq(&t2, in + h * stride, stride, n - h, mean);
        t1 += t2;
        *out += t1;
    }
    else
    {
        float t = 0;
        for (int i = 0; i < n; i++)
        {
            float c = in[i * stride] - mean;
            float c2 = c * c;
            t += c2;
        }
        *out += t;
    }
}

static float n_rsqrt_ps(float x)
{
    float y = _mm_cvtss_f32(_mm_rsqrt_ss(_mm_set_ss(x)));
    return y * (1.5f - x * 0.5f * y * y);
}

static void n_rsqrt_sse(float *v, long n, float rdiv, float mul)
{
    long i = 0;
    __m128 r4 = _mm_set1_ps(rdiv), m4 = _mm_set1_ps(mul * 0.5f), three = _mm_set1_ps(3.0f), zero = _mm_set1_ps(0.0f);
    for (; i + 4 <= n; i += 4)
    {
        __m128 x = _mm_mul_ps(_mm_loadu_ps(v + i), r4);
        __m128 mask = _mm_cmpneq_ps(x, zero);
        __m128 y = _mm_and_ps(_mm_rsqrt_ps(x), mask);
        __m128 y2 = _mm_mul_ps(y, y);
        __m128 xy2 = _mm_mul_ps(x, y2);
        y = _mm_mul_ps(y, _mm_sub_ps(three, xy2));
        y = _mm_mul_ps(y, m4);
        _mm_storeu_ps(v + i, y);
    }
    for (; i < n; i++)
    {
        float x = v[i] * rdiv;
        v[i] = x ? n_rsqrt_ps(x) * mul : 0;
    }
}

/* src/dst: [n][srcStride0] samples with row stride stride1 (elements); roi: n * 4 (begin0, begin1,
 * length0, length1; the begins are not read).  Returns 0, or -1 for an axisMask other than 1..3. */
EXPORT int oracle_normalize_2d(const float *src, long srcStride0, long srcStride1, float *dst, long dstStride0,
                               long dstStride1, int n, unsigned axisMask, float *mean, float *stdDev, int computeMeanStddev,
                               float scale, float shift, const unsigned *roi)
{
    if (axisMask < 1 || axisMask > 3) return -1;
    unsigned maxSize = 1;
    for (int b = 0; b < n; b++)
    {
        unsigned size = 1;
        for (int i = 0; i < 2; i++) size *= (axisMask & (1u << i)) ? 1 : roi[4 * b + 2 + i];
        if (size > maxSize) maxSize = size;
    }
    if (!computeMeanStddev)
    {
        for (unsigned i = 0; i < maxSize; i++) stdDev[i] = (!stdDev[i]) ? 1.0f : scale / stdDev[i];
        maxSize = 0;
    }
    for (int b = 0; b < n; b++)
    {
        const unsigned *length = roi + 4 * b + 2;
        const float *s = src + (long)b * srcStride0;
        float *d = dst + (long)b * dstStride0;
        float *mn = mean + (long)b * maxSize, *sd = stdDev + (long)b * maxSize;
        for (long i = 0; i < dstStride0; i++) d[i] = 0.0f;
        int stride[2], red[2], ps[2];
        if (axisMask == 3) { stride[0] = stride[1] = 1; red[0] = 1; red[1] = length[0] * length[1]; ps[0] = ps[1] = 0; }
        else if (axisMask == 1) { stride[0] = (int)srcStride1; stride[1] = 1; red[0] = length[1]; red[1] = length[0]; ps[0] = 1; ps[1] = 0; }
        else { stride[0] = 1; stride[1] = (int)srcStride1; red[0] = length[0]; red[1] = length[1]; ps[0] = 0; ps[1] = 1; }
        if (computeMeanStddev & 1)
        {
            float nf = (float)(1.0 / red[1]);
            const float *p = s;
            for (int i = 0; i < red[0]; i++)
            {
                mn[i] = 0;
                n_sum(&mn[i], p, stride[0], red[1]);
                p += stride[1];
                mn[i] *= nf;
            }
        }
        if (computeMeanStddev & 2)
        {
            float nf = (float)(1.0 / red[1]);
            const float *p = s;
            for (int i = 0; i < red[0]; i++)
            {
                sd[i] = 0;
                n_dsq(&sd[i], p, stride[0], red[1], mn[i]);
                p += stride[1];
            }
            n_rsqrt_sse(sd, red[0], nf, scale);
        }
        if (ps[1])
        {
            for (unsigned i = 0; i < length[0]; i++)
            {
                const float *sr = s + i * srcStride1;
                float *dr = d + i * dstStride1;
                float m = mn[i], iv = sd[i];
                for (unsigned j = 0; j < length[1]; j++) dr[j] = (sr[j] - m) * iv + shift;
            }
        }
        else
        {
            int pi = 0;
            const float *sr = s;
            float *dr = d;
            for (unsigned i = 0; i < length[0]; i++)
            {
                for (unsigned j = 0; j < length[1]; j++)
                {
                    dr[j] = (sr[j] - mn[pi]) * sd[pi] + shift;
                    pi += ps[0];
                }
                pi = (!ps[1]) ? 0 : pi + ps[1];
                sr += srcStride1;
                dr += dstStride1;
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- normalize (N-D, all types; F32 3-D)
 * src/modules/tensor/cpu/kernel/normalize.cpp:122-244 (3-D and N-D statistics), :244-415 (3-D and
 * N-D normalization), :472-505 (collapse_axis), :507-767 (normalize_f32_f32_host_tensor's 3-D and
 * N-D branches) and :768-868 (normalize_generic_host_tensor, used for U8 / F16 / I8 at every rank);
 * rpp_rsqrt_avx of src/include/common/cpu/rpp_cpu_simd_math.hpp:936-986.
 * Element types: 0 F32, 1 F16, 2 U8, 3 I8.  Deliberate differences from the host path, which this
 * library follows instead of it: integer results are clamped to the type's range before the
 * truncating conversion (the host's conversion of an out-of-range float is undefined; in range
 * both truncate), I8 values are read and written as signed (the host reads them through an
 * unsigned cast and writes unsigned bytes), and F16 results are rounded to nearest even. */
static float h2f(unsigned short h)
{
    const unsigned sign = (unsigned)(h & 0x8000) << 16, e = (h >> 10) & 31, m = h & 1023;
    unsigned u;
    if (e == 31) u = sign | 0x7f800000u | (m << 13);
    else if (e) u = sign | ((e + 112) << 23) | (m << 13);
    else
    {
        float v = (float)m * (1.0f / 16777216.0f);   /* subnormal: m * 2^-24, exact */
        memcpy(&u, &v, 4);
        u |= sign;
    }
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static unsigned short f2h(float f)   /* round to nearest even */
{
    unsigned u;
    memcpy(&u, &f, 4);
    const unsigned sign = (u >> 16) & 0x8000, a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return (unsigned short)(sign | (a > 0x7f800000u ? 0x7e00 : 0x7c00));
    if (a >= 0x477ff000u) return (unsigned short)(sign | 0x7c00);   /* >= 65520: infinity */
    if (a < 0x38800000u)                                             /* below 2^-14: subnormal */
    {
        float v;
        memcpy(&v, &a, 4);
        return (unsigned short)(sign | (unsigned)nearbyintf(v * 16777216.0f));
    }
    const unsigned mant = a & 0x7fffff, rem = mant & 0x1fff;
    unsigned h = ((((a >> 23) - 112) << 10) | (mant >> 13));
    if (rem > 0x1000 || (rem == 0x1000 && (h & 1))) h++;
    return (unsigned short)(sign | h);
}

static float ld_t(const void *p, int t, long i)
{
    switch (t)
    {
    case 0: return ((const float *)p)[i];
    case 1: return h2f(((const unsigned short *)p)[i]);
    case 2: return (float)((const unsigned char *)p)[i];
    default: return (float)((const signed char *)p)[i];
    }
}

static void st_t(void *p, int t, long i, float v)
{
    switch (t)
    {
    case 0: ((float *)p)[i] = v; break;
    case 1: ((unsigned short *)p)[i] = f2h(v); break;
    case 2: ((unsigned char *)p)[i] = (unsigned char)(v > 255.f ? 255.f : v < 0.f ? 0.f : v); break;
    default: ((signed char *)p)[i] = (signed char)(v > 127.f ? 127.f : v < -128.f ? -128.f : v); break;
    }
}

static int esize_t(int t) { return t == 0 ? 4 : t == 1 ? 2 : 1; }

static void t_sum(float *out, const char *in, int t, long stride, long n)
{
    if (n > 32)
    {
        long h = n >> 1;
        float t1 = 0, t2 = 0;
        t_sum(&t1, in, t, stride, h);
        t_sum(&t2, in + h * stride * esize_t(t), t, stride, n - h);
        t1 += t2;
        *out += t1;
    }
    else
    {
        float tmp = 0;
        for (long i = 0; i < n; i++) tmp += ld_t(in, t, i * stride);
        *out += tmp;
    }
}

static void t_dsq(float *out, const char *in, int t, long stride, long n, float mean)
{
    if (n > 32)
    {
        long h = n >> 1;
        float t1 = 0, t2 = 0;
        t_dsq(&t1, in, t, stride, h, mean);
        t_dsq(&t2, in + h * stride * esize_t(t), t, stride, n - h, mean);
        t1 += t2;
        *out += t1;
    }
    else
    {
        float tmp = 0;
        for (long i = 0; i < n; i++)
        {
            float c = ld_t(in, t, i * stride) - mean;
            float c2 = c * c;
            tmp += c2;
        }
        *out += tmp;
    }
}

__attribute__((target("avx"))) static void n_rsqrt_avx(float *v, long n, float rdiv, float scale)
{
    long i = 0;
    const __m256 r = _mm256_set1_ps(rdiv), m = _mm256_set1_ps(scale * 0.5f), three = _mm256_set1_ps(3.0f);
    for (; i + 8 <= n; i += 8)
    {
        __m256 x = _mm256_mul_ps(_mm256_loadu_ps(v + i), r);
        __m256 mask = _mm256_cmp_ps(x, _mm256_setzero_ps(), _CMP_NEQ_OQ);
        __m256 y = _mm256_and_ps(_mm256_rsqrt_ps(x), mask);
        __m256 xy2 = _mm256_mul_ps(x, _mm256_mul_ps(y, y));
        y = _mm256_mul_ps(_mm256_mul_ps(y, _mm256_sub_ps(three, xy2)), m);
        _mm256_storeu_ps(v + i, y);
    }
    for (; i < n; i++)
    {
        float x = v[i] * rdiv;
        v[i] = x ? n_rsqrt_ps(x) * scale : 0;
    }
}

/* compute_ND_mean / compute_ND_stddev (normalize.cpp:200-242), restated with the same recursion. */
static void nd_stat(int sq, const char *src, int t, float *mean, float *std, const unsigned *dims, const unsigned *stride,
                    const unsigned *axis, unsigned T, unsigned level, unsigned index, unsigned size, unsigned norm,
                    unsigned last)
{
    const int es = esize_t(t);
    if (level == T - 1 && axis[T - 1])
    {
        if (sq) t_dsq(&std[index], src, t, stride[level], dims[level], mean[index]);
        else t_sum(&mean[index], src, t, stride[level], dims[level]);
    }
    else if (level == T)
    {
        if (sq) t_dsq(&std[index], src, t, stride[norm], dims[norm], mean[index]);
        else t_sum(&mean[index], src, t, stride[norm], dims[norm]);
    }
    else if (!axis[level])
    {
        for (unsigned i = 0; i < dims[level]; i++)
            nd_stat(sq, src + (long)i * stride[level] * es, t, mean, std, dims, stride, axis, T, level + 1,
                    index + i * (size / dims[level]), size / dims[level], norm, last);
    }
    else if (level == last)
        nd_stat(sq, src, t, mean, std, dims, stride, axis, T, level + 1, index, size, level, last);
    else
        for (unsigned i = 0; i < dims[level]; i++)
            nd_stat(sq, src + (long)i * stride[level] * es, t, mean, std, dims, stride, axis, T, level + 1, index,
                    size, level, last);
}

/* The 3-D statistics (normalize.cpp:122-198): dims/stride are the srcReductionDims / srcStride of
 * the axis mask; params i * dims[1] + j (consecutive) or i. */
static void stat3d(int sq, const float *src, float *mean, float *std, const unsigned *dims, const unsigned *stride,
                   float scale, int consecutive)
{
    if (consecutive)
    {
        float nf = (float)(1.0 / dims[2]);
        const float *p = src;
        for (unsigned i = 0; i < dims[0]; i++)
        {
            const float *row = p;
            for (unsigned j = 0; j < dims[1]; j++)
            {
                unsigned idx = i * dims[1] + j;
                if (sq)
                {
                    std[idx] = 0;
                    t_dsq(&std[idx], (const char *)row, 0, stride[0], dims[2], mean[idx]);
                }
                else
                {
                    mean[idx] = 0;
                    t_sum(&mean[idx], (const char *)row, 0, stride[0], dims[2]);
                    mean[idx] *= nf;
                }
                row += stride[1];
            }
            p += stride[2];
        }
        if (sq) n_rsqrt_avx(std, (long)dims[0] * dims[1], nf, scale);
    }
    else
    {
        float nf = (float)(1.0 / (dims[1] * dims[2]));
        const float *p = src;
        for (unsigned i = 0; i < dims[0]; i++)
        {
            if (sq) std[i] = 0;
            else mean[i] = 0;
            const float *row = p;
            for (unsigned j = 0; j < dims[1]; j++)
            {
                if (sq) t_dsq(&std[i], (const char *)row, 0, stride[0], dims[2], mean[i]);
                else t_sum(&mean[i], (const char *)row, 0, stride[0], dims[2]);
                row += stride[1];
            }
            if (!sq) mean[i] *= nf;
            p += stride[2];
        }
        if (sq) n_rsqrt_avx(std, dims[0], nf, scale);
    }
}

/* srcStrides / dstStrides: the descriptors' strides[0 .. tensorDims]; layouts 0 NCHW, 1 NHWC. */
EXPORT int oracle_normalize_nd(const void *src, int srcType, const long *srcStrides, int srcLayout, const int *srcDims,
                               void *dst, int dstType, const long *dstStrides, int dstLayout, int n, int tensorDims,
                               unsigned axisMask, float *mean, float *std, int compute, float scale, float shift,
                               const unsigned *roi)
{
    const int T = tensorDims, ses = esize_t(srcType), des = esize_t(dstType);
    unsigned maxSize = 1;
    for (int b = 0; b < n; b++)
    {
        unsigned size = 1;
        for (int i = 0; i < T; i++) size *= (axisMask & (1u << i)) ? 1 : roi[T * 2 * b + T + i];
        if (size > maxSize) maxSize = size;
    }
    if (!compute)
    {
        for (unsigned i = 0; i < maxSize; i++) std[i] = !std[i] ? 1.0f : scale / std[i];
        maxSize = 0;
    }
    for (int b = 0; b < n; b++)
    {
        const unsigned *begin = roi + b * T * 2, *length = begin + T;
        const char *sb = (const char *)src + (long)b * srcStrides[0] * ses;
        char *db = (char *)dst + (long)b * dstStrides[0] * des;
        float *m = mean + (long)b * maxSize, *sd = std + (long)b * maxSize;
        for (long c = 0; c < dstStrides[0]; c++) st_t(db, dstType, c, 0.0f);
        if (srcType == 0 && T == 3)
        {
            unsigned rd[3] = {0, 0, 0}, rs[3] = {0, 0, 0}, ps[3] = {0, 0, 0};
            const unsigned L0 = length[0], L1 = length[1], L2 = length[2];
            const unsigned S1 = srcStrides[1], S2 = srcStrides[2], S3 = srcStrides[3];
            int consecutive = 1;
            switch (axisMask)
            {
            case 1: rd[0] = L1; rd[1] = L2; rd[2] = L0; rs[0] = S1; rs[1] = S3; rs[2] = S2; ps[1] = ps[2] = 1; break;
            case 2: rd[0] = L0; rd[1] = L2; rd[2] = L1; rs[0] = S2; rs[1] = S3; rs[2] = S1; ps[0] = ps[2] = 1; break;
            case 3: rd[0] = 1; rd[1] = L2; rd[2] = L0 * L1; rs[0] = S2; rs[1] = S3; rs[2] = S3; ps[2] = 1; break;
            case 4: rd[0] = L0; rd[1] = L1; rd[2] = L2; rs[0] = S3; rs[1] = S2; rs[2] = S1; ps[0] = ps[1] = 1; break;
            case 5: rd[0] = L1; rd[1] = L0; rd[2] = L2; rs[0] = S3; rs[1] = S1; rs[2] = S2; ps[1] = 1; consecutive = 0;
                break;
            case 6: rd[0] = 1; rd[1] = L0; rd[2] = L1 * L2; rs[0] = S3; rs[1] = S1; rs[2] = S3; ps[0] = 1; break;
            case 7: rd[0] = 1; rd[1] = 1; rd[2] = L0 * L1 * L2; rs[0] = rs[1] = rs[2] = S3; break;
            default: return -1;
            }
            const float *ch = (const float *)sb + (long)begin[0] * S1 + (long)begin[1] * S2;
            if (compute & 1) stat3d(0, ch, m, sd, rd, rs, scale, consecutive);
            if (compute & 2) stat3d(1, ch, m, sd, rd, rs, scale, consecutive);
            float *d = (float *)db;
            if (axisMask == 3 && srcLayout == 1 && dstLayout == 1 && srcDims[2] == 16)
            {
                /* normalize_3D_tensor_avx_axis3: 16 channel parameters over whole rows */
                unsigned bl = L1 * 16, al = bl / 16 * 16;
                for (unsigned i = 0; i < L0; i++)
                    for (unsigned v = 0; v < al; v++)
                        d[(long)i * dstStrides[1] + v] = ((ch[(long)i * S1 + v] - m[v % 16]) * sd[v % 16]) + shift;
            }
            else if (srcLayout == 1 && dstLayout == 1)
            {
                for (unsigned i = 0; i < L0; i++)
                    for (unsigned j = 0; j < L1; j++)
                        for (unsigned k = 0; k < L2; k++)
                        {
                            unsigned p = (ps[0] ? i : 0);
                            p = p * (ps[1] ? L1 : 1) + (ps[1] ? j : 0);
                            p = p * (ps[2] ? L2 : 1) + (ps[2] ? k : 0);
                            d[(long)i * dstStrides[1] + (long)j * dstStrides[2] + k] =
                                ((ch[(long)i * S1 + (long)j * S2 + k] - m[p]) * sd[p]) + shift;
                        }
            }
            else if (axisMask == 3 && srcLayout == 1 && dstLayout == 0)
            {
                for (unsigned i = 0; i < L0; i++)
                    for (unsigned j = 0; j < L1; j++)
                        for (unsigned k = 0; k < L2; k++)
                            d[(long)k * dstStrides[1] + (long)i * dstStrides[2] + (long)j * dstStrides[3]] =
                                ((ch[(long)i * S1 + (long)j * S2 + k] - m[k]) * sd[k]) + shift;
            }
            continue;
        }
        /* N-D: normalize_generic_host_tensor / the N-D branch of normalize_f32_f32_host_tensor */
        unsigned size = 1, total = 1, axis[16], newAxis[16], newDims[16], lastNorm = 0;
        const char *ch = sb;
        for (int i = 0; i < T; i++)
        {
            axis[i] = (axisMask & (1u << i)) ? 1 : 0;
            size *= axis[i] ? 1 : length[i];
            total *= axis[i] ? length[i] : 1;
            ch += (long)begin[i] * srcStrides[i + 1] * ses;
            newAxis[i] = newDims[i] = 0;
        }
        /* collapse_axis (normalize.cpp:472-505) */
        int skipped = 0, prev = -2, k = 0;
        unsigned nT = T;
        for (int i = 0; i < T; i++)
        {
            if (axis[i])
            {
                int temp = i - skipped;
                if (temp != prev + 1)
                {
                    newAxis[k] = 1;
                    newDims[k] = length[i];
                    prev = i;
                    k++;
                }
                else if (prev >= 0)
                {
                    newDims[prev] *= length[i];
                    skipped++;
                }
            }
            else
            {
                newDims[k] = length[i];
                k++;
            }
        }
        nT -= skipped;
        for (unsigned i = 0; i < nT; i++)
            if (newAxis[i]) lastNorm = i;
        unsigned dstr[16];
        {
            unsigned v = 1;
            for (unsigned i = nT - 1; i > 0; i--)
            {
                dstr[i] = v;
                v *= newDims[i];
            }
            dstr[0] = v;
        }
        if (compute & 1)
        {
            nd_stat(0, ch, srcType, m, sd, newDims, dstr, newAxis, nT, 0, 0, size, 0, lastNorm);
            float nf = 1.0 / total;
            for (unsigned i = 0; i < size; i++) m[i] *= nf;
        }
        if (compute & 2)
        {
            nd_stat(1, ch, srcType, m, sd, newDims, dstr, newAxis, nT, 0, 0, size, 0, lastNorm);
            float nf = (float)(1.0 / total);
            n_rsqrt_avx(sd, size, nf, scale);
        }
        /* normalize_ND_tensor_nontoggle: dense positions from the roi start (source) and the sample
         * start (destination); the parameter is the row-major index over the unnormalized dims */
        long count = 1;
        for (unsigned i = 0; i < nT; i++) count *= newDims[i];
        for (long e = 0; e < count; e++)
        {
            long rem = e;
            unsigned p = 0;
            for (unsigned l = 0; l < nT; l++)
            {
                unsigned c = (unsigned)(rem / dstr[l]);
                rem -= (long)c * dstr[l];
                if (!newAxis[l]) p = p * newDims[l] + c;
            }
            st_t(db, dstType, e, ((ld_t(ch, srcType, e) - m[p]) * sd[p]) + shift);
        }
    }
    return 0;
}
