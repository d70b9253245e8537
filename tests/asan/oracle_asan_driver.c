/*
 * Memory-safety check of the oracle (oracle/rppb_oracle.c), the CPU checker every parity test relies
 * on.  Built with -fsanitize=address,undefined by tests/test_oracle_asan.py and run on edge-case
 * batches: lengths 0, 1, 2, shorter than the window, and long ones, in buffers allocated to exactly
 * the sizes the descriptors give, so that a read or write past a sample's stride or past the batch is
 * reported.  Exit status 0 when every call completes cleanly.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void oracle_pre_emphasis(const float *, long, float *, long, int, const int *, const float *, int);
void oracle_down_mixing(const float *, long, float *, long, int, const int *, int);
void oracle_resample(const float *, long, float *, long, int, const float *, const float *, const int *,
                     const float *, int, float, float, int);
int oracle_num_windows(int, int, int, int);
void oracle_spectrogram_f64(const float *, long, double *, long, long, int, const int *, int, int, const float *,
                            int, int, int, int, int, int, const float *, int);
void oracle_mel_filter_bank(const float *, long, long, float *, long, long, int, const int *, float, float, int, int,
                            float, int);
void oracle_to_decibels(const float *, long, long, float *, long, long, int, const unsigned *, float, float, float);
void oracle_nsr(const float *, long, int, const int *, int *, int *, float, int, float, int, float *, float *);
void oracle_windowed_sinc(int, int, float *, float *);
void oracle_slice(const void *, long, long, void *, long, long, int, int, const int *, const int *, const unsigned *,
                  const void *, int, int);
int oracle_normalize_2d(const float *, long, long, float *, long, long, int, unsigned, float *, float *, int, float,
                        float, const unsigned *);

#define N 6
static const int kLens[N] = {0, 1, 2, 300, 1601, 9000};   /* 300 < window 400; 9000 > reset interval 8192 */

static float *signal(long count, unsigned seed)
{
    float *x = malloc((size_t)(count > 0 ? count : 1) * sizeof(float));
    for (long i = 0; i < count; i++)
    {
        seed = seed * 1664525u + 1013904223u;
        x[i] = ((float)(seed >> 8) / 16777216.0f - 0.5f) * (i % 97 < 60 ? 1.0f : 1e-4f);
    }
    return x;
}

static int max_len(void)
{
    int m = 1;
    for (int b = 0; b < N; b++) m = kLens[b] > m ? kLens[b] : m;
    return m;
}

static void check_time_domain(void)
{
    const long S = max_len();
    float *x = signal(N * S, 1), *y = signal(N * S, 2), coeff[N];
    for (int b = 0; b < N; b++) coeff[b] = 0.97f;
    for (int border = 0; border < 3; border++) oracle_pre_emphasis(x, S, y, S, N, kLens, coeff, border);

    /* interleaved channels: stride = S * 3 for up to 3 channels, mono destination */
    float *xs = signal(N * S * 3, 3);
    int dims[2 * N];
    for (int b = 0; b < N; b++)
    {
        dims[2 * b] = kLens[b];
        dims[2 * b + 1] = 1 + b % 3;
    }
    oracle_down_mixing(xs, S * 3, y, S, N, dims, 0);
    oracle_down_mixing(xs, S * 3, y, S, N, dims, 1);

    /* resampling to 18.4 kHz and down from 48 kHz, mono: destination stride = longest output */
    const int lobes = 16, coeffs = lobes * 64 + 1;
    float *lut = malloc((coeffs + 5) * sizeof(float)), out[3];
    oracle_windowed_sinc(coeffs, lobes, lut, out);
    float inRate[N], outRate[N];
    long D = 1;
    for (int b = 0; b < N; b++)
    {
        inRate[b] = b % 2 ? 48000.f : 16000.f;
        outRate[b] = b % 2 ? 16000.f : 18400.f;
        dims[2 * b] = kLens[b];
        dims[2 * b + 1] = 1;
        const long o = (long)ceilf((float)kLens[b] * outRate[b] / inRate[b]);
        D = o > D ? o : D;
    }
    float *yr = signal(N * D, 4);
    oracle_resample(x, S, yr, D, N, inRate, outRate, dims, lut, coeffs + 5, out[0], out[1], (int)out[2]);

    /* non-silent regions: window 2048, reset interval 8192 and whole-length (-1) */
    int begin[N], length[N];
    float *mms = signal(N * S, 5), cut[N];
    oracle_nsr(x, S, N, kLens, begin, length, -60.f, 2048, 0.f, 8192, mms, cut);
    oracle_nsr(x, S, N, kLens, begin, length, -60.f, 2048, 0.f, -1, NULL, cut);

    /* slice of each clip's first half, with and without padding */
    int anchor[N], shape[N];
    unsigned roi[2 * N];
    for (int b = 0; b < N; b++)
    {
        anchor[b] = kLens[b] / 4;
        shape[b] = kLens[b] / 2 + 3;
        roi[2 * b] = 0;
        roi[2 * b + 1] = (unsigned)kLens[b];
    }
    const float fill = -1.f;
    oracle_slice(x, S, 0, y, S, 0, N, 1, anchor, shape, roi, &fill, 0, 4);
    oracle_slice(x, S, 0, y, S, 0, N, 1, anchor, shape, roi, &fill, 1, 4);
    free(x); free(y); free(xs); free(lut); free(yr); free(mms);
}

static void check_spectral(int center, int nft)
{
    const long S = max_len();
    const int nfft = 512, W = 400, hop = 160, bins = nfft / 2 + 1, nmel = 128;
    int F = 1, frames[N];
    for (int b = 0; b < N; b++)
    {
        frames[b] = oracle_num_windows(kLens[b], W, hop, center);
        if (frames[b] < 0) frames[b] = 0;
        F = frames[b] > F ? frames[b] : F;
    }
    float *x = signal(N * S, 6), coeff[N];
    for (int b = 0; b < N; b++) coeff[b] = 0.97f;
    double *spec64 = malloc((size_t)N * bins * F * sizeof(double));
    const long hs = nft ? F : bins;
    oracle_spectrogram_f64(x, S, spec64, (long)bins * F, hs, N, kLens, center, 1, NULL, nfft, 2, W, hop, nft, 1, coeff,
                           0);
    oracle_spectrogram_f64(x, S, spec64, (long)bins * F, hs, N, kLens, center, 0, NULL, nfft, 1, W, hop, nft, 0, NULL,
                           0);
    if (!nft)
    {
        free(x); free(spec64);
        return;
    }
    /* mel and decibels on a float spectrum [N][bins][F] */
    float *spec = malloc((size_t)N * bins * F * sizeof(float));
    for (long i = 0; i < (long)N * bins * F; i++) spec[i] = (float)spec64[i];
    int dims[2 * N];
    unsigned wh[2 * N], nroi[4 * N];
    for (int b = 0; b < N; b++)
    {
        dims[2 * b] = bins;
        dims[2 * b + 1] = frames[b];
        wh[2 * b] = (unsigned)frames[b];
        wh[2 * b + 1] = nmel;
        nroi[4 * b] = 0;
        nroi[4 * b + 1] = 0;
        nroi[4 * b + 2] = nmel;
        nroi[4 * b + 3] = (unsigned)frames[b];
    }
    float *mel = malloc((size_t)N * nmel * F * sizeof(float)), *db = malloc((size_t)N * nmel * F * sizeof(float));
    oracle_mel_filter_bank(spec, (long)bins * F, F, mel, (long)nmel * F, F, N, dims, 8000.f, 0.f, 0, nmel, 16000.f, 1);
    oracle_mel_filter_bank(spec, (long)bins * F, F, mel, (long)nmel * F, F, N, dims, 0.f, 300.f, 1, nmel, 16000.f, 0);
    oracle_to_decibels(mel, (long)nmel * F, F, db, (long)nmel * F, F, N, wh, -80.f, 10.f, 0.f);
    oracle_to_decibels(mel, (long)nmel * F, F, db, (long)nmel * F, F, N, wh, -80.f, 10.f, 1.f);
    /* one parameter per column (axis 1), per row (axis 2) or per sample (axis 3) */
    const long P = (long)N * (F > nmel ? F : nmel);
    float *mean = malloc((size_t)P * sizeof(float)), *sd = malloc((size_t)P * sizeof(float));
    for (unsigned axis = 1; axis <= 3; axis++)
    {
        for (long i = 0; i < P; i++) mean[i] = 0.f, sd[i] = 1.f;
        oracle_normalize_2d(db, (long)nmel * F, F, mel, (long)nmel * F, F, N, axis, mean, sd, 3, 1.f, 0.f, nroi);
    }
    free(x); free(spec64); free(spec); free(mel); free(db); free(mean); free(sd);
}

int main(void)
{
    check_time_domain();
    for (int center = 0; center < 2; center++)
        for (int nft = 0; nft < 2; nft++) check_spectral(center, nft);
    printf("oracle asan ok\n");
    return 0;
}
