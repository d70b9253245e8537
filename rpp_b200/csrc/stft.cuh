// One tile of STFT frames -> power (or magnitude) spectrum in shared memory.
//
// Shared by the plain spectrogram kernel and the fused front end so both produce bit-identical
// spectra.  Framing follows src/modules/tensor/cpu/kernel/spectrogram.cpp:116-212: frame f
// starts at f * hop - centerOffset, samples outside the signal are reflected or zero, the frame
// is multiplied by the window and placed at offset (nfft - W)/2 of the nfft buffer.  The signal
// is read through a Source functor, which lets the fused kernel apply pre-emphasis while it
// gathers (reflection then applies to the pre-emphasized signal, exactly as when the two ops run
// one after the other).
//
// A frame is transformed by G = R2 threads: pack the nfft real samples as M = nfft/2 complex
// points, stage-1 R1-point register DFT + twiddle, one shared-memory exchange, stage-2 R2-point
// register DFT, then unpack the nfft/2+1 bins of the real transform (fft.cuh).
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace rppb {

template <int NFFT>
struct Plan;
template <>
struct Plan<128> { static constexpr int R1 = 8, R2 = 8, TF = 32; };
template <>
struct Plan<256> { static constexpr int R1 = 16, R2 = 8, TF = 32; };
template <>
struct Plan<512> { static constexpr int R1 = 16, R2 = 16, TF = 32; };
template <>
struct Plan<1024> { static constexpr int R1 = 32, R2 = 16, TF = 16; };
template <>
struct Plan<2048> { static constexpr int R1 = 32, R2 = 32, TF = 16; };

template <int NFFT, int THREADS>
struct StftShape
{
    static constexpr int M = NFFT / 2;
    static constexpr int R1 = Plan<NFFT>::R1, R2 = Plan<NFFT>::R2, TF = Plan<NFFT>::TF;
    static constexpr int G = R2;                       // threads per frame
    static constexpr int FPP = THREADS / G;            // frames per pass
    static constexpr int PASSES = (TF + FPP - 1) / FPP;
    static constexpr int BINS = M + 1;
    static constexpr int FFT_SLOT = R1 * (R2 + 1);     // float2 per frame slot (padded rows)
    static constexpr int OUT_LD = TF + 1;              // leading dimension of the [BINS][TF] tile
    static constexpr size_t fft_bytes = size_t(FPP) * FFT_SLOT * 8;
    static constexpr size_t out_bytes = size_t(BINS) * OUT_LD * 4;
    static_assert(R1 * R2 == M, "plan");
    static_assert(R1 % G == 0, "stage 2 assigns R1 / G rows per thread");
};

// The signal as stored.
struct PlainSource
{
    const float* x;
    int L;
    bool reflect;
    __device__ __forceinline__ float operator()(int i) const
    {
        if (i >= 0 && i < L) return __ldg(x + i);
        if (!reflect || L <= 0) return 0.f;
        return __ldg(x + reflect_index(i, 0, L));
    }
};

// The pre-emphasized signal y[0] = x[0] - c*border, y[i] = x[i] - c*x[i-1]
// (pre_emphasis_filter.cpp:46-71, same roundings as the pre_emphasis_filter kernel).
struct PreemphSource
{
    const float* x;
    int L;
    bool reflect;
    float c, border;
    __device__ __forceinline__ float at(int i) const
    {
        const float prev = i == 0 ? border : __ldg(x + i - 1);
        return __fsub_rn(__ldg(x + i), __fmul_rn(c, prev));
    }
    __device__ __forceinline__ float operator()(int i) const
    {
        if (i >= 0 && i < L) return at(i);
        if (!reflect || L <= 0) return 0.f;
        return at(reflect_index(i, 0, L));
    }
};

// Computes frames f0 .. f0+TF-1 (those < F) of one sample into s_out[bin * OUT_LD + f] and
// leaves the other columns undefined.  All THREADS threads of the CTA must call it.
template <int NFFT, int THREADS, class Src>
__device__ __forceinline__ void stft_tile(const Src& src, int f0, int F, int W, int hop, int centerOffset, int power,
                                          const float* __restrict__ s_win, const float2* __restrict__ s_tw,
                                          float2* __restrict__ s_fft, float* __restrict__ s_out)
{
    using S = StftShape<NFFT, THREADS>;
    constexpr int M = S::M, R1 = S::R1, R2 = S::R2, TF = S::TF, G = S::G, FPP = S::FPP, BINS = S::BINS;
    const int j = threadIdx.x % G;
    const int slot = threadIdx.x / G;
    float2* buf = s_fft + slot * S::FFT_SLOT;
    const int off = (W < NFFT) ? (NFFT - W) / 2 : 0;
#pragma unroll 1
    for (int pass = 0; pass < S::PASSES; ++pass)
    {
        const int fl = pass * FPP + slot;
        const int frame = f0 + fl;
        const int ws = frame * hop - centerOffset;
        const bool live = fl < TF && frame < F;
        float2 z[R1];
#pragma unroll
        for (int m = 0; m < R1; ++m)
        {
            const int t0 = 2 * (j + R2 * m) - off;   // window index of the real part
            float re = 0.f, im = 0.f;
            if (live)
            {
                if (t0 >= 0 && t0 < W) re = s_win[t0] * src(ws + t0);
                if (t0 + 1 >= 0 && t0 + 1 < W) im = s_win[t0 + 1] * src(ws + t0 + 1);
            }
            z[m] = make_float2(re, im);
        }
        fft::Dft<R1>::run(z);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1)
        {
            const float2 t = s_tw[(2 * j * k1) & (NFFT - 1)];
            buf[k1 * (R2 + 1) + j] = fft::cmul_conj(z[k1], t.x, t.y);
        }
        __syncwarp();
        constexpr int ROWS = R1 / G;
        float2 y[ROWS][R2];
#pragma unroll
        for (int r = 0; r < ROWS; ++r)
        {
            const int k1 = j + G * r;
#pragma unroll
            for (int jj = 0; jj < R2; ++jj) y[r][jj] = buf[k1 * (R2 + 1) + jj];
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < ROWS; ++r)
        {
            const int k1 = j + G * r;
            fft::Dft<R2>::run(y[r]);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) buf[k1 + R1 * k2] = y[r][k2];   // Z in natural order
        }
        __syncwarp();
        if (fl < TF)
        {
            for (int k = j; k < BINS; k += G)
            {
                const float2 A = buf[k & (M - 1)];
                const float2 B = buf[(M - k) & (M - 1)];
                // E = (A + conj(B)) / 2,  O = (A - conj(B)) / (2i),  X = E + W_nfft^k O
                const float er = 0.5f * (A.x + B.x), ei = 0.5f * (A.y - B.y);
                const float orr = 0.5f * (A.y + B.y), oi = -0.5f * (A.x - B.x);
                const float2 t = s_tw[k & (NFFT - 1)];
                const float xr = er + fmaf(orr, t.x, oi * t.y);
                const float xi = ei + fmaf(oi, t.x, -orr * t.y);
                const float p = fmaf(xr, xr, xi * xi);
                s_out[k * S::OUT_LD + fl] = (power == 1) ? sqrtf(p) : p;
            }
        }
        __syncwarp();
    }
}

}  // namespace rppb
