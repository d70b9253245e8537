// One tile of STFT frames -> power (or magnitude) spectrum in shared memory.
//
// Shared by the plain spectrogram kernel and the fused front end so both produce bit-identical
// spectra.  Framing follows src/modules/tensor/cpu/kernel/spectrogram.cpp:116-212: frame f
// starts at f * hop - centerOffset, samples outside the signal are reflected or zero, the frame
// is multiplied by the window and placed at offset (nfft - W)/2 of the nfft buffer.
//
// Per tile of TF frames:
//   1. the tile's input span ((TF-1)*hop + W samples) is staged in shared memory with coalesced
//      loads (float4 when the span lies inside the signal and is 16-byte aligned); the Source
//      functor applies reflect/zero padding and, in the fused kernel, pre-emphasis, so padding is
//      resolved once per sample rather than once per frame;
//   2. each frame is transformed by G = R2 threads as a real FFT: the nfft samples are packed into
//      M = nfft/2 complex points, stage 1 is an R1-point register DFT with twiddles W_M^(j*k1) from a
//      [k1][j] table (conflict-free), one shared-memory exchange, stage 2 an R2-point register DFT;
//   3. the real spectrum is unpacked in bin pairs (k, M-k), which share their two loads:
//      X[k] = E + W^k O and X[M-k] = conj(E - W^k O) with E = (Z[k] + conj Z[M-k]) / 2,
//      O = (Z[k] - conj Z[M-k]) / 2i.
#pragma once

#include <type_traits>

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
struct Plan<512> { static constexpr int R1 = 16, R2 = 16, TF = 16; };
template <>
struct Plan<1024> { static constexpr int R1 = 32, R2 = 16, TF = 16; };
template <>
struct Plan<2048> { static constexpr int R1 = 32, R2 = 32, TF = 16; };

// TFX: frames per tile (Plan<NFFT>::TF by default; the fused kernel also instantiates other sizes,
// which change the schedule and never the arithmetic of a frame).
template <int NFFT, int THREADS, int TFX = Plan<NFFT>::TF>
struct StftShape
{
    static constexpr int M = NFFT / 2;
    static constexpr int R1 = Plan<NFFT>::R1, R2 = Plan<NFFT>::R2, TF = TFX;
    static constexpr int G = R2;                       // threads per frame
    static constexpr int FPP = THREADS / G;            // frames per pass
    static constexpr int PASSES = (TF + FPP - 1) / FPP;
    static constexpr int BINS = M + 1;
    static constexpr int FFT_SLOT = R1 * (R2 + 1);     // float2 per frame slot (padded rows)
    static constexpr int OUT_LD = TF + 2;              // leading dimension of the [BINS][TF] tile: even, so
                                                       // frame pairs load as float2; conflict-free unpack stores
    static constexpr size_t fft_bytes = size_t(FPP) * FFT_SLOT * 8;
    static constexpr size_t out_bytes = size_t(BINS) * OUT_LD * 4;
    static constexpr size_t tw_bytes = (size_t(M / 2 + 1) * 8 + 15) & ~size_t(15);   // W_nfft^k, k <= M/2
    static constexpr size_t tw1_bytes = size_t(R1) * R2 * 8;      // W_M^(j*k1) as [k1][j]
    static_assert(R1 * R2 == M, "plan");
    static_assert(R1 % G == 0, "stage 2 assigns R1 / G rows per thread");
    // The window starts at offset (nfft - W) / 2 of the nfft buffer (0 when W >= nfft).
    __host__ __device__ static int window_offset(int W) { return W < NFFT ? (NFFT - W) / 2 : 0; }
    // Span buffer: span_pad zero floats (>= the window offset, a multiple of 4), the tile's
    // (TF - 1) * hop + W staged samples, then up to nfft - offset - W more zeros, so every frame
    // reads a full nfft-sample buffer without bounds checks (the window is 0 outside [0, W)).
    __host__ __device__ static int span_pad(int W) { return (window_offset(W) + 3) & ~3; }
    __host__ __device__ static int span_tail(int W)
    {
        const int t = NFFT - window_offset(W) - W;
        return t > 0 ? t : 0;
    }
    __host__ __device__ static size_t span_bytes(int W, int hop)
    {
        return (size_t(span_pad(W) + (TF - 1) * hop + W + span_tail(W)) * 4 + 15) & ~size_t(15);
    }
};

// The signal as stored.
struct PlainSource
{
    const float* x;
    int L;
    bool reflect;
    __device__ __forceinline__ float operator()(int i) const
    {
        if (i >= 0 && i < L) return __ldg(RPPB_RD(x + i));
        if (!reflect || L <= 0) return 0.f;
        return __ldg(RPPB_RD(x + reflect_index(i, 0, L)));
    }
    // 4 consecutive in-range samples from 16-byte aligned x + i
    __device__ __forceinline__ float4 quad(int i) const
    {
        return __ldg(RPPB_RD(reinterpret_cast<const float4*>(x + i)));
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
        const float prev = i == 0 ? border : __ldg(RPPB_RD(x + i - 1));
        return __fsub_rn(__ldg(RPPB_RD(x + i)), __fmul_rn(c, prev));
    }
    __device__ __forceinline__ float operator()(int i) const
    {
        if (i >= 0 && i < L) return at(i);
        if (!reflect || L <= 0) return 0.f;
        return at(reflect_index(i, 0, L));
    }
    __device__ __forceinline__ float4 quad(int i) const
    {
        const float4 v = __ldg(RPPB_RD(reinterpret_cast<const float4*>(x + i)));
        const float p = i == 0 ? border : __ldg(RPPB_RD(x + i - 1));
        return make_float4(__fsub_rn(v.x, __fmul_rn(c, p)), __fsub_rn(v.y, __fmul_rn(c, v.x)),
                           __fsub_rn(v.z, __fmul_rn(c, v.y)), __fsub_rn(v.w, __fmul_rn(c, v.z)));
    }
};

// Fills the per-CTA constant tables: s_tw[k] = W_nfft^k (k <= M/2, the unpack twiddles), s_tw1[k1][j] =
// W_M^(j*k1) = W_nfft^(2*j*k1), s_win[n] = the window in buffer coordinates (window[n - offset] for
// n - offset in [0, W), else 0), and zeroes the span buffer's leading pad (never staged over).
// All threads call; ends with __syncthreads.
template <int NFFT, int THREADS>
__device__ __forceinline__ void stft_tables(const float2* __restrict__ twiddle, const float* __restrict__ window, int W,
                                            float2* s_tw, float2* s_tw1, float* s_win, float* s_span)
{
    using S = StftShape<NFFT, THREADS>;
    for (int i = threadIdx.x; i <= S::M / 2; i += THREADS) s_tw[i] = *RPPB_RD(twiddle + i);
    for (int i = threadIdx.x; i < S::R1 * S::R2; i += THREADS)
    {
        const int k1 = i / S::R2, j = i % S::R2;
        s_tw1[i] = *RPPB_RD(twiddle + ((2 * j * k1) & (NFFT - 1)));
    }
    const int off = S::window_offset(W);
    for (int i = threadIdx.x; i < NFFT; i += THREADS)
        s_win[i] = (i >= off && i - off < W) ? *RPPB_RD(window + (i - off)) : 0.f;
    for (int i = threadIdx.x; i < S::span_pad(W); i += THREADS) s_span[i] = 0.f;
    __syncthreads();
}

// Stages the input span of frames f0 .. f0+TF-1 (those < F) in s_span after its zero pad and zeroes
// the tail, so that buffer sample n of tile frame fl is s_span[span_pad(W) + fl * hop - offset + n]
// for every n in [0, nfft).  All THREADS threads call it; ends with __syncthreads.
template <int NFFT, int THREADS, int TFX = Plan<NFFT>::TF, class Src>
__device__ __forceinline__ void stft_stage_span(const Src& src, int f0, int F, int W, int hop, int centerOffset,
                                                float* __restrict__ s_span)
{
    using S = StftShape<NFFT, THREADS, TFX>;
    constexpr int TF = S::TF;
    const int Tv = min(TF, F - f0);
    const int spanStart = f0 * hop - centerOffset;
    const int spanLen = (Tv - 1) * hop + W;
    float* const s_data = s_span + S::span_pad(W);
    if (spanStart >= 0 && spanStart + spanLen <= src.L &&
        (reinterpret_cast<uintptr_t>(src.x + spanStart) & 15) == 0)
    {
        const int quads = spanLen >> 2;
        // 4 quads per thread in flight before their stores
        for (int q0 = threadIdx.x; q0 < quads; q0 += 4 * THREADS)
        {
            float4 v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (q0 + j * THREADS < quads) v[j] = src.quad(spanStart + 4 * (q0 + j * THREADS));
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (q0 + j * THREADS < quads) reinterpret_cast<float4*>(s_data)[q0 + j * THREADS] = v[j];
        }
        for (int i = (quads << 2) + threadIdx.x; i < spanLen; i += THREADS) s_data[i] = src(spanStart + i);
    }
    else
    {
        for (int i = threadIdx.x; i < spanLen; i += THREADS) s_data[i] = src(spanStart + i);
    }
    for (int i = threadIdx.x; i < S::span_tail(W); i += THREADS) s_data[spanLen + i] = 0.f;
    __syncthreads();
}

// Computes frames f0 .. f0+TF-1 (those < F) of one sample into s_out[bin * OUT_LD + f] and
// leaves the other columns undefined.  All THREADS threads of the CTA must call it.
template <int NFFT, int THREADS, int TFX = Plan<NFFT>::TF, class Src>
__device__ __forceinline__ void stft_tile(const Src& src, int f0, int F, int W, int hop, int centerOffset, int power,
                                          const float* __restrict__ s_win, const float2* __restrict__ s_tw,
                                          const float2* __restrict__ s_tw1, float* __restrict__ s_span,
                                          float2* __restrict__ s_fft, float* __restrict__ s_out)
{
    using S = StftShape<NFFT, THREADS, TFX>;
    constexpr int M = S::M, R1 = S::R1, R2 = S::R2, TF = S::TF, G = S::G, FPP = S::FPP, BINS = S::BINS;

    // ---- 1. stage the tile's input span (after the zero pad), then zero its tail
    stft_stage_span<NFFT, THREADS, TFX>(src, f0, F, W, hop, centerOffset, s_span);
    const int Tv = min(TF, F - f0);
    float* const s_data = s_span + S::span_pad(W);

    const int j = threadIdx.x % G;
    const int slot = threadIdx.x / G;
    float2* buf = s_fft + slot * S::FFT_SLOT;
    const int off = S::window_offset(W);
    const bool pairs = ((off | hop) & 1) == 0;   // (window, sample) pairs are 8-byte aligned

    // power (2) or magnitude (1) of bins k and M - k, as the two halves of the unpack share loads;
    // thread j takes k = j + G*i for i < M / (2G) (every k below M/2 once), thread 0 also k = M/2.
    // Fully unrolled with constant offsets: Z[M] (a copy of Z[0], stored with the natural-order
    // spectrum) stands in for Z[(M - k) mod M] at k = 0.
    constexpr int LD = S::OUT_LD;
    auto bin_pair = [&](auto magTag, float2 A, float2 B, float2 t, float& p0, float& p1) {
        constexpr bool kMag = decltype(magTag)::value;
        // E = (A + conj(B)) / 2,  O = (A - conj(B)) / (2i),  P = W^k O
        const float2 sum = fft::mul2(make_float2(0.5f, 0.5f), fft::add2(A, B));   // (er, orr)
        const float2 dif = fft::mul2(make_float2(-0.5f, 0.5f), fft::sub2(A, B));  // (oi, ei)
        const float er = sum.x, orr = sum.y, oi = dif.x, ei = dif.y;
        const float pr = fmaf(orr, t.x, oi * t.y);
        const float pi = fmaf(oi, t.x, -orr * t.y);
        const float2 X = fft::add2(make_float2(er, ei), make_float2(pr, pi));   // X[k] = E + P
        const float2 Y = fft::sub2(make_float2(er, ei), make_float2(pr, pi));   // X[M-k] = conj(E - P)
        const float2 sq = fft::mul2(make_float2(X.y, Y.y), make_float2(X.y, Y.y));
        p0 = fmaf(X.x, X.x, sq.x);
        p1 = fmaf(Y.x, Y.x, sq.y);
        if (kMag)
        {
            p0 = sqrtf(p0);
            p1 = sqrtf(p1);
        }
    };
    auto unpack = [&](auto magTag, int fl) {
        const float2* pa = buf + j;
        const float2* pb = buf + (M - j);
        const float2* pt = s_tw + j;
        float* o1 = s_out + j * LD + fl;
        float* o2 = s_out + (M - j) * LD + fl;
#pragma unroll
        for (int i = 0; i < M / (2 * G); ++i)
        {
            float p0, p1;
            bin_pair(magTag, pa[G * i], pb[-G * i], pt[G * i], p0, p1);
            o1[G * i * LD] = p0;
            o2[-G * i * LD] = p1;
        }
        if (j == 0)
        {
            float p0, p1;
            bin_pair(magTag, buf[M / 2], buf[M / 2], s_tw[M / 2], p0, p1);
            s_out[(M / 2) * LD + fl] = p0;
        }
    };

#pragma unroll 1
    for (int pass = 0; pass < S::PASSES; ++pass)
    {
        const int fl = pass * FPP + slot;
        const bool live = fl < Tv;
        // buffer sample n of frame fl is fs[n]; the pads make every n in [0, nfft) readable
        const float* fs = s_data + fl * hop - off;
        float2 z[R1];
        if (live && pairs)
        {
#pragma unroll
            for (int m = 0; m < R1; ++m)
            {
                const int n = 2 * (j + R2 * m);
                z[m] = fft::mul2(*reinterpret_cast<const float2*>(s_win + n), *reinterpret_cast<const float2*>(fs + n));
            }
        }
        else if (live)
        {
#pragma unroll
            for (int m = 0; m < R1; ++m)
            {
                const int n = 2 * (j + R2 * m);
                z[m] = make_float2(s_win[n] * fs[n], s_win[n + 1] * fs[n + 1]);
            }
        }
        else
        {
#pragma unroll
            for (int m = 0; m < R1; ++m) z[m] = make_float2(0.f, 0.f);
        }
        fft::Dft<R1>::run(z);
        buf[j] = z[0];   // W_M^(j*0) = 1
#pragma unroll
        for (int k1 = 1; k1 < R1; ++k1)
        {
            const float2 t = s_tw1[k1 * R2 + j];
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
            if (k1 == 0) buf[M] = y[r][0];                                    // Z[M] = Z[0]
        }
        __syncwarp();
        if (fl < TF)
        {
            if (power == 1) unpack(std::true_type{}, fl);
            else unpack(std::false_type{}, fl);
        }
        __syncwarp();
    }
    (void)BINS;
}

}  // namespace rppb
