// spectrogram: short-time power (or magnitude) spectrum of each sample.
//
// Reference: src/modules/tensor/cpu/kernel/spectrogram.cpp:71-251.  Frames of windowLength
// samples start every windowStep samples (minus windowLength/2 when centred); samples outside
// the signal are reflected (get_idx_reflect, :55-69) or zero; each frame is multiplied by the
// window, placed at offset (nfft - windowLength)/2 of an nfft buffer and transformed; bin k of
// the nfft/2+1 bins gets re^2 + im^2 (power 2) or |X| (power 1).  NFT stores
// dst[bin * hStride + frame], NTF dst[frame * hStride + bin].
//
// B200 design.  Persistent CTAs walk a flat list of (sample, frame tile) units of the ragged
// batch.  For power-of-two nfft from 128 to 2048 a frame is transformed by a group of G
// threads as a real FFT: the nfft real samples are packed into M = nfft/2 complex points,
// transformed by a two-stage register FFT (fft.cuh; stage 1 R1-point, stage 2 R2-point, one
// shared-memory exchange) and unpacked into the nfft/2+1 bins with the W_nfft^k table.  The
// windowed frame is gathered straight from global memory (reflect/zero padding resolved per
// index; overlapping frames hit L1/L2), and the tile's spectrum is staged in shared memory so
// both layouts are written with coalesced rows: a warp writes 32 consecutive frames of one bin
// (NFT) or consecutive bins of one frame (NTF).  Other nfft values (including the reference's
// non-power-of-two plans) use a direct DFT kernel with the same framing.  Twiddles and the Hann
// window are computed on the host in FP64 and rounded once to float.
//
// FP32 arithmetic in a different order than the reference's third-party FFT: results match the
// host path within 1e-5 of each frame's largest bin (ffts' own FP32 error is of the same order).
#include "common.cuh"
#include "fft.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

using fft::Dft;

constexpr int kThreads = 256;

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

struct SpecCount
{
    const int* len;
    int W, hop, maxFrames, tile;
    bool center;
    __device__ long long operator()(int b) const
    {
        int F = min(num_windows(len[b], W, hop, center), maxFrames);
        return F <= 0 ? 0 : (F + tile - 1) / tile;
    }
};

// Sample of the (padded) signal at index i.
__device__ __forceinline__ float padded_sample(const float* __restrict__ x, int L, int i, bool reflect)
{
    if (i >= 0 && i < L) return __ldg(x + i);
    if (!reflect || L <= 0) return 0.f;
    return __ldg(x + reflect_index(i, 0, L));
}

template <int NFFT>
struct SmemLayout
{
    static constexpr int M = NFFT / 2;
    static constexpr int R1 = Plan<NFFT>::R1, R2 = Plan<NFFT>::R2, TF = Plan<NFFT>::TF;
    static constexpr int G = R2;
    static constexpr int FPP = kThreads / G;                 // frames per pass
    static constexpr int BINS = M + 1;
    static constexpr int FFT_SLOT = R1 * (R2 + 1);           // float2 per frame slot
    static constexpr size_t tw = 0;                                   // NFFT float2
    static constexpr size_t fftBuf = tw + size_t(NFFT) * 8;          // FPP * FFT_SLOT float2
    static constexpr size_t out = fftBuf + size_t(FPP) * FFT_SLOT * 8;   // BINS * (TF+1) float
    static constexpr size_t win = out + size_t(BINS) * (TF + 1) * 4;     // NFFT floats (window <= nfft)
    static constexpr size_t bytes = win + size_t(NFFT) * 4;
};

template <int NFFT>
__global__ void __launch_bounds__(kThreads) spectrogram_fft_kernel(SpectrogramArgs a, const float2* __restrict__ twiddle,
                                                                   const long long* __restrict__ prefix)
{
    using S = SmemLayout<NFFT>;
    constexpr int M = S::M, R1 = S::R1, R2 = S::R2, TF = S::TF, G = S::G, FPP = S::FPP, BINS = S::BINS;
    static_assert(R1 * R2 == M, "plan");
    static_assert(R1 % G == 0 || G % R1 == 0, "plan");
    extern __shared__ __align__(16) unsigned char smem[];
    float2* s_tw = reinterpret_cast<float2*>(smem + S::tw);
    float2* s_fft = reinterpret_cast<float2*>(smem + S::fftBuf);
    float* s_out = reinterpret_cast<float*>(smem + S::out);
    float* s_win = reinterpret_cast<float*>(smem + S::win);

    const int W = a.windowLength;
    for (int i = threadIdx.x; i < NFFT; i += kThreads) s_tw[i] = twiddle[i];
    for (int i = threadIdx.x; i < W; i += kThreads) s_win[i] = a.window[i];
    __syncthreads();

    const int j = threadIdx.x % G;          // thread within the frame group
    const int slot = threadIdx.x / G;       // frame slot within a pass
    float2* buf = s_fft + slot * S::FFT_SLOT;
    const int off = (W < NFFT) ? (NFFT - W) / 2 : 0;
    const int centerOffset = a.center ? W / 2 : 0;
    const long long total = prefix[a.n];

    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int f0 = int(w - prefix[b]) * TF;
        const int L = a.len[b];
        const int F = min(num_windows(L, W, a.windowStep, a.center), a.maxFrames);
        const float* x = a.src + size_t(b) * a.srcStride;

        for (int pass = 0; pass < TF / FPP + (TF % FPP ? 1 : 0); ++pass)
        {
            const int fl = pass * FPP + slot;        // frame within the tile
            const int frame = f0 + fl;
            const int ws = frame * a.windowStep - centerOffset;
            // ---- gather the windowed frame: z[n] = v[2n] + i v[2n+1], thread holds n = j + R2*m
            float2 z[R1];
#pragma unroll
            for (int m = 0; m < R1; ++m)
            {
                const int t0 = 2 * (j + R2 * m) - off;   // window index of the real part
                float re = 0.f, im = 0.f;
                if (fl < TF && frame < F)
                {
                    if (t0 >= 0 && t0 < W) re = s_win[t0] * padded_sample(x, L, ws + t0, a.reflect);
                    if (t0 + 1 >= 0 && t0 + 1 < W) im = s_win[t0 + 1] * padded_sample(x, L, ws + t0 + 1, a.reflect);
                }
                z[m] = make_float2(re, im);
            }
            // ---- stage 1: R1-point DFT over m, twiddle W_M^(j*k1) = W_nfft^(2*j*k1)
            Dft<R1>::run(z);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1)
            {
                const float2 t = s_tw[(2 * j * k1) & (NFFT - 1)];
                buf[k1 * (R2 + 1) + j] = fft::cmul_conj(z[k1], t.x, t.y);
            }
            __syncwarp();
            // ---- stage 2: R2-point DFTs over j for k1 = j, j+G, ...
            constexpr int ROWS = R1 / G > 0 ? R1 / G : 1;
            float2 y[ROWS][R2];
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
            {
                const int k1 = j + G * r;
#pragma unroll
                for (int jj = 0; jj < R2; ++jj) y[r][jj] = (k1 < R1) ? buf[k1 * (R2 + 1) + jj] : make_float2(0.f, 0.f);
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
            {
                const int k1 = j + G * r;
                Dft<R2>::run(y[r]);
                if (k1 < R1)
                {
#pragma unroll
                    for (int k2 = 0; k2 < R2; ++k2) buf[k1 + R1 * k2] = y[r][k2];   // Z in natural order
                }
            }
            __syncwarp();
            // ---- unpack the real spectrum: X[k] = E[k] + W_nfft^k O[k]
            if (fl < TF)
            {
                for (int k = j; k < BINS; k += G)
                {
                    const float2 A = buf[k & (M - 1)];
                    const float2 Bc = buf[(M - k) & (M - 1)];
                    // E = (A + conj(B)) / 2,  O = (A - conj(B)) / (2i)
                    const float er = 0.5f * (A.x + Bc.x), ei = 0.5f * (A.y - Bc.y);
                    const float orr = 0.5f * (A.y + Bc.y), oi = -0.5f * (A.x - Bc.x);
                    const float2 t = s_tw[k & (NFFT - 1)];
                    // X = E + (orr + i oi)(c - i s)
                    const float xr = er + fmaf(orr, t.x, oi * t.y);
                    const float xi = ei + fmaf(oi, t.x, -orr * t.y);
                    const float p = fmaf(xr, xr, xi * xi);
                    s_out[k * (TF + 1) + fl] = (a.power == 1) ? sqrtf(p) : p;
                }
            }
            __syncwarp();
        }
        __syncthreads();
        // ---- store the tile
        const int Tv = min(TF, F - f0);
        float* y = a.dst + size_t(b) * a.dstNStride;
        if (a.nft)
        {
            for (int idx = threadIdx.x; idx < BINS * TF; idx += kThreads)
            {
                const int k = idx / TF, f = idx % TF;
                if (f < Tv) y[size_t(k) * a.dstHStride + f0 + f] = s_out[k * (TF + 1) + f];
            }
        }
        else
        {
            for (int idx = threadIdx.x; idx < BINS * TF; idx += kThreads)
            {
                const int f = idx / BINS, k = idx % BINS;
                if (f < Tv) y[size_t(f0 + f) * a.dstHStride + k] = s_out[k * (TF + 1) + f];
            }
        }
        __syncthreads();
    }
}

// Direct DFT for any nfft: one unit per (sample, frame).
struct FrameCount
{
    const int* len;
    int W, hop, maxFrames;
    bool center;
    __device__ long long operator()(int b) const
    {
        int F = min(num_windows(len[b], W, hop, center), maxFrames);
        return F <= 0 ? 0 : F;
    }
};

__global__ void __launch_bounds__(kThreads) spectrogram_dft_kernel(SpectrogramArgs a, const float2* __restrict__ twiddle,
                                                                   const long long* __restrict__ prefix)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int N = a.nfft;
    float2* s_tw = reinterpret_cast<float2*>(smem);
    float* s_v = reinterpret_cast<float*>(smem + size_t(N) * 8);
    for (int i = threadIdx.x; i < N; i += kThreads) s_tw[i] = twiddle[i];
    const int W = a.windowLength;
    const int off = (W < N) ? (N - W) / 2 : 0;
    const int centerOffset = a.center ? W / 2 : 0;
    const int bins = N / 2 + 1;
    const long long total = prefix[a.n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int frame = int(w - prefix[b]);
        const int L = a.len[b];
        const float* x = a.src + size_t(b) * a.srcStride;
        const int ws = frame * a.windowStep - centerOffset;
        __syncthreads();
        for (int t = threadIdx.x; t < N; t += kThreads)
        {
            const int u = t - off;
            s_v[t] = (u >= 0 && u < W) ? a.window[u] * padded_sample(x, L, ws + u, a.reflect) : 0.f;
        }
        __syncthreads();
        float* y = a.dst + size_t(b) * a.dstNStride;
        for (int k = threadIdx.x; k < bins; k += kThreads)
        {
            float re = 0.f, im = 0.f;
            int e = 0;
            for (int t = 0; t < N; ++t)
            {
                const float v = s_v[t];
                const float2 tw = s_tw[e];
                re = fmaf(v, tw.x, re);
                im = fmaf(-v, tw.y, im);
                e += k;
                if (e >= N) e -= N;
            }
            const float p = fmaf(re, re, im * im);
            const float o = (a.power == 1) ? sqrtf(p) : p;
            if (a.nft) y[size_t(k) * a.dstHStride + frame] = o;
            else y[size_t(frame) * a.dstHStride + k] = o;
        }
    }
}

template <int NFFT>
void launch_fft(Handle& h, long long* prefix, const SpectrogramArgs& a, const float2* tw)
{
    using S = SmemLayout<NFFT>;
    launch_ragged_prefix(SpecCount{a.len, a.windowLength, a.windowStep, a.maxFrames, S::TF, a.center}, a.n, prefix,
                         h.stream());
    const size_t smem = S::bytes;
    check_cuda(cudaFuncSetAttribute(spectrogram_fft_kernel<NFFT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(smem)),
               "smem attr");
    int grid = persistent_grid(h, reinterpret_cast<const void*>(spectrogram_fft_kernel<NFFT>), kThreads, smem);
    spectrogram_fft_kernel<NFFT><<<grid, kThreads, smem, h.stream()>>>(a, tw, prefix);
    check_cuda(cudaGetLastError(), "spectrogram_fft_kernel");
}

void build_twiddle(float* out, size_t count, const void* ctx)
{
    const int N = *static_cast<const int*>(ctx);
    // out holds N (cos, sin) pairs of 2*pi*e/N, FP64 then rounded
    for (int e = 0; e < N; ++e)
    {
        out[2 * e] = float(fft::cos_2pi(e, N));
        out[2 * e + 1] = float(fft::cos_2pi(4L * e - N, 4L * N));
    }
    (void)count;
}

}  // namespace

const float2* spectrogram_twiddles(Handle& h, int nfft)
{
    return reinterpret_cast<const float2*>(
        h.table("twiddle" + std::to_string(nfft), size_t(nfft) * 2, build_twiddle, &nfft));
}

void launch_spectrogram(Handle& h, void* scratch, const SpectrogramArgs& a)
{
    if (a.n <= 0) return;
    long long* prefix = static_cast<long long*>(scratch);
    const float2* tw = spectrogram_twiddles(h, a.nfft);
    switch (a.nfft)
    {
        case 128: launch_fft<128>(h, prefix, a, tw); return;
        case 256: launch_fft<256>(h, prefix, a, tw); return;
        case 512: launch_fft<512>(h, prefix, a, tw); return;
        case 1024: launch_fft<1024>(h, prefix, a, tw); return;
        case 2048: launch_fft<2048>(h, prefix, a, tw); return;
        default: break;
    }
    launch_ragged_prefix(FrameCount{a.len, a.windowLength, a.windowStep, a.maxFrames, a.center}, a.n, prefix,
                         h.stream());
    const size_t smem = size_t(a.nfft) * 12;
    if (smem > 200 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "nfft too large for the direct DFT");
    check_cuda(cudaFuncSetAttribute(spectrogram_dft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "smem attr");
    int grid = persistent_grid(h, reinterpret_cast<const void*>(spectrogram_dft_kernel), kThreads, smem);
    spectrogram_dft_kernel<<<grid, kThreads, smem, h.stream()>>>(a, tw, prefix);
    check_cuda(cudaGetLastError(), "spectrogram_dft_kernel");
}

}  // namespace rppb
