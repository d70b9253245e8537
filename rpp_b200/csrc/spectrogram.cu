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
#include "ops.hpp"
#include "stft.cuh"

namespace rppb {
namespace {

constexpr int kThreads = 256;

struct SpecCount
{
    const int* len;
    int W, hop, maxFrames, tile;
    bool center;
    __device__ long long operator()(int b) const
    {
        int F = min(num_windows(*RPPB_RD(len + b), W, hop, center), maxFrames);
        return F <= 0 ? 0 : (F + tile - 1) / tile;
    }
};

// Shared memory plan (bytes) for one nfft, window and hop; identical on host and device.
template <int NFFT>
struct SmemLayout
{
    using S = StftShape<NFFT, kThreads>;
    size_t tw, tw1, win, span, fftBuf, out, bytes;
    __host__ __device__ SmemLayout(int W, int hop)
    {
        tw = 0;
        tw1 = tw + S::tw_bytes;
        win = tw1 + S::tw1_bytes;
        span = win + size_t(NFFT) * 4;
        fftBuf = span + S::span_bytes(W, hop);
        out = fftBuf + S::fft_bytes;
        bytes = out + S::out_bytes;
    }
};

template <int NFFT>
__global__ void __launch_bounds__(kThreads, (NFFT <= 512 ? 3 : 2)) spectrogram_fft_kernel(SpectrogramArgs a,
                                                                      const float2* __restrict__ twiddle,
                                                                      const long long* __restrict__ prefix)
{
    using S = StftShape<NFFT, kThreads>;
    constexpr int TF = S::TF, BINS = S::BINS;
    extern __shared__ __align__(16) unsigned char smem[];
    const SmemLayout<NFFT> lay(a.windowLength, a.windowStep);
    float2* s_tw = reinterpret_cast<float2*>(smem + lay.tw);
    float2* s_tw1 = reinterpret_cast<float2*>(smem + lay.tw1);
    float* s_win = reinterpret_cast<float*>(smem + lay.win);
    float* s_span = reinterpret_cast<float*>(smem + lay.span);
    float2* s_fft = reinterpret_cast<float2*>(smem + lay.fftBuf);
    float* s_out = reinterpret_cast<float*>(smem + lay.out);

    const int W = a.windowLength;
    stft_tables<NFFT, kThreads>(twiddle, a.window, W, s_tw, s_tw1, s_win, s_span);
    const int centerOffset = a.center ? W / 2 : 0;
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, a.n, s_prefix);
    const long long total = prefix[a.n];

    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int f0 = int(w - prefix[b]) * TF;
        const int L = *RPPB_RD(a.len + b);
        const int F = min(num_windows(L, W, a.windowStep, a.center), a.maxFrames);
        const PlainSource src{a.src + size_t(b) * a.srcStride, L, a.reflect};
        stft_tile<NFFT, kThreads>(src, f0, F, W, a.windowStep, centerOffset, a.power, s_win, s_tw, s_tw1, s_span,
                                  s_fft, s_out);
        __syncthreads();
        // store the tile: a warp writes consecutive frames of one bin (NFT) or bins of one frame (NTF)
        const int Tv = min(TF, F - f0);
        float* y = a.dst + size_t(b) * a.dstNStride;
        if (a.nft)
        {
            // thread -> (frame f, bins k, k + kThreads / TF, ...): pointers advance by a fixed step
            constexpr int KS = kThreads / TF;
            const int f = threadIdx.x % TF;
            int k = threadIdx.x / TF;
            if (f < Tv)
            {
                const float* sp = s_out + k * S::OUT_LD + f;
                float* yp = y + size_t(k) * a.dstHStride + f0 + f;
                const size_t ystep = size_t(KS) * a.dstHStride;
                for (; k < BINS; k += KS, sp += KS * S::OUT_LD, yp += ystep) *RPPB_WR(yp) = *sp;
            }
        }
        else
        {
            for (int idx = threadIdx.x; idx < BINS * TF; idx += kThreads)
            {
                const int f = idx / BINS, k = idx % BINS;
                if (f < Tv) *RPPB_WR(y + (size_t(f0 + f) * a.dstHStride + k)) = s_out[k * S::OUT_LD + f];
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
        int F = min(num_windows(*RPPB_RD(len + b), W, hop, center), maxFrames);
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
    for (int i = threadIdx.x; i < N; i += kThreads) s_tw[i] = *RPPB_RD(twiddle + i);
    const int W = a.windowLength;
    const int off = (W < N) ? (N - W) / 2 : 0;
    const int centerOffset = a.center ? W / 2 : 0;
    const int bins = N / 2 + 1;
    __shared__ long long s_prefix[kPrefixCache];
    prefix = cache_prefix(prefix, a.n, s_prefix);
    const long long total = prefix[a.n];
    for (long long w = blockIdx.x; w < total; w += gridDim.x)
    {
        const int b = ragged_find(prefix, a.n, w);
        const int frame = int(w - prefix[b]);
        const int L = *RPPB_RD(a.len + b);
        const float* x = a.src + size_t(b) * a.srcStride;
        const int ws = frame * a.windowStep - centerOffset;
        __syncthreads();
        for (int t = threadIdx.x; t < N; t += kThreads)
        {
            const int u = t - off;
            s_v[t] = (u >= 0 && u < W) ? *RPPB_RD(a.window + u) * PlainSource{x, L, a.reflect}(ws + u) : 0.f;
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
            if (a.nft) *RPPB_WR(y + (size_t(k) * a.dstHStride + frame)) = o;
            else *RPPB_WR(y + (size_t(frame) * a.dstHStride + k)) = o;
        }
    }
}

template <int NFFT>
void launch_fft(Handle& h, long long* prefix, const SpectrogramArgs& a, const float2* tw)
{
    launch_ragged_prefix(SpecCount{a.len, a.windowLength, a.windowStep, a.maxFrames, Plan<NFFT>::TF, a.center}, a.n, prefix,
                         h.stream());
    const size_t smem = SmemLayout<NFFT>(a.windowLength, a.windowStep).bytes;
    if (smem > 227 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "window/hop too large for the frame tile");
    int grid = persistent_grid(h, reinterpret_cast<const void*>(spectrogram_fft_kernel<NFFT>), kThreads, smem);
    spectrogram_fft_kernel<NFFT><<<grid, kThreads, smem, h.stream()>>>(a, tw, prefix);
    count_launch();
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
    int grid = persistent_grid(h, reinterpret_cast<const void*>(spectrogram_dft_kernel), kThreads, smem);
    spectrogram_dft_kernel<<<grid, kThreads, smem, h.stream()>>>(a, tw, prefix);
    count_launch();
    check_cuda(cudaGetLastError(), "spectrogram_dft_kernel");
}

}  // namespace rppb
