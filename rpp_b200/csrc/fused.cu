// Fused front end: pre-emphasis -> STFT power -> mel filter bank -> decibels in one persistent
// launch (include/rppb_frontend.h).
//
// Work items of two kinds walk one queue, claimed in order with an atomic counter:
//   spectrum tile (clip b, frames f0..f0+TF): gather the pre-emphasized, reflected, windowed
//     frames straight from the raw signal (stft.cuh, PreemphSource), FFT them into a shared
//     power tile, project onto the mel filters from a shared CSR weight table (same weights and
//     the same ascending-bin float accumulation as the mel_filter_bank kernel), write the mel
//     power into dst, fold the tile maximum into the clip's float-ordered atomicMax, then count
//     the tile done;
//   decibel tile (clip b, same frames): wait until every spectrum tile of clip b is counted (a
//     bounded wait: a timeout sets the handle's device error word and skips the tile), then
//     convert the tile in place with the clip's maximum.
// The queue interleaves them per clip slot: [spectrum tiles of clip s][decibel tiles of clip
// s - D], so a clip's mel power is re-read D clips after it was written, while it is still in
// L2.  Claiming items in order makes the waits deadlock-free at any residency: a decibel item's
// spectrum items have lower indices and were claimed by running CTAs.
//
// HBM traffic per clip: the raw signal once, the mel power written, re-read (mostly from L2) and
// overwritten with decibels: 4 L + (4 + 4 + 4) * numFilter * frames bytes at most, against
// 8 L + 4 L + 2*4*bins*frames + ... for the four separate calls.
#include <cfloat>

#include <algorithm>
#include <string>

#include "common.cuh"
#include "mel_tables.cuh"
#include "ops.hpp"
#include "stft.cuh"

namespace rppb {

constexpr int kFusedThreads = 256;
constexpr int kDbFramesDefault = 64;          // frames per decibel item unless tuned
constexpr int kFusedPrefixCache = 320;        // slots cached in shared memory (n + lookahead + 1)
constexpr long long kWaitLimit = 1ll << 24;   // x ~128 ns sleeps: a few seconds

namespace {

// Where clip b lives: uniform-stride batch, or one entry of a clip table.
struct ClipView
{
    const float* x;
    int L;
    float* y;
    uint32_t hStride;
    int maxFrames;
    float coeff;
    bool hasSecond;   // x[1] may be read (REFLECT border of a 1-sample clip)
};

__device__ __forceinline__ ClipView clip_view(const FrontendArgs& a, int b)
{
    if (a.clips)
    {
        const RppbClip c = a.clips[b];
        const int L = c.length <= 0 ? 0 : resampled_length(c.length, c.inRate, a.outRate);
        return {c.work, L, c.dst, uint32_t(c.dstStride), c.dstStride, a.coeffAll, L >= 2};
    }
    return {a.src + size_t(b) * a.srcStride, a.len[b], a.dst + size_t(b) * a.dstNStride, a.dstHStride, a.maxFrames,
            a.coeff[b], size_t(b) * a.srcStride + 1 < a.srcElems};
}

template <int TF>
struct SlotCount
{
    FrontendArgs a;
    int n, D;
    __device__ int frames(int b) const
    {
        const ClipView c = clip_view(a, b);
        return max(0, min(num_windows(c.L, a.W, a.hop, a.center), c.maxFrames));
    }
    __device__ int tiles(int b) const { return (frames(b) + TF - 1) / TF; }
    __device__ int db_tiles(int b) const { return (frames(b) + a.dbFrames - 1) / a.dbFrames; }
    __device__ long long operator()(int s) const
    {
        long long c = 0;
        if (s < n) c += tiles(s);
        if (s - D >= 0 && s - D < n) c += db_tiles(s - D);
        return c;
    }
};

// Shared memory plan (bytes), computed identically on host and device.
template <int NFFT, int TF>
struct FusedLayout
{
    using S = StftShape<NFFT, kFusedThreads, TF>;
    size_t tw, tw1, win, span, work, csrRow, csrBin, csrW, total;
    __host__ __device__ FusedLayout(int numFilter, int W, int hop)
    {
        const int bins = S::BINS;
        tw = 0;
        tw1 = tw + S::tw_bytes;
        win = tw1 + S::tw1_bytes;
        span = win + size_t(NFFT) * 4;
        work = span + S::span_bytes(W, hop);
        // the FFT slots + power tile, or (before the loop) the mel table build
        size_t fftOut = S::fft_bytes + S::out_bytes;
        size_t tables = 2 * size_t(numFilter + 2) * 4 + size_t(numFilter) * 4 + 2 * size_t(numFilter + 1) * 8 +
                        size_t(bins) * 4 + 64;
        size_t workBytes = (fftOut > tables ? fftOut : tables);
        csrRow = (work + workBytes + 15) & ~size_t(15);
        csrBin = (csrRow + size_t(numFilter + 1) * 4 + 15) & ~size_t(15);
        csrW = (csrBin + size_t(2 * bins + 2) * 2 + 15) & ~size_t(15);
        total = (csrW + size_t(2 * bins + 2) * 4 + 15) & ~size_t(15);
    }
};

template <int NFFT, int TFX>
__global__ void __launch_bounds__(kFusedThreads, (NFFT <= 512 ? 3 : 2)) frontend_kernel(FrontendArgs a, const float2* __restrict__ twiddle,
                                                                 const long long* __restrict__ prefix,
                                                                 unsigned long long* __restrict__ workCounter,
                                                                 int* __restrict__ done, unsigned* __restrict__ maxKey,
                                                                 int* __restrict__ errorWord)
{
    using S = StftShape<NFFT, kFusedThreads, TFX>;
    constexpr int TF = S::TF, BINS = S::BINS, LD = S::OUT_LD;
    extern __shared__ __align__(16) unsigned char smem[];
    const FusedLayout<NFFT, TFX> lay(a.mel.numFilter, a.W, a.hop);
    float2* s_tw = reinterpret_cast<float2*>(smem + lay.tw);
    float2* s_tw1 = reinterpret_cast<float2*>(smem + lay.tw1);
    float* s_win = reinterpret_cast<float*>(smem + lay.win);
    float* s_span = reinterpret_cast<float*>(smem + lay.span);
    float2* s_fft = reinterpret_cast<float2*>(smem + lay.work);
    float* s_out = reinterpret_cast<float*>(smem + lay.work + S::fft_bytes);
    int* csrRow = reinterpret_cast<int*>(smem + lay.csrRow);
    unsigned short* csrBin = reinterpret_cast<unsigned short*>(smem + lay.csrBin);   // bin * LD: tile row offset
    float* csrW = reinterpret_cast<float*>(smem + lay.csrW);
    __shared__ long long s_item;
    __shared__ float s_warpMax[kFusedThreads / 32];
    const int nmel = a.mel.numFilter;

    stft_tables<NFFT, kFusedThreads>(twiddle, a.window, a.W, s_tw, s_tw1, s_win);

    // ---- mel weights as CSR rows (filter m: bins of interval m with (1 - wd) * norm, then bins of
    //      interval m + 1 with wd * norm), built in the work region before it holds FFT data
    {
        unsigned char* t = smem + lay.work;
        MelTableView v;
        v.first = reinterpret_cast<int*>(t);
        v.last = v.first + (nmel + 2);
        v.norm = reinterpret_cast<float*>(v.last + (nmel + 2));
        size_t o = (size_t(reinterpret_cast<unsigned char*>(v.norm + nmel) - t) + 7) & ~size_t(7);
        v.f0 = reinterpret_cast<double*>(t + o);
        v.f1 = v.f0 + (nmel + 1);
        v.weightsDown = reinterpret_cast<float*>(v.f1 + (nmel + 1));
        v.range = reinterpret_cast<int*>(v.weightsDown + BINS);
        build_mel_tables(v, a.mel, NFFT);   // ends with __syncthreads
        if (threadIdx.x == 0)
        {
            int acc = 0;
            for (int m = 0; m < nmel; ++m)
            {
                csrRow[m] = acc;
                if (v.last[m] > v.first[m]) acc += v.last[m] - v.first[m];
                if (v.last[m + 1] > v.first[m + 1]) acc += v.last[m + 1] - v.first[m + 1];
            }
            csrRow[nmel] = acc;
        }
        __syncthreads();
        for (int m = threadIdx.x; m < nmel; m += kFusedThreads)
        {
            int e = csrRow[m];
            const float nm = v.norm[m];
            for (int k = v.first[m]; k < v.last[m]; ++k, ++e)
            {
                float w = __fsub_rn(1.0f, v.weightsDown[k]);
                csrBin[e] = (unsigned short)(k * LD);
                csrW[e] = a.mel.normalize ? __fmul_rn(w, nm) : w;
            }
            for (int k = v.first[m + 1]; k < v.last[m + 1]; ++k, ++e)
            {
                const float w = v.weightsDown[k];
                csrBin[e] = (unsigned short)(k * LD);
                csrW[e] = a.mel.normalize ? __fmul_rn(w, nm) : w;
            }
        }
        __syncthreads();
    }

    const int centerOffset = a.center ? a.W / 2 : 0;
    const int nslots = a.n + a.lookahead;
    __shared__ long long s_prefix[kFusedPrefixCache];
    prefix = cache_prefix<kFusedPrefixCache>(prefix, nslots, s_prefix);
    const long long total = prefix[nslots];
    const SlotCount<TF> cnt{a, a.n, a.lookahead};
    const int f = threadIdx.x % TF;      // frame column this thread owns in mel / decibel tiles
    const int g = threadIdx.x / TF;
    constexpr int kGroups = kFusedThreads / TF;

    for (;;)
    {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(workCounter, 1ull);
        __syncthreads();
        const long long w = s_item;
        if (w >= total) break;
        const int s = ragged_find(prefix, nslots, w);
        const int local = int(w - prefix[s]);
        const int c1 = s < a.n ? cnt.tiles(s) : 0;
        const bool spectrumItem = local < c1;
        const int b = spectrumItem ? s : s - a.lookahead;
        const int tile = spectrumItem ? local : local - c1;
        const ClipView cv = clip_view(a, b);
        const int L = cv.L;
        const int F = min(num_windows(L, a.W, a.hop, a.center), cv.maxFrames);
        const int f0 = tile * (spectrumItem ? TF : a.dbFrames);
        const int Tv = min(spectrumItem ? TF : a.dbFrames, F - f0);
        float* y = cv.y + f0;
        const uint32_t hs = cv.hStride;

        if (spectrumItem)
        {
            const float* x = cv.x;
            const float bval = a.border == 1 ? x[0] : a.border == 2 ? (cv.hasSecond ? x[1] : 0.f) : 0.f;
            const PreemphSource src{x, L, a.reflect, cv.coeff, bval};
            stft_tile<NFFT, kFusedThreads, TFX>(src, f0, F, a.W, a.hop, centerOffset, a.power, s_win, s_tw, s_tw1, s_span,
                                           s_fft, s_out);
            __syncthreads();
            float tmax = -FLT_MAX;
            if (f < Tv)
            {
                const float* so = s_out + f;
                float* yp = y + size_t(g) * hs + f;
                const size_t ystep = size_t(kGroups) * hs;
                for (int m = g; m < nmel; m += kGroups, yp += ystep)
                {
                    float acc = 0.0f;
                    const int e1 = csrRow[m + 1];
#pragma unroll 4
                    for (int e = csrRow[m]; e < e1; ++e) acc = __fadd_rn(acc, __fmul_rn(so[csrBin[e]], csrW[e]));
                    *yp = acc;
                    tmax = fmaxf(tmax, acc);
                }
            }
            tmax = warp_max(tmax);
            if ((threadIdx.x & 31) == 0) s_warpMax[threadIdx.x >> 5] = tmax;
            __threadfence();   // each thread's mel stores are visible device-wide before the tile is counted
            __syncthreads();
            if (threadIdx.x == 0)
            {
                float v = s_warpMax[0];
                for (int i = 1; i < kFusedThreads / 32; ++i) v = fmaxf(v, s_warpMax[i]);
                atomicMax(maxKey + b, float_key(v));
                __threadfence();
                atomicAdd(done + b, 1);
            }
        }
        else
        {
            if (threadIdx.x == 0)
            {
                const int need = cnt.tiles(b);
                long long spins = 0;
                while (atomicAdd(done + b, 0) < need)
                {
                    if (++spins > kWaitLimit)
                    {
                        atomicOr(errorWord, 1);
                        break;
                    }
                    __nanosleep(128);
                }
                __threadfence();
                s_item = spins > kWaitLimit ? -1 : w;
            }
            __syncthreads();
            if (s_item >= 0)
            {
                float ref = a.refMag;
                if (a.refMag == 0.f)
                {
                    const unsigned k = __ldcg(maxKey + b);
                    ref = k == 0u ? -FLT_MAX : fmaxf(-FLT_MAX, key_float(k));
                }
                const float inv = ref != 0.f ? __fdiv_rn(1.f, ref) : 1.0f;
                const int fd = threadIdx.x & (a.dbFrames - 1);   // dbFrames: power of two <= threads
                const int gd = threadIdx.x / a.dbFrames;
                const int kDbGroups = kFusedThreads / a.dbFrames;
                if (fd < Tv)
                {
                    // 8 rows per step: the loads (mostly L2 hits) are in flight together
                    constexpr int kRows = 8;
                    const size_t step = size_t(kDbGroups) * hs;
                    float* p = y + size_t(gd) * hs + fd;
                    int m = gd;
                    for (; m + (kRows - 1) * kDbGroups < nmel; m += kRows * kDbGroups, p += kRows * step)
                    {
                        float v[kRows];
#pragma unroll
                        for (int r = 0; r < kRows; ++r) v[r] = __ldcg(p + r * step);
#pragma unroll
                        for (int r = 0; r < kRows; ++r)
                        {
                            float t = __fmul_rn(v[r], inv);
                            t = a.minRatio < t ? t : a.minRatio;
                            p[r * step] = __fmul_rn(a.multiplier, log2f(t));
                        }
                    }
                    for (; m < nmel; m += kDbGroups, p += step)
                    {
                        float t = __fmul_rn(__ldcg(p), inv);
                        t = a.minRatio < t ? t : a.minRatio;
                        *p = __fmul_rn(a.multiplier, log2f(t));
                    }
                }
            }
        }
        __syncthreads();
    }
}

template <int NFFT, int TFX>
void launch_fused(Handle& h, const FrontendArgs& a, void* scratch)
{
    using S = StftShape<NFFT, kFusedThreads, TFX>;
    const int nslots = a.n + a.lookahead;
    Carver cv(scratch);
    long long* prefix = cv.take<long long>(nslots + 1);
    unsigned long long* counter = cv.take<unsigned long long>(1);
    int* done = cv.take<int>(a.n);
    unsigned* maxKey = cv.take<unsigned>(a.n);
    const size_t clear = reinterpret_cast<char*>(maxKey + a.n) - reinterpret_cast<char*>(counter);
    check_cuda(cudaMemsetAsync(counter, 0, clear, h.stream()), "memset(frontend state)");
    launch_ragged_prefix(SlotCount<S::TF>{a, a.n, a.lookahead}, nslots, prefix, h.stream());
    const FusedLayout<NFFT, TFX> lay(a.mel.numFilter, a.W, a.hop);
    if (lay.total > 227 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "numFilter too large for the fused tile");
    const float2* tw = spectrogram_twiddles(h, NFFT);
    int grid = persistent_grid(h, reinterpret_cast<const void*>(frontend_kernel<NFFT, TFX>), kFusedThreads, lay.total);
    if (a.ctasPerSm > 0) grid = std::min(grid, a.ctasPerSm * h.num_sms());
    if (a.reserveSms > 0 && a.reserveSms < h.num_sms())
        grid = std::max(1, grid / h.num_sms() * (h.num_sms() - a.reserveSms));
    frontend_kernel<NFFT, TFX><<<grid, kFusedThreads, lay.total, h.stream()>>>(a, tw, prefix, counter, done, maxKey,
                                                                          h.device_flags());
    count_launch();
    check_cuda(cudaGetLastError(), "frontend_kernel");
}

}  // namespace

size_t frontend_scratch_bytes(int n, int lookahead)
{
    Carver cv(nullptr);
    cv.take<long long>(n + lookahead + 1);
    cv.take<unsigned long long>(1);
    cv.take<int>(n);
    cv.take<unsigned>(n);
    return cv.used();
}

namespace {

// Tile frames: the plan's default or twice it (both bit-identical; the autotuner picks).
template <int NFFT>
void launch_nfft(Handle& h, const FrontendArgs& a, void* scratch)
{
    constexpr int T0 = Plan<NFFT>::TF;
    if (a.tileFrames == 0 || a.tileFrames == T0) launch_fused<NFFT, T0>(h, a, scratch);
    else if (a.tileFrames == 2 * T0) launch_fused<NFFT, 2 * T0>(h, a, scratch);
    else fail(RPP_ERROR_NOT_IMPLEMENTED, "tileFrames must be 0, " + std::to_string(T0) + " or " + std::to_string(2 * T0));
}

}  // namespace

void launch_frontend(Handle& h, void* scratch, const FrontendArgs& args)
{
    if (args.n <= 0) return;
    FrontendArgs a = args;
    if (a.dbFrames == 0) a.dbFrames = kDbFramesDefault;
    if (a.dbFrames < 16 || a.dbFrames > kFusedThreads || (a.dbFrames & (a.dbFrames - 1)))
        fail(RPP_ERROR_NOT_IMPLEMENTED, "dbFrames must be 0 or a power of two from 16 to 256");
    if (a.ctasPerSm < 0) fail(RPP_ERROR_INVALID_ARGUMENTS, "ctasPerSm must not be negative");
    switch (a.nfft)
    {
        case 128: launch_nfft<128>(h, a, scratch); return;
        case 256: launch_nfft<256>(h, a, scratch); return;
        case 512: launch_nfft<512>(h, a, scratch); return;
        case 1024: launch_nfft<1024>(h, a, scratch); return;
        case 2048: launch_nfft<2048>(h, a, scratch); return;
        default: fail(RPP_ERROR_NOT_IMPLEMENTED, "fused front end needs a power-of-two nfft from 128 to 2048");
    }
}

}  // namespace rppb
