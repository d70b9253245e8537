// Fused front end: pre-emphasis -> STFT power -> mel filter bank -> decibels in one persistent
// launch (include/rppb_frontend.h).
//
// Work items of two kinds walk one queue, claimed in order with an atomic counter:
//   spectrum tile (clip b, frames f0..f0+TF): gather the pre-emphasized, reflected, windowed
//     frames straight from the raw signal (stft.cuh, PreemphSource), FFT them into a shared
//     power tile, project onto the mel filters with one sweep over the bins per thread group
//     (same weights and the same ascending-bin float accumulation per filter as the
//     mel_filter_bank kernel), write the mel power into dst, fold the tile maximum into the
//     clip's float-ordered atomicMax, then count the tile done;
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
#include <cstring>
#include <string>

#include "common.cuh"
#include "fused_queue.cuh"
#include "mel_tables.cuh"
#include "ops.hpp"
#include "stft.cuh"

namespace rppb {
namespace {

template <int NFFT, int TFX>
__global__ void __launch_bounds__(kFusedThreads, (NFFT <= 512 ? 3 : 2)) frontend_kernel(FrontendArgs a, const float2* __restrict__ twiddle,
                                                                 const long long* __restrict__ prefix,
                                                                 unsigned long long* __restrict__ workCounter,
                                                                 int* __restrict__ done, unsigned* __restrict__ maxKey,
                                                                 int* __restrict__ errorWord,
                                                                 const uint4* __restrict__ melTables)
{
    using S = StftShape<NFFT, kFusedThreads, TFX>;
    constexpr int TF = S::TF, LD = S::OUT_LD;
    extern __shared__ __align__(16) unsigned char smem[];
    const FusedLayout<NFFT, TFX> lay(a.mel.numFilter, a.W, a.hop);
    float2* s_tw = reinterpret_cast<float2*>(smem + lay.tw);
    float2* s_tw1 = reinterpret_cast<float2*>(smem + lay.tw1);
    float* s_win = reinterpret_cast<float*>(smem + lay.win);
    float* s_span = reinterpret_cast<float*>(smem + lay.span);
    float2* s_fft = reinterpret_cast<float2*>(smem + lay.work);
    float* s_out = reinterpret_cast<float*>(smem + lay.work + S::fft_bytes);
    float2* melW = reinterpret_cast<float2*>(smem + lay.melW);   // bin k: (weight into filter i, into filter i - 1)
    int2* melIv = reinterpret_cast<int2*>(smem + lay.melIv);     // interval i: bins [x, y)
    int* melGrp = reinterpret_cast<int*>(smem + lay.melGrp);     // thread group g: filters [g], [g + 1])
    __shared__ float s_warpMax[kFusedThreads / 32];
    const int nmel = a.mel.numFilter;

    // The per-CTA setup (tables below) runs in a loop whose trip count, always one, the compiler
    // cannot prove: the setup's registers are then allocated apart from the work loop's, which keeps
    // the work loop free of spills at the 80-register cap (ptxas, nfft 512: 0 bytes of spill stores
    // instead of 48; 263 -> 253 us on the 256-clip batch, bit-identical).
    for (int setupPass = 0, setupPasses = 1 + (a.n < 0); setupPass < setupPasses; ++setupPass)
    {
        stft_tables<NFFT, kFusedThreads>(twiddle, a.window, a.W, s_tw, s_tw1, s_win, s_span);

        // the mel tables: copied from the handle's cache when the launch has them, else built here
        if (melTables)
        {
            uint4* t = reinterpret_cast<uint4*>(smem + lay.melW);
            for (int i = threadIdx.x; i < int((lay.total - lay.melW) / 16); i += kFusedThreads) t[i] = __ldg(RPPB_RD(melTables + i));
            __syncthreads();
        }
        else
            build_fused_mel<NFFT, TFX>(a, smem, lay);
    }

    const int centerOffset = a.center ? a.W / 2 : 0;
    const int nslots = a.n + a.lookahead;
    __shared__ long long s_prefix[kFusedPrefixCache];
    grid_dependency_wait();   // the prefix and the zeroed counters of the prefix kernel
    prefix = cache_prefix<kFusedPrefixCache>(prefix, nslots, s_prefix);
    const long long total = prefix[nslots];
    const SlotCount<TF> cnt{a, a.n, a.lookahead};
    const int f = 2 * (threadIdx.x % (TF / 2));   // first of the two frame columns this thread owns in mel tiles
    const int g = threadIdx.x / (TF / 2);

    // Thread 0 keeps two items decoded ahead in a two-entry ring (the claim's and the decode's
    // latencies overlap the current item) and asks L2 for each decoded spectrum item's input span
    // one item before it is staged; in the last 2 x grid items of the queue it reserves nothing
    // beyond the next item and claims each one when it decodes it.  A CTA's current item always has
    // a lower index than the ones it holds claimed, so the lowest unfinished item is always some
    // CTA's current one, whose decibel wait (on lower spectrum items only) ends: claiming ahead
    // keeps the waits deadlock-free.
    __shared__ Item s_it[2];
    __shared__ int s_ok;
    const int itemFrames = TF * a.subTiles;
    auto prefetch_span = [&](const Item& n) {
        if (n.kind != 0) return;
        const int last = min(n.f0 + itemFrames, n.F) - 1;
        const long long s0 = max(0ll, (long long)n.f0 * a.hop - centerOffset);
        const long long s1 = min((long long)n.L, (long long)last * a.hop - centerOffset + a.W);
        l2_prefetch(n.x + s0, n.x + s1);
    };
    long long wAfter = 0;   // thread 0: the claimed item two after the current one (-1: none reserved)
    int cur = 0;
    if (threadIdx.x == 0)
    {
        const long long w0 = (long long)atomicAdd(RPPB_WR(workCounter), 1ull);
        const long long w1 = (long long)atomicAdd(RPPB_WR(workCounter), 1ull);
        wAfter = w1 < total - 2ll * gridDim.x ? (long long)atomicAdd(RPPB_WR(workCounter), 1ull) : -1ll;
        s_it[0] = decode_item<TF>(a, cnt, prefix, nslots, total, w0);
        s_it[1] = decode_item<TF>(a, cnt, prefix, nslots, total, w1);
        prefetch_span(s_it[1]);
    }
    __syncthreads();
    for (;;)
    {
        // s_it[cur] is rewritten only after the barrier that ends this item's work
        const Item it = s_it[cur];
        if (it.kind < 0) break;
        const int b = it.b;
        const uint32_t hs = it.hs;

        if (it.kind == 0)
        {
            // subTiles tiles of TF frames; each tile's staging barrier also orders the previous
            // tile's mel reads of s_out before this tile's FFT overwrites it
            const PreemphSource src{it.x, it.L, a.reflect, it.coeff, it.bval};
            float tmax = -FLT_MAX;
            for (int t = 0; t < a.subTiles; ++t)
            {
                const int f0 = it.f0 + t * TF;
                if (f0 >= it.F) break;   // uniform over the CTA
                stft_tile<NFFT, kFusedThreads, TFX>(src, f0, it.F, a.W, a.hop, centerOffset, a.power, s_win, s_tw,
                                                    s_tw1, s_span, s_fft, s_out);
                __syncthreads();
                if (f < it.F - f0)
                {
                    // one sweep over the group's intervals for frames f and f + 1; each power
                    // pair is read once.  Scalar __fmul_rn / __fadd_rn: a paired multiply feeding
                    // a paired add may be contracted into one rounding by the assembler.
                    const bool second = f + 1 < it.F - f0;
                    const int m0 = melGrp[g], m1 = melGrp[g + 1];
                    float* yp = it.y + size_t(f0 - it.f0) + size_t(m0) * hs + f;
                    float2 fall = make_float2(0.f, 0.f);   // filter i - 1: rising sum, then falling terms
                    for (int i = m0; i <= m1; ++i)
                    {
                        const int2 iv = melIv[i];
                        const float* sp = s_out + iv.x * LD + f;
                        float2 rise = make_float2(0.f, 0.f);   // filter i
#pragma unroll 1
                        for (int k = iv.x; k < iv.y; ++k, sp += LD)
                        {
                            const float2 pw = *reinterpret_cast<const float2*>(sp);
                            const float2 w = melW[k];
                            fall.x = __fadd_rn(fall.x, __fmul_rn(pw.x, w.y));
                            fall.y = __fadd_rn(fall.y, __fmul_rn(pw.y, w.y));
                            rise.x = __fadd_rn(rise.x, __fmul_rn(pw.x, w.x));
                            rise.y = __fadd_rn(rise.y, __fmul_rn(pw.y, w.x));
                        }
                        if (i > m0)
                        {
                            *RPPB_WR(yp) = fall.x;
                            tmax = fmaxf(tmax, fall.x);
                            if (second)
                            {
                                *RPPB_WR(yp + 1) = fall.y;
                                tmax = fmaxf(tmax, fall.y);
                            }
                            yp += hs;
                        }
                        fall = rise;
                    }
                }
            }
            tmax = warp_max(tmax);
            if ((threadIdx.x & 31) == 0) s_warpMax[threadIdx.x >> 5] = tmax;
        }
        else
        {
            if (threadIdx.x == 0)
            {
                const int need = cnt.tiles(b) + a.waitExtra;
                const long long limit = a.waitLimit > 0 ? a.waitLimit : kWaitLimit;
                long long spins = 0;
                while (atomicAdd(RPPB_WR(done + b), 0) < need)
                {
                    if (++spins > limit)
                    {
                        atomicOr(RPPB_WR(errorWord), 1);
                        break;
                    }
                    __nanosleep(128);
                }
                __threadfence();
                s_ok = spins <= limit;
            }
            __syncthreads();
            if (s_ok)
            {
                float ref = a.refMag;
                if (a.refMag == 0.f)
                {
                    const unsigned k = __ldcg(RPPB_RD(maxKey + b));
                    ref = k == 0u ? -FLT_MAX : fmaxf(-FLT_MAX, key_float(k));
                }
                const float inv = ref != 0.f ? __fdiv_rn(1.f, ref) : 1.0f;
                const int fd = threadIdx.x & (a.dbFrames - 1);   // dbFrames: power of two <= threads
                const int gd = threadIdx.x / a.dbFrames;
                const int kDbGroups = kFusedThreads / a.dbFrames;
                if (fd < it.Tv)
                {
                    // 16 rows per step: the loads (mostly L2 hits) are in flight together (8: 1 % slower)
                    constexpr int kRows = 16;
                    const size_t step = size_t(kDbGroups) * hs;
                    float* p = it.y + size_t(gd) * hs + fd;
                    int m = gd;
                    for (; m + (kRows - 1) * kDbGroups < nmel; m += kRows * kDbGroups, p += kRows * step)
                    {
                        float v[kRows];
#pragma unroll
                        for (int r = 0; r < kRows; ++r) v[r] = __ldcg(RPPB_RD(p + r * step));
#pragma unroll
                        for (int r = 0; r < kRows; ++r)
                        {
                            float t = __fmul_rn(v[r], inv);
                            t = a.minRatio < t ? t : a.minRatio;
                            *RPPB_WR(p + r * step) = __fmul_rn(a.multiplier, __log2f(t));
                        }
                    }
                    for (; m < nmel; m += kDbGroups, p += step)
                    {
                        float t = __fmul_rn(__ldcg(RPPB_RD(p)), inv);
                        t = a.minRatio < t ? t : a.minRatio;
                        *RPPB_WR(p) = __fmul_rn(a.multiplier, __log2f(t));
                    }
                }
            }
        }
        __syncthreads();
        // after the item's last barrier, in parallel with the other warps starting the next item:
        // warp 0 claims and decodes the item after next into the slot just read (no thread reads
        // that slot again before the next item's end barrier); warp 1 publishes a finished
        // spectrum item.  No second barrier: the next item was decoded one item earlier, and the
        // shared values written here (s_it[cur]) or read here (s_warpMax) are next touched by the
        // other threads only after a later barrier that warps 0 and 1 also reach.
        if (threadIdx.x == 0)
        {
            // the last 2 x grid items are claimed when needed, not reserved ahead, so that no CTA
            // holds work that an idle one could start (small batches: 0.039 -> 0.033 ms for one 1 s clip)
            const long long w = wAfter >= 0 ? wAfter : (long long)atomicAdd(RPPB_WR(workCounter), 1ull);
            wAfter = w < total - 2ll * gridDim.x ? (long long)atomicAdd(RPPB_WR(workCounter), 1ull) : -1ll;
            const Item nx = decode_item<TF>(a, cnt, prefix, nslots, total, w);
            prefetch_span(nx);
            s_it[cur] = nx;
        }
        else if (threadIdx.x == 32 && it.kind == 0)
        {
            // the barrier orders every thread's mel stores before this thread's release, which
            // orders them (and the maximum) before the count
            float v = s_warpMax[0];
            for (int i = 1; i < kFusedThreads / 32; ++i) v = fmaxf(v, s_warpMax[i]);
            atomicMax(RPPB_WR(maxKey + b), float_key(v));
            asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(RPPB_WR(done + b)) : "memory");
        }
        cur ^= 1;
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
    const FusedLayout<NFFT, TFX> lay(a.mel.numFilter, a.W, a.hop);
    if (lay.total > 227 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "numFilter too large for the fused tile");
    const float2* tw = spectrogram_twiddles(h, NFFT);
    // the mel tables, built once per handle, mel parameters and tile (not while the stream is being
    // captured: then each CTA builds them)
    uint4* melTables = fused_mel_table_cache<NFFT, TFX>(h, a);
    // the prefix kernel also zeroes the queue counter, the tile counts and the maxima
    const size_t clear = reinterpret_cast<char*>(maxKey + a.n) - reinterpret_cast<char*>(counter);
    launch_ragged_prefix(SlotCount<S::TF>{a, a.n, a.lookahead}, nslots, prefix, h.stream(),
                         reinterpret_cast<unsigned*>(counter), int(clear / 4));
    int grid = persistent_grid(h, reinterpret_cast<const void*>(frontend_kernel<NFFT, TFX>), kFusedThreads, lay.total);
    if (a.ctasPerSm > 0) grid = std::min(grid, a.ctasPerSm * h.num_sms());
    if (a.reserveSms > 0 && a.reserveSms < h.num_sms())
        grid = std::max(1, grid / h.num_sms() * (h.num_sms() - a.reserveSms));
    // starts while the prefix kernel runs: the tables are built before grid_dependency_wait()
    launch_dependent(frontend_kernel<NFFT, TFX>, dim3(grid), dim3(kFusedThreads), lay.total, h.stream(),
                     "frontend_kernel", a, tw, static_cast<const long long*>(prefix), counter, done, maxKey,
                     h.device_flags(), static_cast<const uint4*>(melTables));
    count_launch();
}

}  // namespace

size_t frontend_scratch_bytes(int n, int lookahead, int numFilter)
{
    Carver cv(nullptr);
    cv.take<long long>(n + lookahead + 1);
    cv.take<unsigned long long>(1);
    cv.take<int>(n);
    cv.take<unsigned>(n);
    cv.take<char>(fused_mel_table_bytes_512(numFilter, 512, 1));   // the tensor-core engine's mel tables
    return cv.used();
}

namespace {

// Frames per spectrum item: the plan's tile (default) or 2 or 4 of them, computed one tile after
// another (all bit-identical; the autotuner picks).
template <int NFFT>
void launch_nfft(Handle& h, const FrontendArgs& args, void* scratch)
{
    constexpr int T0 = Plan<NFFT>::TF;
    FrontendArgs a = args;
    a.subTiles = a.tileFrames == 0 ? kSubTilesDefault : a.tileFrames / T0;
    if (a.tileFrames != 0 && (a.tileFrames % T0 != 0 || (a.subTiles != 1 && a.subTiles != 2 && a.subTiles != 4)))
        fail(RPP_ERROR_NOT_IMPLEMENTED, "tileFrames must be 0 or 1, 2 or 4 times " + std::to_string(T0));
    launch_fused<NFFT, T0>(h, a, scratch);
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
    // wait fault injection (test only): every decibel item waits for a tile that is never counted
    a.waitExtra = h.wait_injection() ? 1 : 0;
    a.waitLimit = h.wait_injection() ? kInjectedWaitLimit : 0;
    if (a.engine == 1)
    {
        // the factored DFT on tensor cores: nfft 512, tiles of 16 frames, 1, 2 or 4 per spectrum item
        if (!frontend_tc_supported(a))
            fail(RPP_ERROR_NOT_IMPLEMENTED, "the tensor-core spectrum engine needs nfft 512 and windowLength <= 512");
        a.subTiles = a.tileFrames == 0 ? kSubTilesDefault : a.tileFrames / 16;
        if (a.tileFrames != 0 && (a.tileFrames % 16 != 0 || (a.subTiles != 1 && a.subTiles != 2 && a.subTiles != 4)))
            fail(RPP_ERROR_NOT_IMPLEMENTED, "tileFrames must be 0, 16, 32 or 64");
        Carver cv(scratch);
        cv.take<long long>(a.n + a.lookahead + 1);
        cv.take<unsigned long long>(1);
        cv.take<int>(a.n);
        cv.take<unsigned>(a.n);
        uint4* melScratch = cv.take<uint4>(fused_mel_table_bytes_512(a.mel.numFilter, a.W, a.hop) / 16);
        launch_frontend_tc(h, a, scratch, melScratch);
        return;
    }
    if (a.engine != 0) fail(RPP_ERROR_INVALID_ARGUMENTS, "spectrumEngine must be 0 or 1");
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
