// Fused front end on tensor cores: pre-emphasis -> STFT power -> mel filter bank -> decibels in one
// persistent launch, with the spectrum of each tile of 16 frames computed as a factored DFT on the
// 5th-generation tensor cores (tcgen05) in F16 hi/lo x3 with FP32 accumulation.  Same work queue,
// mel sums and decibel items as the FP32 fused kernel (fused_queue.cuh, fused.cu); only the
// spectrum engine differs, so the outputs carry the factored DFT's rounding instead of matching the
// plain calls bit for bit.
//
// The 512-point real DFT of a windowed frame x (n = n1 + 16 n2, k = 32 k1 + k2; n1, k1 < 16,
// n2, k2 < 32) factors as
//   Y[n1][k2]  = sum_n2 x[n1 + 16 n2] W32^(n2 k2)                 (stage 1: 16 real 32-point DFTs)
//   Y'[n1][k2] = Y[n1][k2] W512^(n1 k2)                            (twiddle, FP32 on the CUDA cores)
//   X[32 k1 + k2] = sum_n1 Y'[n1][k2] W16^(n1 k1)                  (stage 2: 17 complex 16-point DFTs)
// with k2 <= 16 only (x is real, so Y[n1][32 - k2] = conj Y[n1][k2]); the bins above 256 fold onto
// the conjugate ones, and bins k2 in 17..31 come from k2' = 32 - k2, k1' = 15 - k1.  Both stages are
// GEMMs of M = 128 rows x N = 32 columns x K = 32 on the tensor cores:
//   stage 1, for j = 0, 1: A1_j row (f, q) = x_f[8 j + q + 16 n2] (n2 = K), 16 frames x 8 phases;
//           B1 = the real 32-point DFT basis, columns (Re k2=0, Re k2=16, Re k2, Im k2 for k2 = 1..15);
//   stage 2, for i = 0, 1, 2: A2_i row (f, q') = the twiddled Y'[.][k2 = 8 i + q'] over K = (q, j, re/im)
//           (i = 2 holds k2 = 16 in rows q' = 0); B2 = the complex 16-point DFT basis as a real 32 x 32.
// Each frame is scaled by a power of two so that its largest windowed sample lies in [0.5, 1) (then
// |Y| <= 32, inside the F16 range at both stages; the power is scaled back at the end).  Each operand
// is split x = hi + lo into two F16 values (hi + lo holds x to ~2^-22 of the frame's scale) and the
// products hi*hi + hi*lo + lo*hi are accumulated in FP32 in tensor memory (6 MMAs of K = 16 per 32 of
// K), so the spectrum stays within ~1e-6 of each frame's largest bin against FP64.  The operand tiles
// (128 rows x 128 bytes: 32 F16 of hi then 32 of lo per row) use the 128-byte-swizzled K-major layout;
// A2 reuses A1's shared memory.
//
// Per tile: stage the span (CUDA cores) -> build A1 -> one thread issues 12 MMAs and commits to an
// mbarrier -> epilogue 1 reads the stage-1 accumulators (tcgen05.ld), twiddles and splits them into A2
// -> 18 MMAs -> epilogue 2 reads the bins and writes the power tile -> the mel sums of the FP32 kernel.
// Every mbarrier wait is bounded: on a timeout the kernel sets bit 4 of the handle's device error word,
// waits once more (bounded) for its MMAs in flight, frees its tensor memory and leaves.
#include <cuda_fp16.h>

#include <map>
#include <mutex>
#include <set>

#include "fused_queue.cuh"
#include "tcgen05.cuh"

namespace rppb {
namespace {

constexpr int kTcNfft = 512;
constexpr int kTcTF = 16;                         // frames per tile
constexpr uint32_t kTcTile = 128 * 128;           // one operand tile: 128 rows x 128 bytes
constexpr uint32_t kTcABytes = 3 * kTcTile;       // A1 (tiles 0-1) and A2 (tiles 0-2), aliased
constexpr uint32_t kTcBBytes = 32 * 128;          // one 32-row basis tile
constexpr int kTcTmemCols = 256;
constexpr uint32_t kTcD1 = 0, kTcD2 = 64;         // tensor-memory columns of the accumulators
constexpr uint32_t kTcIdesc = tc::idesc_f16(128, 32);
constexpr long long kTcWaitLimit = 1ll << 21;     // mbarrier polls before a tensor-core wait gives up

// Stage-1 K order: index kk < 16 holds n2 = 2 kk, kk >= 16 holds n2 = 2 (kk - 16) + 1.
__host__ __device__ constexpr int s1_n2(int kk) { return kk < 16 ? 2 * kk : 2 * (kk - 16) + 1; }

// Row of the stage-2 operand for frame f (of 16) within the 16-row block of its k2: a permutation
// that puts frames f and f + 1 four rows apart inside their 8-row swizzle atom, so the epilogue's
// 8-byte stores of two frames land in disjoint bank groups.
__host__ __device__ constexpr int s2_row(int f) { return 8 * (f >> 3) + 4 * (f & 1) + ((f >> 1) & 3); }
__host__ __device__ constexpr int s2_frame(int r) { return 8 * (r >> 3) + 2 * (r & 3) + ((r >> 2) & 1); }

// Shared memory plan (bytes from a 1024-byte aligned base).
struct TcLayout
{
    size_t a, b1, b2, w512, scale, win, span, out, mel, melIv, melGrp, total, melBytes;
    __host__ __device__ TcLayout(int numFilter, int W, int hop)
    {
        using S = StftShape<kTcNfft, kFusedThreads, kTcTF>;
        const FusedLayout<kTcNfft, kTcTF> f(numFilter, W, hop);
        a = 0;
        b1 = a + kTcABytes;
        b2 = b1 + kTcBBytes;
        w512 = b2 + kTcBBytes;
        scale = w512 + 16 * 17 * 8;
        win = scale + kTcTF * 4;
        span = win + size_t(kTcNfft) * 4;
        out = (span + S::span_bytes(W, hop) + 15) & ~size_t(15);
        mel = (out + S::out_bytes + 15) & ~size_t(15);
        // the mel tables keep the FP32 kernel's relative layout (same cached table block)
        melBytes = f.total - f.melW;
        melIv = mel + (f.melIv - f.melW);
        melGrp = mel + (f.melGrp - f.melW);
        total = mel + melBytes;
    }
};

// Per-CTA constant tables: the two F16 hi/lo bases in the swizzled layout and the twiddles
// W512^(n1 k2) as [n1][k2] (n1 < 16, k2 <= 16).
// twiddle[e] = (cos, sin)(2 pi e / 512), so W512^e = x - i y.
__device__ __forceinline__ void tc_tables(const float2* __restrict__ twiddle, unsigned char* b1, unsigned char* b2,
                                          float2* w512)
{
    auto put = [](unsigned char* t, int row, int k, float v) {
        const __half hi = __float2half_rn(v);
        const __half lo = __float2half_rn(v - __half2float(hi));
        *reinterpret_cast<__half*>(t + tc::sw128(row, 2 * k)) = hi;
        *reinterpret_cast<__half*>(t + tc::sw128(row, 64 + 2 * k)) = lo;
    };
    for (int i = threadIdx.x; i < 32 * 32; i += kFusedThreads)
    {
        // B1 row c, K index kk (n2 = s1_n2(kk)): Re k2 = 0, Re k2 = 16, then (Re, Im) of W32^(n2 k2) for
        // k2 = 1..15
        const int c = i >> 5, kk = i & 31, n2 = s1_n2(kk);
        float v;
        if (c == 0) v = 1.f;
        else if (c == 1) v = (n2 & 1) ? -1.f : 1.f;
        else
        {
            const float2 w = twiddle[(16 * (c >> 1) * n2) & (kTcNfft - 1)];
            v = (c & 1) ? -w.y : w.x;
        }
        put(b1, c, kk, v);
        // B2 row c = 2 k1 + (0: Re X, 1: Im X), K = 4 q + 2 j + (0: Re Y', 1: Im Y') with n1 = 8 j + q:
        // X = sum Y' W16^(n1 k1), W = wc + i ws, wc = cos, ws = -sin
        const int r2 = i >> 5, K = i & 31;
        const int k1 = r2 >> 1, reX = (r2 & 1) == 0, q = K >> 2, j = (K >> 1) & 1, reY = (K & 1) == 0;
        const float2 w = twiddle[(32 * (8 * j + q) * k1) & (kTcNfft - 1)];
        const float wc = w.x, ws = -w.y;
        float u;
        if (reX) u = reY ? wc : -ws;
        else u = reY ? ws : wc;
        put(b2, r2, K, u);
    }
    // the twiddles of epilogue 1 by (n1, k2): W512^(n1 k2), 17 per n1
    for (int e = threadIdx.x; e < 16 * 17; e += kFusedThreads) w512[e] = *RPPB_RD(twiddle + (e / 17) * (e % 17));
}

// Stage-1 operand: A1_j row (f, q) = q + 8 f, K index kk (hi 0..31 | lo 0..31) holding n2 = s1_n2(kk), value
// = window * sample of buffer position n = 8 j + q + 16 n2 of tile frame f (zero for frames past the
// tile's valid ones).  Lane l of warp w takes n1 = l % 16 and the 16 n2 of parity h = l / 16 of frame
// 8 p + w (p = pass), so the 32 lanes read 32 consecutive buffer samples, and writes them as K indices
// 16 h .. 16 h + 15: the even n2 first, then the odd ones (B1 uses the same order).
__device__ __forceinline__ void tc_build_a1(unsigned char* A, const float* __restrict__ s_data,
                                            const float* __restrict__ s_win, int hop, int off, int Tv,
                                            float* __restrict__ s_scale)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n1 = lane & 15, h = lane >> 4;
    const int q = n1 & 7, j = n1 >> 3;
#pragma unroll 1
    for (int p = 0; p < 2; ++p)
    {
        const int f = 8 * p + warp;
        float v[16];
        if (f < Tv)
        {
            const float* fs = s_data + f * hop - off;
#pragma unroll
            for (int m = 0; m < 16; ++m)
            {
                const int n = n1 + 16 * h + 32 * m;
                v[m] = __fmul_rn(s_win[n], fs[n]);
            }
        }
        else
        {
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = 0.f;
        }
        // the warp holds the whole frame: scale it by a power of two so its largest |value| lies in
        // [0.5, 1) (F16 range for both stages: |Y| <= 32); the power is scaled back in epilogue 2
        float m = 0.f;
#pragma unroll
        for (int i = 0; i < 16; ++i) m = fmaxf(m, fabsf(v[i]));
        m = warp_max(m);
        int ex = int((__float_as_uint(m) >> 23) & 0xFFu) - 126;   // m = [0.5, 1) * 2^ex for normal m
        ex = m > 0.f ? min(max(ex, -120), 120) : -120;
        const float sc = __uint_as_float(uint32_t(127 - ex) << 23);
        if (lane == 0) s_scale[f] = __uint_as_float(uint32_t(127 + ex) << 23);
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) tc::split_f16x2(v[2 * i] * sc, v[2 * i + 1] * sc, hi[i], lo[i]);
        unsigned char* t = A + j * kTcTile;
        const int r = q + 8 * f;
        *reinterpret_cast<uint4*>(t + tc::sw128(r, 32 * h)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(t + tc::sw128(r, 32 * h + 16)) = make_uint4(hi[4], hi[5], hi[6], hi[7]);
        *reinterpret_cast<uint4*>(t + tc::sw128(r, 64 + 32 * h)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        *reinterpret_cast<uint4*>(t + tc::sw128(r, 80 + 32 * h)) = make_uint4(lo[4], lo[5], lo[6], lo[7]);
    }
}

// Epilogue 1: the stage-1 accumulators of this thread's row (f, q) for j = 0, 1 -> twiddled Y'[n1][k2]
// for k2 in [K0, K1) -> A2 rows (f, k2 % 8) of tile k2 / 8 at K = 4 q + 2 j + (re, im).
// The first half (k2 = 0..8) needs accumulator columns 0 and 2..17, the second (k2 = 9..16) columns 1
// and 18..31: each loads 16 + 2 columns per j into d[c] at the column's own index.
template <int K0, int K1>
__device__ __forceinline__ void tc_epilogue1(unsigned char* A, uint32_t tmem, const float2* __restrict__ w512)
{
    const int lane = threadIdx.x & 31, quarter = (threadIdx.x >> 5) & 3;
    const int r = 32 * quarter + lane;
    const int q = r & 7, f = r >> 3;
    constexpr int C16 = K0 == 0 ? 0 : 16, C2 = K0 == 0 ? 16 : 0;   // columns of the x16 and the x2 load
    uint32_t d0[32], d1[32];
    const uint32_t t = tmem + (uint32_t(32 * quarter) << 16) + kTcD1;
    tc::tmem_ld16(t + C16, d0 + C16);
    tc::tmem_ld2(t + C2, d0 + C2);
    tc::tmem_ld16(t + 32 + C16, d1 + C16);
    tc::tmem_ld2(t + 32 + C2, d1 + C2);
    tc::tmem_ld_wait();
    const int sr = s2_row(f);
    const uint32_t offHi = tc::sw128(sr, 8 * q), offLo = tc::sw128(sr, 64 + 8 * q);
#pragma unroll
    for (int k2 = K0; k2 < K1; ++k2)
    {
        const int cRe = k2 == 0 ? 0 : k2 == 16 ? 1 : 2 * k2;
        float y[2][2];
#pragma unroll
        for (int jj = 0; jj < 2; ++jj)
        {
            const uint32_t* d = jj ? d1 : d0;
            const float yr = __uint_as_float(d[cRe]);
            const float yi = (k2 == 0 || k2 == 16) ? 0.f : __uint_as_float(d[2 * k2 + 1]);
            if (k2 == 0)
            {
                y[jj][0] = yr;
                y[jj][1] = 0.f;
            }
            else
            {
                // Y * W512^(n1 k2), W = c - i s
                const float2 t = w512[(8 * jj + q) * 17 + k2];
                y[jj][0] = fmaf(yr, t.x, yi * t.y);
                y[jj][1] = fmaf(yi, t.x, -yr * t.y);
            }
        }
        uint32_t h0, l0, h1, l1;
        tc::split_f16x2(y[0][0], y[0][1], h0, l0);
        tc::split_f16x2(y[1][0], y[1][1], h1, l1);
        *reinterpret_cast<uint2*>(A + 2048 * k2 + offHi) = make_uint2(h0, h1);
        *reinterpret_cast<uint2*>(A + 2048 * k2 + offLo) = make_uint2(l0, l1);
    }
}

// Epilogue 2: stage-2 accumulator i of this thread's row (f, q') holds X[32 k1 + k2], k2 = 8 i + q',
// k1 = 0..15; the needed bins (<= 256) go to the power tile.
template <bool MAGNITUDE>
__device__ __forceinline__ void tc_epilogue2(uint32_t tmem, int i, float* __restrict__ s_out,
                                             const float* __restrict__ s_scale)
{
    constexpr int LD = StftShape<kTcNfft, kFusedThreads, kTcTF>::OUT_LD;
    const int lane = threadIdx.x & 31, quarter = (threadIdx.x >> 5) & 3;
    const int r = 32 * quarter + lane;
    const int qp = r >> 4, f = s2_frame(r & 15);
    const int k2 = 8 * i + qp;
    uint32_t v[32];
    tc::tmem_ld32(tmem + (uint32_t(32 * quarter) << 16) + kTcD2 + 32 * i, v);
    tc::tmem_ld_wait();
    if (i == 2 && qp != 0) return;   // tile 2 holds k2 = 16 in rows q' = 0 only
    const float u = s_scale[f];      // the frame's scale: X = u * (the accumulator)
    float* lo = s_out + k2 * LD + f;                 // bins 32 k1 + k2
    float* hi = s_out + (kTcNfft - k2) * LD + f;     // bins 512 - 32 k1 - k2
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1)
    {
        const float re = __uint_as_float(v[2 * k1]), im = __uint_as_float(v[2 * k1 + 1]);
        float p = fmaf(re, re, im * im);
        p = MAGNITUDE ? sqrtf(p) * u : p * (u * u);
        if (k1 < 8) lo[32 * k1 * LD] = p;
        else if (k2 == 0 && k1 == 8) lo[32 * 8 * LD] = p;   // bin 256
        else if (k2 != 0 && k2 != 16) hi[-32 * k1 * LD] = p;
    }
}

template <int TFX>
__global__ void __launch_bounds__(kFusedThreads, 2)
    frontend_tc_kernel(FrontendArgs a, const float2* __restrict__ twiddle, const long long* __restrict__ prefix,
                       unsigned long long* __restrict__ workCounter, int* __restrict__ done,
                       unsigned* __restrict__ maxKey, int* __restrict__ errorWord, const uint4* __restrict__ melTables)
{
    static_assert(TFX == kTcTF, "the tensor-core engine works on tiles of 16 frames");
    using S = StftShape<kTcNfft, kFusedThreads, TFX>;
    constexpr int TF = S::TF, LD = S::OUT_LD;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const TcLayout lay(a.mel.numFilter, a.W, a.hop);
    unsigned char* sA = smem + lay.a;
    unsigned char* sB1 = smem + lay.b1;
    unsigned char* sB2 = smem + lay.b2;
    float2* s_w512 = reinterpret_cast<float2*>(smem + lay.w512);
    float* s_scale = reinterpret_cast<float*>(smem + lay.scale);
    float* s_win = reinterpret_cast<float*>(smem + lay.win);
    float* s_span = reinterpret_cast<float*>(smem + lay.span);
    float* s_out = reinterpret_cast<float*>(smem + lay.out);
    float2* melW = reinterpret_cast<float2*>(smem + lay.mel);
    int2* melIv = reinterpret_cast<int2*>(smem + lay.melIv);
    int* melGrp = reinterpret_cast<int*>(smem + lay.melGrp);
    __shared__ float s_warpMax[kFusedThreads / 32];
    __shared__ uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int nmel = a.mel.numFilter;

    // ---- setup (before the grid-dependency wait: overlaps the prefix kernel)
    if (threadIdx.x < 32) tc::tmem_alloc<kTcTmemCols>(&s_tmem);
    if (threadIdx.x == 0)
    {
        tc::mbar_init(&s_bar, 1);
        tc::fence_mbar_init();
    }
    tc_tables(twiddle, sB1, sB2, s_w512);
    {
        const int off = S::window_offset(a.W);
        for (int i = threadIdx.x; i < kTcNfft; i += kFusedThreads)
            s_win[i] = (i >= off && i - off < a.W) ? a.window[i - off] : 0.f;
        for (int i = threadIdx.x; i < S::span_pad(a.W); i += kFusedThreads) s_span[i] = 0.f;
        uint4* t = reinterpret_cast<uint4*>(smem + lay.mel);
        for (int i = threadIdx.x; i < int(lay.melBytes / 16); i += kFusedThreads) t[i] = __ldg(RPPB_RD(melTables + i));
    }
    tc::fence_async_smem();   // the bases are read by the tensor core
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = s_tmem;
    uint32_t phase = 0;       // parity of the next mbarrier phase to wait for
    int pending = 0;          // commits not yet waited for (0 or 1)
    bool abort = false;

    const int centerOffset = a.center ? a.W / 2 : 0;
    const int off = S::window_offset(a.W);
    const int nslots = a.n + a.lookahead;
    __shared__ long long s_prefix[kFusedPrefixCache];
    grid_dependency_wait();   // the prefix and the zeroed counters of the prefix kernel
    prefix = cache_prefix<kFusedPrefixCache>(prefix, nslots, s_prefix);
    const long long total = prefix[nslots];
    const SlotCount<TF> cnt{a, a.n, a.lookahead};
    const int fcol = 2 * (threadIdx.x % (TF / 2));   // first of the two frame columns this thread owns in mel tiles
    const int g = threadIdx.x / (TF / 2);

    // one bounded wait for the MMAs committed last: thread 0 polls the mbarrier (the others wait at the
    // barrier, issuing nothing), and the barrier hands its observation of the MMAs' completion to every
    // thread, each of which then orders its tensor-memory reads after it (fence::after_thread_sync)
    auto wait_mma = [&]() -> bool {
        bool ok = true;
        if (threadIdx.x == 0) ok = tc::mbar_wait(&s_bar, phase, kTcWaitLimit);
        const bool bad = __syncthreads_or(!ok);
        if (!bad)
        {
            phase ^= 1u;
            pending = 0;
        }
        tc::fence_after();
        if (bad && threadIdx.x == 0) atomicOr(RPPB_WR(errorWord), 4);
        return !bad;
    };

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
    long long wAfter = 0;
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
        const Item it = s_it[cur];
        if (it.kind < 0) break;
        const int b = it.b;
        const uint32_t hs = it.hs;

        if (it.kind == 0)
        {
            const PreemphSource src{it.x, it.L, a.reflect, it.coeff, it.bval};
            float tmax = -FLT_MAX;
            for (int t = 0; t < a.subTiles && !abort; ++t)
            {
                const int f0 = it.f0 + t * TF;
                if (f0 >= it.F) break;   // uniform over the CTA
                const int Tv = min(TF, it.F - f0);
                // span -> stage-1 operand (the span barrier also ends the previous tile's mel reads)
                stft_stage_span<kTcNfft, kFusedThreads, TFX>(src, f0, it.F, a.W, a.hop, centerOffset, s_span);
                tc_build_a1(sA, s_span + S::span_pad(a.W), s_win, a.hop, off, Tv, s_scale);
                tc::fence_async_smem();
                __syncthreads();
                if (threadIdx.x == 0)
                {
                    tc::fence_after();
                    const uint64_t dB = tc::desc_sw128(tc::smem_addr(sB1));
#pragma unroll
                    for (int j = 0; j < 2; ++j)
                    {
                        const uint64_t dA = tc::desc_sw128(tc::smem_addr(sA + j * kTcTile));
                        const uint32_t d = tmem + kTcD1 + 32 * j;
                        // K steps of 32 bytes: hi at +0, +32; lo at +64, +96 (descriptor units of 16 bytes)
                        tc::mma_f16(d, dA + 0, dB + 0, kTcIdesc, 0u);
                        tc::mma_f16(d, dA + 2, dB + 2, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 0, dB + 4, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 2, dB + 6, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 4, dB + 0, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 6, dB + 2, kTcIdesc, 1u);
                    }
                    tc::commit(&s_bar);
                }
                pending = 1;
                if (!wait_mma())
                {
                    abort = true;
                    break;
                }
                // epilogue 1: warps 0-3 take k2 = 0..8, warps 4-7 k2 = 9..16 (A2 overwrites A1)
                if (threadIdx.x < 128) tc_epilogue1<0, 9>(sA, tmem, s_w512);
                else tc_epilogue1<9, 17>(sA, tmem, s_w512);
                tc::fence_async_smem();
                tc::fence_before();
                __syncthreads();
                if (threadIdx.x == 0)
                {
                    tc::fence_after();
                    const uint64_t dB = tc::desc_sw128(tc::smem_addr(sB2));
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                    {
                        const uint64_t dA = tc::desc_sw128(tc::smem_addr(sA + i * kTcTile));
                        const uint32_t d = tmem + kTcD2 + 32 * i;
                        tc::mma_f16(d, dA + 0, dB + 0, kTcIdesc, 0u);
                        tc::mma_f16(d, dA + 2, dB + 2, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 0, dB + 4, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 2, dB + 6, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 4, dB + 0, kTcIdesc, 1u);
                        tc::mma_f16(d, dA + 6, dB + 2, kTcIdesc, 1u);
                    }
                    tc::commit(&s_bar);
                }
                pending = 1;
                if (!wait_mma())
                {
                    abort = true;
                    break;
                }
                // epilogue 2: warps 0-3 take k2 = q' (tile 0), warps 4-7 k2 = 8 + q' (tile 1); warp 0
                // also k2 = 16 (tile 2)
                if (a.power == 1)
                {
                    tc_epilogue2<true>(tmem, threadIdx.x < 128 ? 0 : 1, s_out, s_scale);
                    if (threadIdx.x < 32) tc_epilogue2<true>(tmem, 2, s_out, s_scale);
                }
                else
                {
                    tc_epilogue2<false>(tmem, threadIdx.x < 128 ? 0 : 1, s_out, s_scale);
                    if (threadIdx.x < 32) tc_epilogue2<false>(tmem, 2, s_out, s_scale);
                }
                tc::fence_before();
                __syncthreads();
                if (fcol < Tv)
                {
                    // the FP32 kernel's mel sweep over the power tile (see fused.cu)
                    const bool second = fcol + 1 < Tv;
                    const int m0 = melGrp[g], m1 = melGrp[g + 1];
                    float* yp = it.y + size_t(f0 - it.f0) + size_t(m0) * hs + fcol;
                    float2 fall = make_float2(0.f, 0.f);
                    for (int i = m0; i <= m1; ++i)
                    {
                        const int2 iv = melIv[i];
                        const float* sp = s_out + iv.x * LD + fcol;
                        float2 rise = make_float2(0.f, 0.f);
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
            if (abort) break;
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
                const int fd = threadIdx.x & (a.dbFrames - 1);
                const int gd = threadIdx.x / a.dbFrames;
                const int kDbGroups = kFusedThreads / a.dbFrames;
                if (fd < it.Tv)
                {
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
        if (threadIdx.x == 0)
        {
            const long long w = wAfter >= 0 ? wAfter : (long long)atomicAdd(RPPB_WR(workCounter), 1ull);
            wAfter = w < total - 2ll * gridDim.x ? (long long)atomicAdd(RPPB_WR(workCounter), 1ull) : -1ll;
            const Item nx = decode_item<TF>(a, cnt, prefix, nslots, total, w);
            prefetch_span(nx);
            s_it[cur] = nx;
        }
        else if (threadIdx.x == 32 && it.kind == 0)
        {
            float v = s_warpMax[0];
            for (int i = 1; i < kFusedThreads / 32; ++i) v = fmaxf(v, s_warpMax[i]);
            atomicMax(RPPB_WR(maxKey + b), float_key(v));
            asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(RPPB_WR(done + b)) : "memory");
        }
        cur ^= 1;
    }

    // leave: after a timeout, wait once more (bounded) for the MMAs in flight, then free tensor memory
    if (pending && threadIdx.x == 0) tc::mbar_wait(&s_bar, phase, kTcWaitLimit);
    tc::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc<kTcTmemCols>(tmem);
}

}  // namespace

bool frontend_tc_supported(const FrontendArgs& a) { return a.nfft == kTcNfft && a.W <= kTcNfft; }

size_t frontend_tc_smem_bytes(const FrontendArgs& a) { return TcLayout(a.mel.numFilter, a.W, a.hop).total + 1024; }

void launch_frontend_tc(Handle& h, const FrontendArgs& a, void* scratch, uint4* melScratch)
{
    const int nslots = a.n + a.lookahead;
    Carver cv(scratch);
    long long* prefix = cv.take<long long>(nslots + 1);
    unsigned long long* counter = cv.take<unsigned long long>(1);
    int* done = cv.take<int>(a.n);
    unsigned* maxKey = cv.take<unsigned>(a.n);
    const TcLayout lay(a.mel.numFilter, a.W, a.hop);
    const size_t smem = lay.total + 1024;
    if (smem > 227 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "numFilter too large for the fused tile");
    const float2* tw = spectrogram_twiddles(h, kTcNfft);
    // the mel tables (the FP32 kernel's block): cached per handle and parameters, or, while the stream
    // is being captured with parameters the handle has not seen, built into the call's scratch
    uint4* melTables = fused_mel_table_cache<kTcNfft, kTcTF>(h, a);
    if (!melTables)
    {
        melTables = melScratch;
        const FusedLayout<kTcNfft, kTcTF> fl(a.mel.numFilter, a.W, a.hop);
        const void* tk = reinterpret_cast<const void*>(fused_mel_tables_kernel<kTcNfft, kTcTF>);
        persistent_grid(h, tk, kFusedThreads, fl.total);
        fused_mel_tables_kernel<kTcNfft, kTcTF><<<1, kFusedThreads, fl.total, h.stream()>>>(a, melTables);
        count_launch();
        check_cuda(cudaGetLastError(), "fused_mel_tables_kernel");
    }
    const size_t clear = reinterpret_cast<char*>(maxKey + a.n) - reinterpret_cast<char*>(counter);
    launch_ragged_prefix(SlotCount<kTcTF>{a, a.n, a.lookahead}, nslots, prefix, h.stream(),
                         reinterpret_cast<unsigned*>(counter), int(clear / 4));
    const void* k = reinterpret_cast<const void*>(frontend_tc_kernel<kTcTF>);
    // two CTAs need 2 x ~100 KB of shared memory: ask for the largest carveout, or the driver may pick
    // one that holds a single CTA (a function attribute of this kernel only)
    {
        static std::mutex mu;
        static std::set<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (done.insert(h.device()).second)
            check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                            int(cudaSharedmemCarveoutMaxShared)),
                       "shared memory carveout");
    }
    persistent_grid(h, k, kFusedThreads, smem);   // sets the kernel's shared-memory opt-in
    // CTAs per SM: two (registers: 256 threads x 128; tensor memory: 2 x 256 columns) when their shared
    // memory fits the SM, counted directly (the occupancy query reports one for this kernel, while two
    // run side by side)
    int perSm = 2;
    {
        static std::mutex mu;
        static std::map<int, std::pair<int, size_t>> smInfo;   // device -> (shared memory per SM, static)
        std::lock_guard<std::mutex> lock(mu);
        auto it = smInfo.find(h.device());
        if (it == smInfo.end())
        {
            int perSmBytes = 0;
            check_cuda(cudaDeviceGetAttribute(&perSmBytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h.device()),
                       "shared memory per SM");
            cudaFuncAttributes fa{};
            check_cuda(cudaFuncGetAttributes(&fa, k), "cudaFuncGetAttributes");
            it = smInfo.emplace(h.device(), std::make_pair(perSmBytes, size_t(fa.sharedSizeBytes))).first;
        }
        const size_t perCta = smem + it->second.second + 1024;   // + the driver's reserved 1 KB per CTA
        perSm = std::max(1, std::min(2, int(size_t(it->second.first) / perCta)));
    }
    int grid = perSm * h.num_sms();
    if (a.ctasPerSm > 0) grid = std::min(grid, a.ctasPerSm * h.num_sms());
    if (a.reserveSms > 0 && a.reserveSms < h.num_sms())
        grid = std::max(1, grid / h.num_sms() * (h.num_sms() - a.reserveSms));
    launch_dependent(frontend_tc_kernel<kTcTF>, dim3(grid), dim3(kFusedThreads), smem, h.stream(), "frontend_tc_kernel",
                     a, tw, static_cast<const long long*>(prefix), counter, done, maxKey, h.device_flags(),
                     static_cast<const uint4*>(melTables));
    count_launch();
}

}  // namespace rppb
