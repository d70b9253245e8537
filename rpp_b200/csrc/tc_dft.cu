// Tensor-core spectrogram: the short-time DFT as a GEMM on the 5th-generation tensor cores (tcgen05,
// accumulators in tensor memory), for the precision study of the front end.
//
//   power[f][k] = |sum_t frame_f[t] * w[t] * exp(-2 pi i k (t + off) / nfft)|^2
//
// is the GEMM C = A x B^T with A[f][t] = the (pre-emphasized, padded) signal sample of frame f at
// window position t (M = frames, K = window length padded to one 128-byte row) and B[n][t] = the
// window-folded DFT basis, n = 2k -> w[t] cos(.), n = 2k + 1 -> -w[t] sin(.) for bins 1..nfft/2-1;
// column 0 holds bin 0 and column 1 (the identically zero sine of bin 0) holds the Nyquist bin, so
// N = nfft exactly.  The basis is built in FP64 on the host and rounded once to the operand format.
//
// Operand formats (FP32 accumulation in every case):
//   kTcBf16    BF16, one pass;
//   kTcBf16x3  x = hi + lo with both parts BF16; hi*hi + hi*lo + lo*hi (three MMAs per K step);
//   kTcTf32    FP32 rounded to TF32 (round to nearest, ties away) before the MMA;
//   kTcFp8     E4M3; every frame is materialized and scaled so its largest sample maps to 448, the
//              basis is scaled by 256, and the epilogue divides both scales out.
// A is read in place from the padded signal for BF16/TF32: a 3-D tensor map (window position,
// frame, clip) whose frame rows start hop elements apart and overlap, so TMA needs hop * element
// size to be a multiple of 16 bytes; if the driver refuses such a map, or for FP8 (each frame
// carries its own scale), the frames are materialized [frame][kPad] first.
//
// Structure: one persistent CTA per SM (192 threads; work items = (clip, 128-frame tile, 256-column
// chunk)), warp-specialized around a ring of shared-memory stages, each one 64-byte K block of A
// (128 rows) and B (256 rows) in the 64-byte-swizzled K-major layout (8 stages; 4 for the split
// format, which stages hi and lo parts):
//   warp 0, one lane: TMA producer (tiled bulk tensor loads of this GPU's memory, into this CTA only),
//     completing bytes on the stage's "full" mbarrier;
//   warp 1, one lane: issues tcgen05.mma (M 128, N 256, 32 bytes of K per instruction) into one of
//     two tensor-memory accumulators and commits each stage to its "empty" mbarrier, and each
//     finished tile to the accumulator's "full" mbarrier;
//   warps 2-5: epilogue, tcgen05.ld of the finished accumulator (each warp its 32-lane quarter =
//     32 frames), re^2 + im^2 (or the linear output), NFT rows (32 consecutive frames per warp store)
//     or NTF rows, then an arrival on the accumulator's "empty" mbarrier, while the MMAs fill the
//     other accumulator.
// All waits are bounded: a timeout sets the device error word and a CTA abort flag that ends the
// other roles' waits; before the tensor memory is freed the producer waits (bounded) for its last
// loads and the MMA thread for its last MMAs.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "mel_tables.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 192;        // warp 0: TMA producer; warp 1: MMA issuer and tensor-memory owner;
                                     // warps 2-5: epilogue (one 32-lane quarter of tensor memory each)
constexpr int kTileM = 128;          // frames per tile
constexpr int kTileN = 256;          // basis columns per MMA / work item
constexpr int kKBytes = 64;          // bytes of K per operand row and stage (64-byte swizzle)
constexpr int kRowBytes = 128;       // K padding granule of the operands (kPad is a multiple of 128 bytes)
constexpr int kTmemCols = 2 * kTileN;           // two accumulators: MMAs fill one while the epilogue drains the other
constexpr size_t kRingBytes = 192 * 1024;       // shared memory of the stage ring
constexpr long long kWaitLimit = 1ll << 21;     // try_wait polls: on the order of a second
constexpr float kFp8BasisScale = 256.f;
constexpr float kFp8Max = 448.f;

constexpr size_t kABytes = size_t(kTileM) * kKBytes;   // 8 KB
constexpr size_t kBBytes = size_t(kTileN) * kKBytes;   // 16 KB

template <int FMT>
struct Fmt
{
    static constexpr int kElem = (FMT == kTcTf32) ? 4 : (FMT == kTcFp8) ? 1 : 2;
    static constexpr int kBlockK = kKBytes / kElem;         // elements per stage row
    static constexpr bool kSplit = FMT == kTcBf16x3;
    static constexpr uint32_t kStageBytes = uint32_t((kSplit ? 2 : 1) * (kABytes + kBBytes));
    static constexpr int kStages = int(kRingBytes / kStageBytes);   // 8, or 4 for the split format
    // Instruction descriptor: F32 accumulator (bit 4), A/B formats (bits 7, 10), both K-major,
    // N >> 3 at bit 17, M >> 4 at bit 24.  Formats: kind::f16 BF16 = 1, kind::tf32 TF32 = 2,
    // kind::f8f6f4 E4M3 = 0.
    static constexpr uint32_t kFormat = (FMT == kTcTf32) ? 2u : (FMT == kTcFp8) ? 0u : 1u;
    static constexpr uint32_t kIdesc = (1u << 4) | (kFormat << 7) | (kFormat << 10) | (uint32_t(kTileN >> 3) << 17) |
                                       (uint32_t(kTileM >> 4) << 24);
    static_assert(kStages >= 3, "stage ring");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor: K-major, 64-byte swizzle (the layout TMA writes with
// CU_TENSOR_MAP_SWIZZLE_64B), 8-row atoms 512 bytes apart.  Each MMA reads 32 bytes of K; the next
// 32 bytes of a row start 32 bytes later (the swizzle is a function of the address).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFF);            // start address
    d |= uint64_t(1) << 16;                           // leading byte offset (unused for swizzled K-major)
    d |= uint64_t(512 >> 4) << 32;                    // stride byte offset: next 8-row atom
    d |= uint64_t(1) << 46;                           // descriptor version (Blackwell)
    d |= uint64_t(4) << 61;                           // layout: SWIZZLE_64B
    return d;
}

template <int FMT>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    if constexpr (FMT == kTcTf32)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(a), "l"(b), "r"(Fmt<FMT>::kIdesc), "r"(accumulate));
    else if constexpr (FMT == kTcFp8)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(a), "l"(b), "r"(Fmt<FMT>::kIdesc), "r"(accumulate));
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(a), "l"(b), "r"(Fmt<FMT>::kIdesc), "r"(accumulate));
}

// Arrives on the mbarrier once every tcgen05 operation this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the mbarrier phase with parity `parity` to complete (a fresh barrier counts its
// phase before the first as complete, so a wait on parity 1 returns at once).  False on timeout, or
// when another role of the CTA has set *abortFlag.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const volatile int* abortFlag)
{
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kWaitLimit; ++i)
    {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 63) == 63 && *abortFlag) return false;
    }
    return false;
}

// TMA tile loads into shared memory, completing bytes on the mbarrier (this GPU's memory only).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

struct TcArgs
{
    int kPad;
    int nfft;                   // basis rows (N)
    const float* invScale;      // FP8: per frame 1 / (frame scale * basis scale), [n][maxFrames]
    int maxFrames;
    float* dst;
    uint32_t dstNStride, dstHStride;
    bool nft;
    int power;
    const int* frames;          // frames per clip
    int n;
    int* errorWord;
    int validN;                 // linear epilogue: output columns (mel filters)
};

// Tensor maps of the operands: A [clip][frame row][K] (rows may overlap: row stride = hop), B [N][K],
// and the lo parts of the split format.
struct TcMaps
{
    CUtensorMap a, aLo, b, bLo;
};

constexpr int kEpiPower = 0;
constexpr int kEpiLinear = 1;

struct TcCount
{
    const int* frames;
    int chunks;
    __device__ long long operator()(int b) const
    {
        const int F = max(*RPPB_RD(frames + b), 0);
        return (long long)((F + kTileM - 1) / kTileM) * chunks;
    }
};

// Work item w: clip b, frames f0 .. f0 + 127, basis columns n0 .. n0 + 255.
struct TcItem
{
    int b, f0, n0;
};

__device__ __forceinline__ TcItem tc_item(const long long* prefix, int n, int chunks, long long w)
{
    TcItem it;
    it.b = ragged_find(prefix, n, w);
    const int local = int(w - prefix[it.b]);
    it.f0 = (local / chunks) * kTileM;
    it.n0 = (local % chunks) * kTileN;
    return it;
}

// EPI: kEpiPower -- column pairs (cos, -sin) of one bin -> power / magnitude (the spectrogram);
//      kEpiLinear -- column n < validN -> the accumulator itself (the mel projection).
//
// Persistent over work items (every role walks the same sequence w = blockIdx.x + k * gridDim.x):
//   producer (warp 0, one lane): per K block of 64 bytes, wait until the ring stage is free, then TMA
//     loads of A (128 frame rows) and B (256 basis rows), plus their lo parts, onto the stage's
//     "full" barrier with the expected byte count;
//   MMA (warp 1, one lane): per work item, wait until the epilogue has drained the accumulator it
//     fills next; per stage, wait for "full", issue the MMAs (M 128, N 256, 32 bytes of K each; the
//     split format adds hi*lo and lo*hi), commit to the stage's "empty" barrier (frees it for the
//     producer when the MMAs finish); after the last K block, commit to the accumulator's "full";
//   epilogue (warps 2-5): wait for the accumulator, read it with tcgen05.ld (the warp's 32 lanes = 32
//     frames), form power / the linear output, store, and arrive on the accumulator's "empty".
// Every wait is bounded; the first role to time out sets the device error word (bit 2) and the CTA's
// abort flag, and the others leave their loops at their next wait.  Before the tensor memory is
// freed the producer waits (bounded) for its last loads and the MMA thread for its last MMAs.
template <int FMT, int EPI>
__global__ void __launch_bounds__(kThreads, 1) tc_dft_kernel(TcArgs a, const long long* __restrict__ prefix,
                                                              const __grid_constant__ TcMaps maps)
{
    using T = Fmt<FMT>;
    constexpr int S = T::kStages;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t fullBar[S], emptyBar[S], accFull[2], accEmpty[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 1)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0)
    {
        for (int s = 0; s < S; ++s)
        {
            mbar_init(&fullBar[s], 1);
            mbar_init(&emptyBar[s], 1);
        }
        for (int i = 0; i < 2; ++i)
        {
            mbar_init(&accFull[i], 1);
            mbar_init(&accEmpty[i], 4);   // one arrival per epilogue warp
        }
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid == 32)
    {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.a)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.b)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    volatile int* abortFlag = &s_abort;
    auto fail = [&]() {
        if (!*abortFlag)
        {
            *abortFlag = 1;
            atomicOr(RPPB_WR(a.errorWord), 2);
        }
    };

    const int chunks = a.nfft / kTileN;
    const int kBlocks = a.kPad / T::kBlockK;
    const long long total = prefix[a.n];

    if (warp == 0)
    {
        if (lane == 0)
        {
            long long loads = 0;   // stage loads issued
            int s = 0;
            uint32_t ph = 0;
            for (long long w = blockIdx.x; w < total && !*abortFlag; w += gridDim.x)
            {
                const TcItem it = tc_item(prefix, a.n, chunks, w);
                for (int kb = 0; kb < kBlocks; ++kb)
                {
                    if (!mbar_wait(&emptyBar[s], ph ^ 1u, abortFlag))
                    {
                        fail();
                        break;
                    }
                    unsigned char* sA = smem + size_t(s) * T::kStageBytes;
                    unsigned char* sB = sA + kABytes;
                    mbar_expect_tx(&fullBar[s], T::kStageBytes);
                    const int x = kb * T::kBlockK;
                    tma_load_3d(sA, &maps.a, x, it.f0, it.b, &fullBar[s]);
                    tma_load_2d(sB, &maps.b, x, it.n0, &fullBar[s]);
                    if constexpr (T::kSplit)
                    {
                        tma_load_3d(sB + kBBytes, &maps.aLo, x, it.f0, it.b, &fullBar[s]);
                        tma_load_2d(sB + kBBytes + kABytes, &maps.bLo, x, it.n0, &fullBar[s]);
                    }
                    ++loads;
                    if (++s == S)
                    {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            // before the CTA leaves: every issued load has landed (stage s' last load completes the
            // phase with parity (its loads - 1) & 1)
            for (int st = 0; st < S; ++st)
            {
                const long long cnt = loads > st ? (loads - st + S - 1) / S : 0;
                if (cnt > 0) mbar_wait(&fullBar[st], uint32_t((cnt - 1) & 1), abortFlag);
            }
        }
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            int s = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            uint64_t* lastBar = nullptr;
            uint32_t lastParity = 0;
            for (long long w = blockIdx.x; w < total && !*abortFlag; w += gridDim.x)
            {
                if (!mbar_wait(&accEmpty[acc], aph ^ 1u, abortFlag))
                {
                    fail();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + uint32_t(acc * kTileN);
                bool ok = true;
                for (int kb = 0; kb < kBlocks; ++kb)
                {
                    if (!mbar_wait(&fullBar[s], ph, abortFlag))
                    {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sA = smem_u32(smem + size_t(s) * T::kStageBytes);
                    const uint32_t sB = sA + uint32_t(kABytes);
                    const uint64_t dA = umma_desc(sA), dB = umma_desc(sB);
#pragma unroll
                    for (int ks = 0; ks < kKBytes / 32; ++ks)
                    {
                        const uint64_t step = uint64_t(ks * 32) >> 4;   // 32 bytes of K along the swizzled row
                        mma<FMT>(d, dA + step, dB + step, (kb > 0 || ks > 0) ? 1u : 0u);
                        if constexpr (T::kSplit)
                        {
                            const uint64_t dAl = umma_desc(sB + uint32_t(kBBytes));
                            const uint64_t dBl = umma_desc(sB + uint32_t(kBBytes + kABytes));
                            mma<FMT>(d, dA + step, dBl + step, 1u);
                            mma<FMT>(d, dAl + step, dB + step, 1u);
                        }
                    }
                    mma_commit(&emptyBar[s]);
                    lastBar = &emptyBar[s];
                    lastParity = ph;
                    if (++s == S)
                    {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok)
                {
                    fail();
                    break;
                }
                mma_commit(&accFull[acc]);
                if (++acc == 2)
                {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            // the MMAs in flight end before the tensor memory is freed (the last commit covers all)
            if (lastBar) mbar_wait(lastBar, lastParity, abortFlag);
        }
    }
    else
    {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 = tile rows (frames)
        const int q = warp & 3;
        const int r = q * 32 + lane;
        int acc = 0;
        uint32_t aph = 0;
        for (long long w = blockIdx.x; w < total && !*abortFlag; w += gridDim.x)
        {
            const TcItem it = tc_item(prefix, a.n, chunks, w);
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&accFull[acc], aph, abortFlag));
            if (!ok)
            {
                if (lane == 0) fail();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int F = *RPPB_RD(a.frames + it.b);
            const int frame = it.f0 + r;
            float* y = a.dst + size_t(it.b) * a.dstNStride;
            float sc = 1.f;
            if constexpr (FMT == kTcFp8)
                if (frame < F) sc = *RPPB_RD(a.invScale + (size_t(it.b) * a.maxFrames + frame));
#pragma unroll 1
            for (int c0 = 0; c0 < kTileN; c0 += 32)
            {
                uint32_t v[32];
                const uint32_t taddr = tmem + (uint32_t(q * 32) << 16) + uint32_t(acc * kTileN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int n0 = it.n0 + c0;
                if (EPI == kEpiLinear && frame < F)
                {
#pragma unroll
                    for (int k = 0; k < 32; ++k)
                    {
                        const int col = n0 + k;
                        if (col >= a.validN) break;
                        const float o = __uint_as_float(v[k]) * sc;
                        if (a.nft) *RPPB_WR(y + (size_t(col) * a.dstHStride + frame)) = o;
                        else *RPPB_WR(y + (size_t(frame) * a.dstHStride + col)) = o;
                    }
                }
                if (EPI == kEpiPower && frame < F)
                {
#pragma unroll
                    for (int k = 0; k < 16; ++k)
                    {
                        const float re = __uint_as_float(v[2 * k]) * sc, im = __uint_as_float(v[2 * k + 1]) * sc;
                        const int col = n0 + 2 * k;   // even column: bin col/2 (cos, -sin)
                        if (col == 0)
                        {
                            // column 0: bin 0 (real); column 1: Nyquist bin (real)
                            const float p0 = re * re, pn = im * im;
                            const float o0 = a.power == 1 ? sqrtf(p0) : p0;
                            const float on = a.power == 1 ? sqrtf(pn) : pn;
                            const int nyq = a.nfft / 2;
                            if (a.nft)
                            {
                                *RPPB_WR(y + frame) = o0;
                                *RPPB_WR(y + (size_t(nyq) * a.dstHStride + frame)) = on;
                            }
                            else
                            {
                                *RPPB_WR(y + size_t(frame) * a.dstHStride) = o0;
                                *RPPB_WR(y + (size_t(frame) * a.dstHStride + nyq)) = on;
                            }
                            continue;
                        }
                        const int bin = col >> 1;
                        const float p = fmaf(re, re, im * im);
                        const float o = a.power == 1 ? sqrtf(p) : p;
                        if (a.nft) *RPPB_WR(y + (size_t(bin) * a.dstHStride + frame)) = o;
                        else *RPPB_WR(y + (size_t(frame) * a.dstHStride + bin)) = o;
                    }
                }
            }
            // this warp's reads of the accumulator are done: the MMA thread may overwrite it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&accEmpty[acc]);
            if (++acc == 2)
            {
                acc = 0;
                aph ^= 1u;
            }
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
    {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// The sample the spectrogram frames at padded position i (= signal index i - centerOffset): the
// (optionally pre-emphasized) signal with reflect or zero padding, as stft.cuh's sources give it.
struct PaddedSignal
{
    const float* x;
    int L;
    float c, border;
    bool preemph, reflect;
    int centerOffset;
    __device__ __forceinline__ float operator()(long long i) const
    {
        long long t = i - centerOffset;
        if (!(t >= 0 && t < L))
        {
            if (!reflect || L <= 0 || t > 0x3fffffff || t < -0x3fffffff) return 0.f;
            t = reflect_index(int(t), 0, L);
        }
        if (!preemph) return *RPPB_RD(x + t);
        return __fsub_rn(*RPPB_RD(x + t), __fmul_rn(c, t == 0 ? border : *RPPB_RD(x + (t - 1))));
    }
};

__device__ __forceinline__ PaddedSignal padded_signal(const float* src, uint32_t srcStride, size_t srcElems,
                                                      const int* len, const float* coeff, int border, bool reflect,
                                                      int centerOffset, int b)
{
    PaddedSignal p;
    p.x = src + size_t(b) * srcStride;
    p.L = min(*RPPB_RD(len + b), int(srcStride));
    p.preemph = coeff != nullptr;
    p.c = p.preemph ? *RPPB_RD(coeff + b) : 0.f;
    const size_t base = size_t(b) * srcStride;
    p.border = border == 1 ? *RPPB_RD(p.x) : border == 2 ? (base + 1 < srcElems ? *RPPB_RD(p.x + 1) : 0.f) : 0.f;
    p.reflect = reflect;
    p.centerOffset = centerOffset;
    return p;
}

struct PrepArgs
{
    const float* src;
    uint32_t srcStride;
    size_t srcElems;
    const int* len;
    const float* coeff;
    int border;
    bool reflect;
    int centerOffset;
    int n;
};

// BF16 (hi, and lo for the split format) or TF32 copy of the padded signal, [n][clipStride].  Each
// thread takes 8 consecutive positions: where they and the sample before them lie inside the clip
// (the interior: no padding, no border sample), two 4-sample loads and one scalar give the
// pre-emphasized values and the results leave as 16-byte stores (clipStride keeps rows 16-byte
// aligned); at the clip's ends position by position.  Same values either way.
template <int FMT>
__global__ void tc_prep_kernel(PrepArgs p, void* __restrict__ outHi, void* __restrict__ outLo, uint32_t clipStride)
{
    const uint32_t groups = (clipStride + 7) / 8;
    for (int b = blockIdx.y; b < p.n; b += gridDim.y)
    {
        const PaddedSignal sig =
            padded_signal(p.src, p.srcStride, p.srcElems, p.len, p.coeff, p.border, p.reflect, p.centerOffset, b);
        for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x)
        {
            const uint32_t i0 = g * 8;
            const long long t0 = (long long)i0 - sig.centerOffset;
            const bool whole = i0 + 8 <= clipStride;
            float v[8];
            if (whole && t0 >= 1 && t0 + 8 <= sig.L)
            {
                const float* x = sig.x + t0;
                float r[8];
                if ((reinterpret_cast<uintptr_t>(x) & 15) == 0)
                {
                    const float4 a = __ldg(RPPB_RD(reinterpret_cast<const float4*>(x)));
                    const float4 c4 = __ldg(RPPB_RD(reinterpret_cast<const float4*>(x + 4)));
                    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
                    r[4] = c4.x; r[5] = c4.y; r[6] = c4.z; r[7] = c4.w;
                }
                else
#pragma unroll
                    for (int k = 0; k < 8; ++k) r[k] = __ldg(RPPB_RD(x + k));
                if (sig.preemph)
                {
                    float prev = __ldg(RPPB_RD(x - 1));
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                    {
                        v[k] = __fsub_rn(r[k], __fmul_rn(sig.c, prev));
                        prev = r[k];
                    }
                }
                else
#pragma unroll
                    for (int k = 0; k < 8; ++k) v[k] = r[k];
            }
            else
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = i0 + k < clipStride ? sig(i0 + k) : 0.f;
            const size_t o = size_t(b) * clipStride + i0;
            if constexpr (FMT == kTcTf32)
            {
                uint32_t t[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t[k]) : "f"(v[k]));
                uint32_t* out = static_cast<uint32_t*>(outHi) + o;
                if (whole)
                {
                    *RPPB_WR(reinterpret_cast<uint4*>(out)) = make_uint4(t[0], t[1], t[2], t[3]);
                    *RPPB_WR(reinterpret_cast<uint4*>(out) + 1) = make_uint4(t[4], t[5], t[6], t[7]);
                }
                else
                    for (int k = 0; k < 8 && i0 + k < clipStride; ++k) *RPPB_WR(out + k) = t[k];
            }
            else
            {
                uint32_t hw[4], lw[4];
#pragma unroll
                for (int k = 0; k < 8; k += 2)
                {
                    const __nv_bfloat16 h0 = __float2bfloat16_rn(v[k]), h1 = __float2bfloat16_rn(v[k + 1]);
                    hw[k / 2] = uint32_t(__bfloat16_as_ushort(h0)) | (uint32_t(__bfloat16_as_ushort(h1)) << 16);
                    if constexpr (FMT == kTcBf16x3)
                    {
                        const __nv_bfloat16 l0 = __float2bfloat16_rn(v[k] - __bfloat162float(h0));
                        const __nv_bfloat16 l1 = __float2bfloat16_rn(v[k + 1] - __bfloat162float(h1));
                        lw[k / 2] = uint32_t(__bfloat16_as_ushort(l0)) | (uint32_t(__bfloat16_as_ushort(l1)) << 16);
                    }
                }
                __nv_bfloat16* hi = static_cast<__nv_bfloat16*>(outHi) + o;
                __nv_bfloat16* lo = FMT == kTcBf16x3 ? static_cast<__nv_bfloat16*>(outLo) + o : nullptr;
                if (whole)
                {
                    *RPPB_WR(reinterpret_cast<uint4*>(hi)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                    if constexpr (FMT == kTcBf16x3)
                        *RPPB_WR(reinterpret_cast<uint4*>(lo)) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                }
                else
                    for (int k = 0; k < 8 && i0 + k < clipStride; ++k)
                    {
                        *RPPB_WR(hi + k) = __ushort_as_bfloat16(uint16_t(hw[k / 2] >> (16 * (k & 1))));
                        if constexpr (FMT == kTcBf16x3)
                            *RPPB_WR(lo + k) = __ushort_as_bfloat16(uint16_t(lw[k / 2] >> (16 * (k & 1))));
                    }
            }
        }
    }
}

// FP8: one warp per frame; frame f of clip b becomes row [f][kPad] scaled by 448 / max|sample|.
__global__ void tc_prep_fp8_kernel(PrepArgs p, const int* __restrict__ frames, int maxFrames, int W, int hop, int kPad,
                                   __nv_fp8_e4m3* __restrict__ out, float* __restrict__ invScale)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerBlock = blockDim.x >> 5;
    for (int b = blockIdx.y; b < p.n; b += gridDim.y)
    {
        const PaddedSignal sig =
            padded_signal(p.src, p.srcStride, p.srcElems, p.len, p.coeff, p.border, p.reflect, p.centerOffset, b);
        const int F = *RPPB_RD(frames + b);
        for (int f = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5); f < F; f += gridDim.x * warpsPerBlock)
        {
            const long long s0 = (long long)f * hop;
            float m = 0.f;
            for (int t = lane; t < W; t += 32) m = fmaxf(m, fabsf(sig(s0 + t)));
            m = warp_max(m);
            const float scale = m > 0.f ? kFp8Max / m : 1.f;
            __nv_fp8_e4m3* row = out + (size_t(b) * maxFrames + f) * kPad;
            for (int t = lane; t < kPad; t += 32) *RPPB_WR(row + t) = __nv_fp8_e4m3(t < W ? sig(s0 + t) * scale : 0.f);
            if (lane == 0) *RPPB_WR(invScale + (size_t(b) * maxFrames + f)) = 1.f / (scale * kFp8BasisScale);
        }
    }
}

// BF16 (hi, lo) or TF32 frame rows [n][maxFrames][kPad] (window positions >= W are zero): the A
// operand when the driver does not accept a tensor map whose frame rows overlap.
template <int FMT>
__global__ void tc_prep_rows_kernel(PrepArgs p, const int* __restrict__ frames, int maxFrames, int W, int hop,
                                    int kPad, void* __restrict__ outHi, void* __restrict__ outLo)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerBlock = blockDim.x >> 5;
    for (int b = blockIdx.y; b < p.n; b += gridDim.y)
    {
        const PaddedSignal sig =
            padded_signal(p.src, p.srcStride, p.srcElems, p.len, p.coeff, p.border, p.reflect, p.centerOffset, b);
        const int F = *RPPB_RD(frames + b);
        for (int f = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5); f < F; f += gridDim.x * warpsPerBlock)
        {
            const long long s0 = (long long)f * hop;
            const size_t row = (size_t(b) * maxFrames + f) * kPad;
            for (int t = lane; t < kPad; t += 32)
            {
                const float v = t < W ? sig(s0 + t) : 0.f;
                if constexpr (FMT == kTcTf32)
                {
                    uint32_t u;
                    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v));
                    *RPPB_WR(static_cast<uint32_t*>(outHi) + (row + t)) = u;
                }
                else
                {
                    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
                    *RPPB_WR(static_cast<__nv_bfloat16*>(outHi) + (row + t)) = hi;
                    if constexpr (FMT == kTcBf16x3)
                        *RPPB_WR(static_cast<__nv_bfloat16*>(outLo) + (row + t)) =
                            __float2bfloat16_rn(v - __bfloat162float(hi));
                }
            }
        }
    }
}

__global__ void tc_frames_kernel(const int* __restrict__ len, uint32_t srcStride, int n, int W, int hop, bool center,
                                 int maxFrames, int* __restrict__ frames)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
        *RPPB_WR(frames + b) = min(num_windows(min(*RPPB_RD(len + b), int(srcStride)), W, hop, center), maxFrames);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver
// library); null if the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

CUtensorMapDataType map_type(int fmt)
{
    // TF32 operands are FP32 words already rounded to TF32: copied bit for bit
    return fmt == kTcTf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                          : fmt == kTcFp8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}

// A tiled map with 64-byte swizzle, zero fill outside the tensor; false if the driver refuses it.
bool encode_map(CUtensorMap* m, int fmt, int rank, const void* base, const cuuint64_t* dims,
                const cuuint64_t* strides, const cuuint32_t* box)
{
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint32_t one[3] = {1, 1, 1};
    return enc(m, map_type(fmt), cuuint32_t(rank), const_cast<void*>(base), dims, strides, box, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The operands as the kernel's tensor maps see them.
struct TcOperands
{
    const void* a;          // [n][clipStride] elements; frame row f of clip b starts at b * clipStride + f * rowStep
    const void* aLo;        // split format only
    uint32_t rowStep, clipStride;
    int rowsPerClip;        // frame rows a clip may address
    const void* b;          // [bRows][kPad]
    const void* bLo;
    int bRows;
};

template <int FMT>
TcMaps encode_maps(const TcOperands& op, int kPad, int n)
{
    using T = Fmt<FMT>;
    TcMaps maps;
    std::memset(&maps, 0, sizeof maps);
    const cuuint64_t e = T::kElem;
    const cuuint64_t aDims[3] = {cuuint64_t(kPad), cuuint64_t(std::max(op.rowsPerClip, 1)), cuuint64_t(n)};
    const cuuint64_t aStrides[2] = {op.rowStep * e, op.clipStride * e};
    const cuuint32_t aBox[3] = {cuuint32_t(T::kBlockK), cuuint32_t(kTileM), 1};
    const cuuint64_t bDims[2] = {cuuint64_t(kPad), cuuint64_t(op.bRows)};
    const cuuint64_t bStrides[1] = {cuuint64_t(kPad) * e};
    const cuuint32_t bBox[2] = {cuuint32_t(T::kBlockK), cuuint32_t(kTileN)};
    bool ok = encode_map(&maps.a, FMT, 3, op.a, aDims, aStrides, aBox) &&
              encode_map(&maps.b, FMT, 2, op.b, bDims, bStrides, bBox);
    if (T::kSplit)
        ok = ok && encode_map(&maps.aLo, FMT, 3, op.aLo, aDims, aStrides, aBox) &&
             encode_map(&maps.bLo, FMT, 2, op.bLo, bDims, bStrides, bBox);
    if (!ok) fail(RPP_ERROR, "cuTensorMapEncodeTiled refused an operand map of the tensor-core kernel");
    return maps;
}

template <int FMT, int EPI = kEpiPower>
void launch_format(Handle& h, const TcArgs& a, const TcOperands& op, const long long* prefix)
{
    const TcMaps maps = encode_maps<FMT>(op, a.kPad, a.n);
    const size_t smem = size_t(Fmt<FMT>::kStages) * Fmt<FMT>::kStageBytes + 1024;
    const int grid = persistent_grid(h, reinterpret_cast<const void*>(tc_dft_kernel<FMT, EPI>), kThreads, smem);
    tc_dft_kernel<FMT, EPI><<<grid, kThreads, smem, h.stream()>>>(a, prefix, maps);
    count_launch(1);
    check_cuda(cudaGetLastError(), "tc_dft_kernel");
}

int elem_bytes(int fmt) { return fmt == kTcTf32 ? 4 : fmt == kTcFp8 ? 1 : 2; }

uint16_t bf16_rne(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return uint16_t((u >> 16) | 0x40);   // NaN stays NaN
    u += 0x7fffu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}

float bf16_value(uint16_t h)
{
    const uint32_t u = uint32_t(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// FP32 -> TF32 (10 explicit mantissa bits), round to nearest with ties away from zero, finite inputs.
uint32_t tf32_rna(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (u + 0x1000u) & 0xffffe000u;
}

// ---------------------------------------------------------------- mel projection on tensor cores
// mel[f][m] = sum_k power[f][k] * W[m][k] as the GEMM C = A x B^T, A = the spectrum transposed to
// [frame][bin] (K-major, bins padded to one 128-byte row of operand elements), B = the dense filter
// bank [256][kPad] (rows >= numFilter zero).  W holds the mel_filter_bank kernel's weights (same
// tables, same float expressions); the GEMM sums them in the tensor core's order, not the
// reference's, so the result carries the operand precision's error, not bit-exactness.

constexpr int kMelN = 256;

struct MelWeightArgs
{
    MelParams mel;
    int nfft;            // (bins - 1) * 2
    int bins, kPad, fmt;
    unsigned char* b;    // operand [256][kPad] (hi, then lo for the split format)
    float* bScale;       // FP8: scale applied to W (device scalar)
};

// One CTA: the reference's mel tables in shared memory, the dense weights, their largest magnitude
// (FP8 scale: a power of two keeping it <= 448), then the operand copy.
__global__ void __launch_bounds__(256) mel_weights_kernel(MelWeightArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int nf = a.mel.numFilter;
    MelTableView T;
    T.range = reinterpret_cast<int*>(smem);
    T.first = T.range + 4;
    T.last = T.first + (nf + 2);
    T.norm = reinterpret_cast<float*>(T.last + (nf + 2));
    size_t off = (size_t(reinterpret_cast<unsigned char*>(T.norm + nf) - smem) + 7) & ~size_t(7);
    T.f0 = reinterpret_cast<double*>(smem + off);
    T.f1 = T.f0 + (nf + 1);
    T.weightsDown = reinterpret_cast<float*>(T.f1 + (nf + 1));
    __shared__ float s_max[8];
    build_mel_tables(T, a.mel, a.nfft);   // ends with __syncthreads
    auto weight = [&](int m, int k) -> float {
        if (m >= nf || k >= a.bins) return 0.f;
        float w = 0.f;
        if (k >= T.first[m] && k < T.last[m]) w = __fsub_rn(1.0f, T.weightsDown[k]);
        else if (k >= T.first[m + 1] && k < T.last[m + 1]) w = T.weightsDown[k];
        else return 0.f;
        return a.mel.normalize ? __fmul_rn(w, T.norm[m]) : w;
    };
    float mx = 0.f;
    for (int i = threadIdx.x; i < kMelN * a.kPad; i += blockDim.x) mx = fmaxf(mx, fabsf(weight(i / a.kPad, i % a.kPad)));
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = mx;
    __syncthreads();
    float scale = 1.f;
    if (a.fmt == kTcFp8)
    {
        float m = 0.f;
        for (int i = 0; i < 8; ++i) m = fmaxf(m, s_max[i]);
        if (m > 0.f) scale = exp2f(floorf(log2f(kFp8Max / m)));
        if (threadIdx.x == 0) *a.bScale = scale;
    }
    const size_t count = size_t(kMelN) * a.kPad;
    for (int i = threadIdx.x; i < kMelN * a.kPad; i += blockDim.x)
    {
        const float w = weight(i / a.kPad, i % a.kPad);
        if (a.fmt == kTcTf32)
        {
            uint32_t t;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(w));
            reinterpret_cast<uint32_t*>(a.b)[i] = t;
        }
        else if (a.fmt == kTcFp8)
            reinterpret_cast<__nv_fp8_e4m3*>(a.b)[i] = __nv_fp8_e4m3(w * scale);
        else
        {
            const __nv_bfloat16 hi = __float2bfloat16_rn(w);
            reinterpret_cast<__nv_bfloat16*>(a.b)[i] = hi;
            if (a.fmt == kTcBf16x3)
                reinterpret_cast<__nv_bfloat16*>(a.b)[count + i] = __float2bfloat16_rn(w - __bfloat162float(hi));
        }
    }
}

struct MelPrepArgs
{
    const float* src;            // NFT spectra [n][srcRows][srcHStride]
    uint32_t srcNStride, srcHStride;
    int bins, kPad, maxFrames, fmt, n;
    const int* frames;
    unsigned char* aHi;          // [n][maxFrames][kPad]
    unsigned char* aLo;
    float* invScale;             // FP8: 1 / (frame scale * weight scale), [n][maxFrames]
    const float* bScale;
};

// FP8 only: per frame, 448 / the frame's largest power.
__global__ void mel_frame_scale_kernel(MelPrepArgs a)
{
    for (int b = blockIdx.y; b < a.n; b += gridDim.y)
    {
        const float* x = a.src + size_t(b) * a.srcNStride;
        const int F = *RPPB_RD(a.frames + b);
        for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x)
        {
            float m = 0.f;
            for (int k = 0; k < a.bins; ++k) m = fmaxf(m, fabsf(*RPPB_RD(x + (size_t(k) * a.srcHStride + f))));
            const float sc = m > 0.f ? kFp8Max / m : 1.f;
            *RPPB_WR(a.invScale + (size_t(b) * a.maxFrames + f)) = 1.f / (sc * *RPPB_RD(a.bScale));
        }
    }
}

// [bin][frame] -> [frame][bin] in the operand format, 32 x 32 tiles through shared memory; bins
// past the spectrum and up to kPad are zero.
__global__ void __launch_bounds__(256) mel_prep_kernel(MelPrepArgs a)
{
    __shared__ float tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    for (int b = blockIdx.z; b < a.n; b += gridDim.z)
    {
        const int F = *RPPB_RD(a.frames + b);
        const int f0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
        if (f0 >= F || k0 >= a.kPad) continue;
        const float* x = a.src + size_t(b) * a.srcNStride;
        for (int r = ty; r < 32; r += 8)
        {
            const int k = k0 + r, f = f0 + tx;
            tile[r][tx] = (k < a.bins && f < F) ? *RPPB_RD(x + (size_t(k) * a.srcHStride + f)) : 0.f;
        }
        __syncthreads();
        for (int r = ty; r < 32; r += 8)
        {
            const int f = f0 + r, k = k0 + tx;
            if (f < F && k < a.kPad)
            {
                const float v = tile[tx][r];
                const size_t o = (size_t(b) * a.maxFrames + f) * a.kPad + k;
                if (a.fmt == kTcTf32)
                {
                    uint32_t t;
                    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(v));
                    *RPPB_WR(reinterpret_cast<uint32_t*>(a.aHi) + o) = t;
                }
                else if (a.fmt == kTcFp8)
                {
                    const float sc = 1.f / (*RPPB_RD(a.invScale + (size_t(b) * a.maxFrames + f)) * *RPPB_RD(a.bScale));
                    *RPPB_WR(reinterpret_cast<__nv_fp8_e4m3*>(a.aHi) + o) = __nv_fp8_e4m3(v * sc);
                }
                else
                {
                    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
                    *RPPB_WR(reinterpret_cast<__nv_bfloat16*>(a.aHi) + o) = hi;
                    if (a.fmt == kTcBf16x3)
                        *RPPB_WR(reinterpret_cast<__nv_bfloat16*>(a.aLo) + o) = __float2bfloat16_rn(v - __bfloat162float(hi));
                }
            }
        }
        __syncthreads();
    }
}

__global__ void mel_frames_kernel(const int* __restrict__ dims, int n, int maxFrames, int* __restrict__ frames)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
        *RPPB_WR(frames + b) = min(max(*RPPB_RD(dims + (2 * b + 1)), 0), maxFrames);
}

}  // namespace

bool tc_overlap_supported(const void* anyDevicePtr)
{
    // one encode per process of a map whose 128 rows of 512 BF16 elements start 256 bytes apart
    static const bool ok = [anyDevicePtr] {
        CUtensorMap m;
        const cuuint64_t dims[3] = {512, 128, 1};
        const cuuint64_t strides[2] = {256, 65536};
        const cuuint32_t box[3] = {32, 128, 1};
        return encode_map(&m, kTcBf16, 3, anyDevicePtr, dims, strides, box);
    }();
    return ok;
}

TcGeometry tc_geometry(int fmt, int windowLength, int windowStep, int maxFrames, int nfft, bool overlapRows)
{
    const int e = elem_bytes(fmt);
    const int blockK = kRowBytes / e;
    TcGeometry g;
    g.kPad = (windowLength + blockK - 1) / blockK * blockK;
    const int frames = std::max(maxFrames, 1);
    g.materialized = fmt == kTcFp8 || !overlapRows;
    if (g.materialized)
    {
        g.rowStep = uint32_t(g.kPad);
        g.clipStride = uint32_t(size_t(frames) * g.kPad);
    }
    else
    {
        const size_t span = size_t(frames - 1) * windowStep + g.kPad;
        const size_t granule = 16 / e;   // elements per 16 bytes: clip rows stay 16-byte aligned
        g.rowStep = uint32_t(windowStep);
        g.clipStride = uint32_t((span + granule - 1) / granule * granule);
    }
    const size_t bytes = size_t(nfft) * g.kPad * e * (fmt == kTcBf16x3 ? 2 : 1);
    g.basisFloats = (bytes + 3) / 4;
    return g;
}

void tc_build_basis(float* out, int fmt, int nfft, int W, int kPad, const float* win)
{
    const int off = (W < nfft) ? (nfft - W) / 2 : 0;
    const size_t count = size_t(nfft) * kPad;
    uint16_t* h16 = reinterpret_cast<uint16_t*>(out);
    uint32_t* h32 = reinterpret_cast<uint32_t*>(out);
    unsigned char* h8 = reinterpret_cast<unsigned char*>(out);
    for (int n = 0; n < nfft; ++n)
        for (int t = 0; t < kPad; ++t)
        {
            double v = 0.0;
            if (t < W)
            {
                const long long tt = t + off;
                double trig;
                if (n == 0) trig = 1.0;
                else if (n == 1) trig = (tt & 1) ? -1.0 : 1.0;   // Nyquist bin in the zero sine of bin 0
                else
                {
                    const long long bin = n >> 1;
                    const double ang = 2.0 * M_PI * double((bin * tt) % nfft) / double(nfft);
                    trig = (n & 1) ? -std::sin(ang) : std::cos(ang);
                }
                v = double(win[t]) * trig;
            }
            const size_t i = size_t(n) * kPad + t;
            if (fmt == kTcTf32) h32[i] = tf32_rna(float(v));
            else if (fmt == kTcFp8)
                h8[i] = static_cast<unsigned char>(
                    __nv_cvt_float_to_fp8(float(v * kFp8BasisScale), __NV_SATFINITE, __NV_E4M3));
            else
            {
                const uint16_t hi = bf16_rne(float(v));
                h16[i] = hi;
                if (fmt == kTcBf16x3) h16[count + i] = bf16_rne(float(v - double(bf16_value(hi))));
            }
        }
}

size_t tc_spectrogram_scratch_bytes(int n, int fmt, const TcGeometry& g, int maxFrames)
{
    Carver cv(nullptr);
    cv.take<long long>(n + 1);
    cv.take<int>(n);
    const size_t operand = size_t(n) * g.clipStride * elem_bytes(fmt);
    cv.take<char>(operand);
    if (fmt == kTcBf16x3) cv.take<char>(operand);
    if (fmt == kTcFp8) cv.take<float>(size_t(n) * std::max(maxFrames, 1));
    return cv.used();
}

void launch_tc_spectrogram(Handle& h, void* scratch, const TcSpectrogramArgs& s)
{
    if (s.n <= 0) return;
    const int e = elem_bytes(s.fmt);
    Carver cv(scratch);
    long long* prefix = cv.take<long long>(s.n + 1);
    int* frames = cv.take<int>(s.n);
    const size_t operand = size_t(s.n) * s.geo.clipStride * e;
    unsigned char* aHi = cv.take<unsigned char>(operand);
    unsigned char* aLo = s.fmt == kTcBf16x3 ? cv.take<unsigned char>(operand) : nullptr;
    float* invScale = s.fmt == kTcFp8 ? cv.take<float>(size_t(s.n) * std::max(s.maxFrames, 1)) : nullptr;

    tc_frames_kernel<<<(s.n + 255) / 256, 256, 0, h.stream()>>>(s.len, s.srcStride, s.n, s.windowLength,
                                                                 s.windowStep, s.center, s.maxFrames, frames);
    count_launch(1);
    PrepArgs p{s.src, s.srcStride, s.srcElems, s.len, s.coeff, s.border, s.reflect,
               s.center ? s.windowLength / 2 : 0, s.n};
    if (s.fmt == kTcFp8)
    {
        dim3 pg(std::min((std::max(s.maxFrames, 1) + 7) / 8, 256), std::min(s.n, 65535));
        tc_prep_fp8_kernel<<<pg, 256, 0, h.stream()>>>(p, frames, std::max(s.maxFrames, 1), s.windowLength,
                                                       s.windowStep, s.geo.kPad,
                                                       reinterpret_cast<__nv_fp8_e4m3*>(aHi), invScale);
    }
    else if (s.geo.materialized)
    {
        dim3 pg(std::min((std::max(s.maxFrames, 1) + 7) / 8, 256), std::min(s.n, 65535));
        const int mf = std::max(s.maxFrames, 1);
        if (s.fmt == kTcTf32)
            tc_prep_rows_kernel<kTcTf32><<<pg, 256, 0, h.stream()>>>(p, frames, mf, s.windowLength, s.windowStep,
                                                                     s.geo.kPad, aHi, nullptr);
        else if (s.fmt == kTcBf16x3)
            tc_prep_rows_kernel<kTcBf16x3><<<pg, 256, 0, h.stream()>>>(p, frames, mf, s.windowLength, s.windowStep,
                                                                       s.geo.kPad, aHi, aLo);
        else
            tc_prep_rows_kernel<kTcBf16><<<pg, 256, 0, h.stream()>>>(p, frames, mf, s.windowLength, s.windowStep,
                                                                     s.geo.kPad, aHi, nullptr);
    }
    else
    {
        dim3 pg(std::min<uint32_t>((s.geo.clipStride / 8 + 255) / 256 + 1, 64u), std::min(s.n, 65535));
        if (s.fmt == kTcTf32) tc_prep_kernel<kTcTf32><<<pg, 256, 0, h.stream()>>>(p, aHi, nullptr, s.geo.clipStride);
        else if (s.fmt == kTcBf16x3)
            tc_prep_kernel<kTcBf16x3><<<pg, 256, 0, h.stream()>>>(p, aHi, aLo, s.geo.clipStride);
        else tc_prep_kernel<kTcBf16><<<pg, 256, 0, h.stream()>>>(p, aHi, nullptr, s.geo.clipStride);
    }
    count_launch(1);
    const int chunks = s.nfft / kTileN;
    launch_ragged_prefix(TcCount{frames, chunks}, s.n, prefix, h.stream());

    TcOperands op;
    op.a = aHi;
    op.aLo = aLo;
    op.rowStep = s.geo.rowStep;
    op.clipStride = s.geo.clipStride;
    op.rowsPerClip = std::max(s.maxFrames, 1);
    op.b = s.basis;
    op.bLo = s.fmt == kTcBf16x3 ? static_cast<const unsigned char*>(s.basis) + size_t(s.nfft) * s.geo.kPad * 2 : nullptr;
    op.bRows = s.nfft;
    TcArgs a;
    a.kPad = s.geo.kPad;
    a.nfft = s.nfft;
    a.invScale = invScale;
    a.maxFrames = std::max(s.maxFrames, 1);
    a.dst = s.dst;
    a.dstNStride = s.dstNStride;
    a.dstHStride = s.dstHStride;
    a.nft = s.nft;
    a.power = s.power;
    a.frames = frames;
    a.n = s.n;
    a.errorWord = h.device_flags();
    a.validN = 0;
    switch (s.fmt)
    {
    case kTcBf16: launch_format<kTcBf16>(h, a, op, prefix); break;
    case kTcBf16x3: launch_format<kTcBf16x3>(h, a, op, prefix); break;
    case kTcTf32: launch_format<kTcTf32>(h, a, op, prefix); break;
    default: launch_format<kTcFp8>(h, a, op, prefix); break;
    }
}

}  // namespace rppb

namespace rppb {

namespace {
int mel_kpad(int fmt, int bins)
{
    const int blockK = kRowBytes / elem_bytes(fmt);
    return (bins + blockK - 1) / blockK * blockK;
}
}  // namespace

size_t tc_mel_scratch_bytes(int n, int fmt, int bins, int maxFrames)
{
    const int kPad = mel_kpad(fmt, bins);
    const size_t e = elem_bytes(fmt);
    const size_t rows = size_t(n) * std::max(maxFrames, 1);
    Carver cv(nullptr);
    cv.take<long long>(n + 1);
    cv.take<int>(n);
    cv.take<float>(1);
    cv.take<char>(size_t(kMelN) * kPad * e * (fmt == kTcBf16x3 ? 2 : 1));
    cv.take<char>(rows * kPad * e);
    if (fmt == kTcBf16x3) cv.take<char>(rows * kPad * e);
    cv.take<float>(rows);
    return cv.used();
}

void launch_tc_mel(Handle& h, void* scratch, const TcMelArgs& s)
{
    if (s.n <= 0) return;
    const int kPad = mel_kpad(s.fmt, s.bins);
    const size_t e = elem_bytes(s.fmt);
    const int maxFrames = std::max(s.maxFrames, 1);
    const size_t rows = size_t(s.n) * maxFrames;
    Carver cv(scratch);
    long long* prefix = cv.take<long long>(s.n + 1);
    int* frames = cv.take<int>(s.n);
    float* bScale = cv.take<float>(1);
    const size_t bBytes = size_t(kMelN) * kPad * e;
    unsigned char* bOp = cv.take<unsigned char>(bBytes * (s.fmt == kTcBf16x3 ? 2 : 1));
    unsigned char* aHi = cv.take<unsigned char>(rows * kPad * e);
    unsigned char* aLo = s.fmt == kTcBf16x3 ? cv.take<unsigned char>(rows * kPad * e) : nullptr;
    float* invScale = cv.take<float>(rows);

    // dense weights (one CTA) in the operand format
    MelWeightArgs w{s.mel, (s.bins - 1) * 2, s.bins, kPad, s.fmt, bOp, bScale};
    const int nf = s.mel.numFilter;
    size_t tbl = 16 + size_t(2 * (nf + 2)) * 4 + size_t(nf) * 4;
    tbl = ((tbl + 7) & ~size_t(7)) + size_t(2 * (nf + 1)) * 8 + size_t(s.bins) * 4;
    if (tbl > 200 * 1024) fail(RPP_ERROR_OUT_OF_BOUND_SHARED_MEMORY_SIZE, "mel tables too large");
    check_cuda(cudaFuncSetAttribute(mel_weights_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tbl)),
               "cudaFuncSetAttribute(mel_weights_kernel)");
    if (s.fmt != kTcFp8) check_cuda(cudaMemsetAsync(bScale, 0, sizeof(float), h.stream()), "memset(bScale)");
    mel_weights_kernel<<<1, 256, tbl, h.stream()>>>(w);
    count_launch(1);
    mel_frames_kernel<<<(s.n + 255) / 256, 256, 0, h.stream()>>>(s.dims, s.n, maxFrames, frames);
    count_launch(1);
    MelPrepArgs p{s.src, s.srcNStride, s.srcHStride, s.bins, kPad, maxFrames, s.fmt, s.n, frames, aHi, aLo, invScale,
                  bScale};
    if (s.fmt == kTcFp8)
    {
        dim3 g(std::min((maxFrames + 255) / 256, 64), std::min(s.n, 65535));
        mel_frame_scale_kernel<<<g, 256, 0, h.stream()>>>(p);
        count_launch(1);
    }
    dim3 pg((maxFrames + 31) / 32, (kPad + 31) / 32, std::min(s.n, 65535));
    mel_prep_kernel<<<pg, 256, 0, h.stream()>>>(p);
    count_launch(1);
    launch_ragged_prefix(TcCount{frames, 1}, s.n, prefix, h.stream());

    TcOperands op;
    op.a = aHi;
    op.aLo = aLo;
    op.rowStep = uint32_t(kPad);
    op.clipStride = uint32_t(size_t(maxFrames) * kPad);
    op.rowsPerClip = maxFrames;
    op.b = bOp;
    op.bLo = s.fmt == kTcBf16x3 ? bOp + bBytes : nullptr;
    op.bRows = kMelN;
    TcArgs a;
    a.kPad = kPad;
    a.nfft = kMelN;          // one 256-column chunk
    a.invScale = invScale;
    a.maxFrames = maxFrames;
    a.dst = s.dst;
    a.dstNStride = s.dstNStride;
    a.dstHStride = s.dstHStride;
    a.nft = true;
    a.power = 2;
    a.frames = frames;
    a.n = s.n;
    a.errorWord = h.device_flags();
    a.validN = nf;
    switch (s.fmt)
    {
    case kTcBf16: launch_format<kTcBf16, kEpiLinear>(h, a, op, prefix); break;
    case kTcBf16x3: launch_format<kTcBf16x3, kEpiLinear>(h, a, op, prefix); break;
    case kTcTf32: launch_format<kTcTf32, kEpiLinear>(h, a, op, prefix); break;
    default: launch_format<kTcFp8, kEpiLinear>(h, a, op, prefix); break;
    }
}

}  // namespace rppb
