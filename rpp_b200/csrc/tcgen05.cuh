// Building blocks for kernels on the 5th-generation tensor cores (tcgen05, sm_100a): shared-memory
// matrix descriptors of the 128-byte-swizzled K-major operand layout, the instruction descriptor of
// a BF16 x BF16 -> FP32 MMA, MMA issue and completion tracking through an mbarrier, bounded
// mbarrier waits, and tensor-memory (TMEM) allocation and loads.
//
// Operand layout (K-major, 128-byte swizzle): a tile of R rows x 128 bytes of K is stored as R/8
// atoms of 8 rows x 128 bytes (1024 bytes each, 1024-byte aligned); byte b of row r sits at
//   (r / 8) * 1024 + (r % 8) * 128 + ((b / 16) ^ (r % 8)) * 16 + b % 16,
// i.e. the 16-byte chunks of each row are permuted by the row's index within its atom.  One MMA
// instruction of kind::f16 consumes 32 bytes (16 BF16 values) of K per row; the K step inside the
// 128-byte row is taken by advancing the descriptor's start address by 32 bytes.
#pragma once

#include <cstdint>

namespace rppb {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of byte b (0..127) of row r in a 128-byte-swizzled K-major tile.
__host__ __device__ constexpr uint32_t sw128(uint32_t r, uint32_t b)
{
    return (r >> 3) * 1024u + (r & 7u) * 128u + ((((b >> 4) ^ r) & 7u) << 4) + (b & 15u);
}

// Shared-memory matrix descriptor of a 128-byte-swizzled K-major tile starting at `saddr`
// (1024-byte aligned for the first K step): start address, leading byte offset (unused for this
// layout, 1), stride byte offset 1024 (the next 8-row atom), descriptor version 1, swizzle mode
// 128 bytes.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFF);
    d |= uint64_t(1) << 16;
    d |= uint64_t(1024 >> 4) << 32;
    d |= uint64_t(1) << 46;
    d |= uint64_t(2) << 61;
    return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B (both K-major) and an FP32 accumulator:
// accumulator format (bit 4), A format (bits 7-9), B format (bits 10-12), N / 8 (bits 17-22),
// M / 16 (bits 24-28).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// The same with F16 A and B (format 0).
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N)
{
    return (1u << 4) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// D[tmem] (+)= A[a] x B[b]^T, issued by one thread (kind::f16: BF16 or F16 operands, as the
// instruction descriptor says; both operands of one MMA have the same type).
__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// Arrives once on `bar` when every MMA this thread issued before has completed (its shared-memory
// reads and its tensor-memory writes).
__device__ __forceinline__ void commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

// Waits for the phase of `bar` with parity `parity` to complete, at most `limit` polls; false on
// timeout (the caller reports it and leaves: no wait is unbounded).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit)
{
    const uint32_t a = smem_addr(bar);
    for (long long i = 0; i < limit; ++i)
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
    }
    return false;
}

// Orders tensor-core operations around a thread synchronization (before: this thread's tcgen05 ops
// before the barrier; after: the barrier before this thread's later tcgen05 ops).
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's generic-proxy shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Allocates `cols` tensor-memory columns (a power of two >= 32) for the CTA and writes the base
// address to *dst; called by one whole warp.  The permit is relinquished so that other CTAs on the SM
// can allocate.
template <int COLS>
__device__ __forceinline__ void tmem_alloc(uint32_t* dst)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
                 "r"(COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
template <int COLS>
__device__ __forceinline__ void tmem_dealloc(uint32_t base)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(COLS));
}

// 32 consecutive 32-bit columns of this thread's TMEM lane: taddr = base + (lane quarter * 32 << 16)
// + column; warp w of the CTA may read lanes 32 * (w % 4) .. 32 * (w % 4) + 31.  Warp-collective.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : "=r"(v[0]), "=r"(v[1]) : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// (lo, hi) -> one 32-bit word of two BF16 values, each rounded to nearest even; lo in bits 0-15.
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}
// The two BF16 values of a packed word as floats (exact).
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// x = hi + lo split of two floats into BF16 words: hi = bf16(x), lo = bf16(x - hi).  hi + lo keeps
// about 16 significant bits of x.
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo)
{
    hi = pack_bf16x2(a, b);
    lo = pack_bf16x2(a - bf16_lo(hi), b - bf16_hi(hi));
}

// (lo, hi) -> one 32-bit word of two F16 values, each rounded to nearest even; lo in bits 0-15.
__device__ __forceinline__ uint32_t pack_f16x2(float lo, float hi)
{
    uint32_t d;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}
__device__ __forceinline__ void unpack_f16x2(uint32_t w, float& lo, float& hi)
{
    asm("{\n\t.reg .f16 a, b;\n\tmov.b32 {a, b}, %2;\n\tcvt.f32.f16 %0, a;\n\tcvt.f32.f16 %1, b;\n\t}"
        : "=f"(lo), "=f"(hi)
        : "r"(w));
}
// x = hi + lo split of two floats into F16 words: hi = f16(x), lo = f16(x - hi).  For |x| <= 2^15 the
// pair keeps x to about 2^-22 |x| (and 2^-25 absolute, where lo falls into the F16 subnormals).
__device__ __forceinline__ void split_f16x2(float a, float b, uint32_t& hi, uint32_t& lo)
{
    hi = pack_f16x2(a, b);
    float ha, hb;
    unpack_f16x2(hi, ha, hb);
    lo = pack_f16x2(a - ha, b - hb);
}

}  // namespace tc
}  // namespace rppb
