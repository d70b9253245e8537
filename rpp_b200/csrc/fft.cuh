// Register-resident FFT building blocks for the spectrogram kernels.
//
// An M-point complex FFT (M = nfft/2; the real nfft-point input is packed as
// z[n] = x[2n] + i x[2n+1]) is split as M = R1 * R2 (four-step / Cooley-Tukey):
//   stage 1: thread j < R2 holds z[j + R2*m], m < R1, does an R1-point DFT in registers and
//            multiplies output k1 by W_M^(j*k1);
//   stage 2: thread k1 takes the R2 values (j, k1) through shared memory and does an R2-point
//            DFT in registers, giving Z[k1 + R1*k2].
// The in-register DFTs are radix-2 decimation-in-time recursions fully unrolled at compile
// time; their twiddles are compile-time constants (computed below in double precision and
// rounded once to float), with the multiplications by 1, -i and (1 -/+ i)/sqrt(2) specialised.
#pragma once

#include <cuda_runtime.h>

namespace rppb {
namespace fft {

// ---- compile-time cos/sin of 2*pi*k/n (own Taylor evaluation after exact octant reduction)
constexpr double kPi = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double taylor_sin(double x)
{
    double x2 = x * x, term = x, sum = x;
    for (int i = 1; i < 14; ++i)
    {
        term *= -x2 / double((2 * i) * (2 * i + 1));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double taylor_cos(double x)
{
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int i = 1; i < 14; ++i)
    {
        term *= -x2 / double((2 * i - 1) * (2 * i));
        sum += term;
    }
    return sum;
}
// cos(2*pi*k/n) and sin(2*pi*k/n) with the angle reduced to [0, pi/4] using integer octants
__host__ __device__ constexpr double cos_2pi(long k, long n)
{
    k %= n;
    if (k < 0) k += n;
    // 8k/n octant index; r = k/n - oct/8 in [0, 1/8)
    long num = 8 * k;
    long oct = num / n;
    double r = double(num - oct * n) / double(8 * n);   // fraction of a full turn within the octant
    double a = 2.0 * kPi * r;                            // [0, pi/4)
    double b = kPi / 4.0 - a;                            // (0, pi/4]
    switch (oct)
    {
        case 0: return taylor_cos(a);
        case 1: return taylor_sin(b);
        case 2: return -taylor_sin(a);
        case 3: return -taylor_cos(b);
        case 4: return -taylor_cos(a);
        case 5: return -taylor_sin(b);
        case 6: return taylor_sin(a);
        default: return taylor_cos(b);
    }
}

template <int K, int R>
struct Tw
{
    // W_R^K = exp(-2*pi*i*K/R) = c - i*s
    static constexpr float c = float(cos_2pi(K, R));
    static constexpr float s = float(cos_2pi(4 * K - R, 4 * R));   // sin(t) = cos(t - pi/2)
};

// Paired FP32 arithmetic (sm_100 add/sub/mul.rn.f32x2): one instruction for both components,
// each rounded as the scalar operation would be.  The assembler may still contract a paired
// multiply whose only use is a paired add into a fused multiply-add, so code that must round the
// product and the sum separately (the mel sums, which replay the reference) uses __fmul_rn and
// __fadd_rn instead.
#define RPPB_F32X2(NAME, OP)                                                                               \
    __device__ __forceinline__ float2 NAME(float2 a, float2 b)                                             \
    {                                                                                                      \
        float2 r;                                                                                          \
        asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t" OP \
            " pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"                                               \
            : "=f"(r.x), "=f"(r.y)                                                                         \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                                     \
        return r;                                                                                          \
    }
RPPB_F32X2(add2, "add.rn.f32x2")
RPPB_F32X2(sub2, "sub.rn.f32x2")
RPPB_F32X2(mul2, "mul.rn.f32x2")
#undef RPPB_F32X2

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return add2(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return sub2(a, b); }
// a * (c - i s)
__device__ __forceinline__ float2 cmul_conj(float2 a, float c, float s)
{
    return make_float2(fmaf(a.x, c, a.y * s), fmaf(a.y, c, -a.x * s));
}
// a * b
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

template <int K, int R>
__device__ __forceinline__ float2 twiddle_mul(float2 v)
{
    if constexpr (K == 0) return v;
    else if constexpr (4 * K == R) return make_float2(v.y, -v.x);                       // * (-i)
    else if constexpr (8 * K == R)
    {
        constexpr float h = float(0.70710678118654752440084436210485);
        return make_float2(h * (v.x + v.y), h * (v.y - v.x));                             // * (1-i)/sqrt2
    }
    else if constexpr (8 * K == 3 * R)
    {
        constexpr float h = float(0.70710678118654752440084436210485);
        return make_float2(h * (v.y - v.x), -h * (v.x + v.y));                            // * (-1-i)/sqrt2
    }
    else return cmul_conj(v, Tw<K, R>::c, Tw<K, R>::s);
}

template <int R, int K = 0>
__device__ __forceinline__ void combine(float2 (&x)[R], const float2 (&e)[R / 2], const float2 (&o)[R / 2])
{
    if constexpr (K < R / 2)
    {
        const float2 t = twiddle_mul<K, R>(o[K]);
        x[K] = cadd(e[K], t);
        x[K + R / 2] = csub(e[K], t);
        combine<R, K + 1>(x, e, o);
    }
}

// In-place forward DFT of R points held in registers, natural order in and out.
template <int R>
struct Dft
{
    __device__ __forceinline__ static void run(float2 (&x)[R])
    {
        float2 e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i)
        {
            e[i] = x[2 * i];
            o[i] = x[2 * i + 1];
        }
        Dft<R / 2>::run(e);
        Dft<R / 2>::run(o);
        combine<R>(x, e, o);
    }
};
template <>
struct Dft<1>
{
    __device__ __forceinline__ static void run(float2 (&)[1]) {}
};

}  // namespace fft
}  // namespace rppb
