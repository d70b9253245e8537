// Mono value of one interleaved multi-channel frame, in the reference's down-mixing order
// (src/modules/tensor/cpu/kernel/down_mixing.cpp:42-117): channels in SIMD groups (4 lanes below 8
// channels, 8 lanes from 8 up) whose lane sums fold in rpp_hsum_ps order
// (src/include/common/cpu/rpp_cpu_simd_math.hpp:846-867), then the leftover channels one by one.
// Shared by the down_mixing kernel and the fused down-mix + resample kernel, so both give the
// same bits.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace rppb {

struct MonoMix
{
    const float* x;   // interleaved [frames][C]
    int C;
    float wc;         // weight of every channel: 1/C, normalized to sum 1 when requested

    // Channel weight as the reference computes it (down_mixing.cpp:57-69).
    __device__ __forceinline__ static float weight(int C, bool normalize)
    {
        const float w0 = __fdiv_rn(1.f, float(C));
        if (!normalize) return w0;
        float sum = 0.0f;
        for (int c = 0; c < C; ++c) sum = __fadd_rn(sum, w0);
        return __fmul_rn(w0, __double2float_rn(__ddiv_rn(1.0, double(sum))));
    }

    __device__ __forceinline__ float operator()(long long t) const
    {
        if (C == 1) return __ldg(RPPB_RD(x + t));
        const float* xs = x + t * C;
        if (C == 2)   // fewer than 4 channels: the SIMD part sums nothing
            return __fadd_rn(__fadd_rn(0.f, __fmul_rn(__ldg(RPPB_RD(xs)), wc)), __fmul_rn(__ldg(RPPB_RD(xs + 1)), wc));
        const int lanes = C > 7 ? 8 : 4;
        const int aligned = (C / lanes) * lanes;
        float p[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int g = 0; g < aligned; g += lanes)
            for (int l = 0; l < lanes; ++l) p[l] = __fadd_rn(p[l], __fmul_rn(__ldg(RPPB_RD(xs + g + l)), wc));
        float acc = lanes == 8 ? __fadd_rn(__fadd_rn(__fadd_rn(p[0], p[4]), __fadd_rn(p[2], p[6])),
                                           __fadd_rn(__fadd_rn(p[1], p[5]), __fadd_rn(p[3], p[7])))
                               : __fadd_rn(__fadd_rn(p[0], p[1]), __fadd_rn(p[2], p[3]));
        for (int c = aligned; c < C; ++c) acc = __fadd_rn(acc, __fmul_rn(__ldg(RPPB_RD(xs + c)), wc));
        return acc;
    }
};

}  // namespace rppb
