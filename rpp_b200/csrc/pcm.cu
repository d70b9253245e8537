// 16-bit PCM ingest: int16 samples (interleaved channels) -> float32 / 32768, the conversion the
// reference's audio test suite applies when it reads WAV files
// (utilities/test_suite/rpp_test_suite_audio.h:143-178: libsndfile's sf_read_float on int16 data).
// Only each clip's valid frames x channels are converted; the destination tail is left as it was.
// x / 32768 is exact in float, so the output equals the host conversion bit for bit.  HBM-bound:
// 2 bytes read, 4 written per sample; 8 samples per thread step (16-byte loads when aligned).
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16384;   // samples per work unit

__global__ void __launch_bounds__(kThreads) pcm16_kernel(const short* __restrict__ src, uint32_t srcStride,
                                                         float* __restrict__ dst, uint32_t dstStride,
                                                         const int* __restrict__ len, int channels, int n,
                                                         int unitsPerSample)
{
    const long long units = (long long)n * unitsPerSample;
    for (long long u = blockIdx.x; u < units; u += gridDim.x)
    {
        const int b = int(u / unitsPerSample);
        const long long count = min((long long)max(*RPPB_RD(len + b), 0) * channels, (long long)min(srcStride, dstStride));
        const long long i0 = (u % unitsPerSample) * (long long)kChunk;
        if (i0 >= count) continue;
        const long long i1 = min(i0 + kChunk, count);
        const short* s = src + size_t(b) * srcStride;
        float* d = dst + size_t(b) * dstStride;
        const bool vec = ((reinterpret_cast<uintptr_t>(s + i0) & 15) | (reinterpret_cast<uintptr_t>(d + i0) & 15)) == 0;
        long long i = i0 + 8 * threadIdx.x;
        if (vec)
        {
            for (; i + 8 <= i1; i += 8 * kThreads)
            {
                const int4 v = *RPPB_RD(reinterpret_cast<const int4*>(s + i));
                const short* p = reinterpret_cast<const short*>(&v);
                const float k = 1.0f / 32768.0f;
                *RPPB_WR(reinterpret_cast<float4*>(d + i)) = make_float4(p[0] * k, p[1] * k, p[2] * k, p[3] * k);
                *RPPB_WR(reinterpret_cast<float4*>(d + i + 4)) = make_float4(p[4] * k, p[5] * k, p[6] * k, p[7] * k);
            }
        }
        for (; i < i1; i += 8 * kThreads)
            for (int j = 0; j < 8 && i + j < i1; ++j) *RPPB_WR(d + (i + j)) = float(*RPPB_RD(s + (i + j))) * (1.0f / 32768.0f);
    }
}

}  // namespace

void launch_pcm16(Handle& h, const short* src, uint32_t srcStride, float* dst, uint32_t dstStride, const int* len,
                  int channels, int n)
{
    if (n <= 0) return;
    const int ups = int((size_t(std::min(srcStride, dstStride)) + kChunk - 1) / kChunk);
    if (ups <= 0) return;
    const int grid = int(std::min<long long>((long long)n * ups,
                                             persistent_grid(h, reinterpret_cast<const void*>(pcm16_kernel), kThreads, 0)));
    pcm16_kernel<<<grid, kThreads, 0, h.stream()>>>(src, srcStride, dst, dstStride, len, channels, n, ups);
    count_launch(1);
    check_cuda(cudaGetLastError(), "pcm16_kernel");
}

}  // namespace rppb
