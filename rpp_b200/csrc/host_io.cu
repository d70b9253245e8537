// PCIe movers of the host-tensor front end (rppb_frontend_host_gpu): kernels that read pinned host
// memory (mapped into the device address space) and write it, so that one launch moves a whole chunk
// of ragged clips.  One DMA copy per clip costs a few microseconds of setup each; a kernel keeps
// thousands of 16-byte PCIe requests in flight and moves only the valid part of every clip.
//
// Both kernels run on their own streams next to the persistent front-end kernel, which leaves them
// a few SMs (FrontendArgs::reserveSms).
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kMoverThreads = 256;
constexpr int kSegment = 8192;   // floats per (clip, segment) work unit of the gather

// dst[b][0 .. cnt_b) = src[(c0 + b) * nStride ..], cnt_b = min(nStride, max(len_b, 2), dstStride):
// the valid samples of each clip plus the second sample, which the REFLECT pre-emphasis border reads.
__global__ void __launch_bounds__(kMoverThreads) host_gather_kernel(const float* __restrict__ src, size_t nStride,
                                                                    const int* __restrict__ len, int clips,
                                                                    float* __restrict__ dst, uint32_t dstStride,
                                                                    int segsPerClip)
{
    const long long units = (long long)clips * segsPerClip;
    for (long long u = blockIdx.x; u < units; u += gridDim.x)
    {
        const int b = int(u / segsPerClip), seg = int(u % segsPerClip);
        const long long cnt = min(min((long long)nStride, (long long)max(*RPPB_RD(len + b), 2)), (long long)dstStride);
        const long long s0 = (long long)seg * kSegment;
        if (s0 >= cnt) continue;
        const int m = int(min((long long)kSegment, cnt - s0));
        const float* s = src + size_t(b) * nStride + s0;
        float* d = dst + size_t(b) * dstStride + s0;
        if (((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d)) & 15) == 0)
        {
            // the warps' loads follow the 128-byte lines of the host row: the samples before the first
            // line boundary (a multiple of 4, at most 28) go one per thread, the rest 16 bytes per
            // thread from the boundary on, so each warp load reads 4 whole lines rather than parts of 5
            const int head = min(m, int(((128u - unsigned(reinterpret_cast<uintptr_t>(s) & 127u)) & 127u) >> 2));
            if (int(threadIdx.x) < head) *RPPB_WR(d + threadIdx.x) = *RPPB_RD(s + threadIdx.x);
            const float* sa = s + head;
            float* da = d + head;
            const int ma = m - head;
            const int q = ma >> 2;
            const float4* s4 = reinterpret_cast<const float4*>(sa);
            float4* d4 = reinterpret_cast<float4*>(da);
            // 8 loads in flight per thread before the stores
            constexpr int kUnroll = kSegment / 4 / kMoverThreads;
            float4 v[kUnroll];
#pragma unroll
            for (int k = 0; k < kUnroll; ++k)
            {
                const int i = threadIdx.x + k * kMoverThreads;
                if (i < q) v[k] = *RPPB_RD(s4 + i);
            }
#pragma unroll
            for (int k = 0; k < kUnroll; ++k)
            {
                const int i = threadIdx.x + k * kMoverThreads;
                if (i < q) *RPPB_WR(d4 + i) = v[k];
            }
            for (int i = (q << 2) + threadIdx.x; i < ma; i += kMoverThreads) *RPPB_WR(da + i) = *RPPB_RD(sa + i);
        }
        else
        {
            for (int i = threadIdx.x; i < m; i += kMoverThreads) *RPPB_WR(d + i) = *RPPB_RD(s + i);
        }
    }
}

// dst[(c0 + b) * dstNStride + r * dstHStride + f] = src[b * srcNStride + r * srcHStride + f] for
// rows r < rows and frames f < frames_b: one warp per row, each store one 128-byte line of dst.
__global__ void __launch_bounds__(kMoverThreads) host_scatter_kernel(const float* __restrict__ src, uint32_t srcNStride,
                                                                     uint32_t srcHStride,
                                                                     const int* __restrict__ frames, int clips,
                                                                     int rows, float* __restrict__ dst,
                                                                     size_t dstNStride, size_t dstHStride)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (kMoverThreads / 32);
    const long long total = (long long)clips * rows;
    for (long long w = blockIdx.x * (long long)(kMoverThreads / 32) + (threadIdx.x >> 5); w < total; w += warps)
    {
        const int b = int(w / rows), r = int(w % rows);
        const int F = *RPPB_RD(frames + b);
        const float* s = src + size_t(b) * srcNStride + size_t(r) * srcHStride;
        float* d = dst + size_t(b) * dstNStride + size_t(r) * dstHStride;
        // the warp's stores follow the 128-byte lines of the destination row: lane l first takes frame
        // l - head (when that is >= 0), the rest of the line that d[0] lies in, so every later store
        // of the warp fills one whole line (one PCIe write rather than two partial ones)
        const int head = int((reinterpret_cast<uintptr_t>(d) >> 2) & 31);
        int f = lane - head;
        if (f >= 0 && f < F) *RPPB_WR(d + f) = *RPPB_RD(s + f);
        f += 32;
        for (; f + 96 < F; f += 128)
        {
            const float v0 = *RPPB_RD(s + f), v1 = *RPPB_RD(s + (f + 32)), v2 = *RPPB_RD(s + (f + 64)),
                        v3 = *RPPB_RD(s + (f + 96));
            *RPPB_WR(d + f) = v0;
            *RPPB_WR(d + (f + 32)) = v1;
            *RPPB_WR(d + (f + 64)) = v2;
            *RPPB_WR(d + (f + 96)) = v3;
        }
        for (; f < F; f += 32) *RPPB_WR(d + f) = *RPPB_RD(s + f);
    }
}

// A list of contiguous copies (host pinned <-> device, or device <-> device) done by one launch:
// job j moves jobs[j].count floats from jobs[j].src to jobs[j].dst, split into segments of kSegment
// floats numbered from jobs[j].unit0 (an exclusive scan of the segment counts, so the grid walks a
// flat list of segments); 16-byte loads and stores where both ends are 16-byte aligned.  The job list
// itself may sit in pinned host memory.
__global__ void __launch_bounds__(kMoverThreads) copy_jobs_kernel(const CopyJob* __restrict__ jobs, int njobs,
                                                                  long long units)
{
    for (long long u = blockIdx.x; u < units; u += gridDim.x)
    {
        int lo = 0, hi = njobs - 1;   // last job with unit0 <= u
        while (lo < hi)
        {
            const int mid = (lo + hi + 1) >> 1;
            if (RPPB_RD(jobs + mid)->unit0 <= u) lo = mid;
            else hi = mid - 1;
        }
        const CopyJob jb = *RPPB_RD(jobs + lo);
        const long long s0 = (u - jb.unit0) * kSegment;
        if (s0 >= jb.count) continue;
        const int m = int(min((long long)kSegment, jb.count - s0));
        const float* s = jb.src + s0;
        float* d = jb.dst + s0;
        if (((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(d)) & 15) == 0)
        {
            const int q = m >> 2;
            const float4* s4 = reinterpret_cast<const float4*>(s);
            float4* d4 = reinterpret_cast<float4*>(d);
            constexpr int kUnroll = kSegment / 4 / kMoverThreads;
            float4 v[kUnroll];
#pragma unroll
            for (int k = 0; k < kUnroll; ++k)
            {
                const int i = threadIdx.x + k * kMoverThreads;
                if (i < q) v[k] = *RPPB_RD(s4 + i);
            }
#pragma unroll
            for (int k = 0; k < kUnroll; ++k)
            {
                const int i = threadIdx.x + k * kMoverThreads;
                if (i < q) *RPPB_WR(d4 + i) = v[k];
            }
            for (int i = (q << 2) + threadIdx.x; i < m; i += kMoverThreads) *RPPB_WR(d + i) = *RPPB_RD(s + i);
        }
        else
        {
            for (int i = threadIdx.x; i < m; i += kMoverThreads) *RPPB_WR(d + i) = *RPPB_RD(s + i);
        }
    }
}

}  // namespace

long long copy_job_segments(long long count) { return (count + kSegment - 1) / kSegment; }

void launch_copy_jobs(cudaStream_t stream, const CopyJob* jobs, int njobs, long long units, int ctas)
{
    if (njobs <= 0 || units <= 0) return;
    copy_jobs_kernel<<<ctas, kMoverThreads, 0, stream>>>(jobs, njobs, units);
    count_launch(1);
    check_cuda(cudaGetLastError(), "copy_jobs_kernel");
}

void launch_host_gather(cudaStream_t stream, const float* src, size_t nStride, const int* len, int clips, float* dst,
                        uint32_t dstStride, int ctas)
{
    if (clips <= 0) return;
    const int segs = int((size_t(dstStride) + kSegment - 1) / kSegment);
    host_gather_kernel<<<ctas, kMoverThreads, 0, stream>>>(src, nStride, len, clips, dst, dstStride, std::max(segs, 1));
    count_launch(1);
    check_cuda(cudaGetLastError(), "host_gather_kernel");
}

void launch_host_scatter(cudaStream_t stream, const float* src, uint32_t srcNStride, uint32_t srcHStride,
                         const int* frames, int clips, int rows, float* dst, size_t dstNStride, size_t dstHStride,
                         int ctas)
{
    if (clips <= 0 || rows <= 0) return;
    host_scatter_kernel<<<ctas, kMoverThreads, 0, stream>>>(src, srcNStride, srcHStride, frames, clips, rows, dst,
                                                            dstNStride, dstHStride);
    count_launch(1);
    check_cuda(cudaGetLastError(), "host_scatter_kernel");
}

}  // namespace rppb
