// slice: copy each sample's box [anchor, anchor + shape) of a 1-D to 4-D tensor, clipped to the
// sample's roi lengths, with optional fill padding.
//
// Reference: src/modules/tensor/cpu/kernel/slice.cpp:40-60 and :197-228 (1-D, 2-D), :61-196 (3-D,
// 4-D; the host path the oracle restates).  Per sample b with numDims d (the batch excluded):
//   maxLen_k = min(shape_k, length_k - anchor_k), length_k = roi[b * 2d + d + k] (the roi begin
//   values are not read);
//   if any anchor_k + shape_k > length_k and padding is enabled, elements [0, dstStride0 - 1) of the
//   sample are set to the fill value (the last element of the sample's stride is left as it was);
//   the clipped box is copied to the start of the sample (rows of dstStride1 in 2-D).
// 3-D / 4-D: the box is taken over the spatial dims only (H, W or D, H, W).  Channel-first layouts
// (NCHW, NCDHW) copy every channel, the destination stepping by the source's channel stride between
// channels as the reference does; channel-last layouts (NHWC, NDHWC) copy rows of width x channels
// elements.  The padding test reads the spatial dims only.  Extents are also clipped to the
// destination's dims, which the caller's descriptors must nest (checked by the dispatch).
// Every destination element is written at most once: the kernel decides per element whether it
// belongs to the box (source value), to the fill range (fill value) or to neither (untouched), so
// the reference's fill-then-copy order needs no second pass.  A negative extent copies nothing (the
// reference turns it into a huge unsigned length).  HBM-bound: one read per copied element, one
// write per written element.
#include "common.cuh"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 8192;   // destination elements per work unit

template <class T>
__global__ void __launch_bounds__(kThreads) slice_kernel(SliceArgs a, const T* __restrict__ src, T* __restrict__ dst,
                                                         const T* __restrict__ fill)
{
    const long long units = (long long)a.n * a.unitsPerSample;
    const T fv = a.enablePadding ? *RPPB_RD(fill) : T(0);
    for (long long u = blockIdx.x; u < units; u += gridDim.x)
    {
        const int b = int(u / a.unitsPerSample);
        const long long i0 = (u % a.unitsPerSample) * (long long)kChunk;
        const int* an = a.anchor + b * a.numDims;
        const int* sh = a.shape + b * a.numDims;
        const int* len = reinterpret_cast<const int*>(a.roi + b * a.numDims * 2 + a.numDims);
        const unsigned rowBytes = unsigned(a.numDims) * sizeof(int);
        if (!RPPB_RANGE_OK(an, rowBytes) || !RPPB_RANGE_OK(sh, rowBytes) || !RPPB_RANGE_OK(len, rowBytes)) continue;
        bool need = false;
        int m0 = 0, m1 = 1;
        for (int k = 0; k < a.numDims; ++k)
        {
            if (an[k] + sh[k] > len[k]) need = true;
            // lengths stay inside the sample's extent; a negative anchor copies nothing
            const int ext = int(k == 0 ? a.srcDim0 : a.srcDim1);
            const int m = an[k] < 0 ? 0 : max(min(sh[k], min(len[k], ext) - an[k]), 0);
            if (k == 0) m0 = m;
            else m1 = m;
        }
        const bool pad = need && a.enablePadding;
        const T* s = src + size_t(b) * a.srcStride0;
        T* d = dst + size_t(b) * a.dstStride0;
        const long long iEnd = min(i0 + kChunk, (long long)a.dstStride0);
        if (a.numDims == 1)
        {
            const long long writeEnd = pad ? max((long long)m0, (long long)a.dstStride0 - 1) : (long long)m0;
            if (i0 >= writeEnd) continue;   // nothing of this unit is written
            const T* sa = s + an[0];
            // 4 consecutive elements per thread: one vector store when all 4 are written and aligned
            const bool vec = (a.dstStride0 & 3) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
            for (long long i = i0 + 4 * threadIdx.x; i < iEnd; i += 4 * kThreads)
            {
                T v[4];
                int written = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const long long e = i + j;
                    if (e < m0)
                    {
                        v[j] = *RPPB_RD(sa + e);
                        written |= 1 << j;
                    }
                    else if (pad && e < (long long)a.dstStride0 - 1)
                    {
                        v[j] = fv;
                        written |= 1 << j;
                    }
                }
                if (vec && written == 15 && i + 3 < iEnd)
                {
                    if constexpr (sizeof(T) == 4)
                        *RPPB_WR(reinterpret_cast<float4*>(d + i)) = make_float4(v[0], v[1], v[2], v[3]);
                    else
                        *RPPB_WR(reinterpret_cast<uchar4*>(d + i)) = make_uchar4(v[0], v[1], v[2], v[3]);
                }
                else
                {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if ((written >> j & 1) && i + j < iEnd) *RPPB_WR(d + (i + j)) = v[j];
                }
            }
        }
        else if (a.numDims >= 3)
        {
            // the box as up to four nested levels (outermost first) of (count, source stride,
            // destination stride); every destination element is decoded into level indices
            const int sp = a.numDims - 1;                  // spatial dims
            const bool first = a.layoutKind == 1;
            const int o0 = first ? 1 : 0;
            int cnt[4];
            uint32_t ss[4], ds[4];
            int nl = 0;
            bool none = false, padS = false;
            size_t base = 0;
            int m[3];
            for (int k = 0; k < sp; ++k)
            {
                const int d = o0 + k;
                if (an[d] + sh[d] > len[d]) padS = true;
                const int ext = min(len[d], int(a.srcDims[d]));
                m[k] = an[d] < 0 ? 0 : min(max(min(sh[d], ext - an[d]), 0), int(a.dstDims[d]));
                if (m[k] == 0) none = true;
            }
            const bool padN = padS && a.enablePadding;
            if (first)
            {
                cnt[nl] = int(a.srcDims[0]);
                ss[nl] = a.srcStrides[1];
                ds[nl++] = a.srcStrides[1];   // the source's channel stride, as the reference steps
                for (int k = 0; k < sp; ++k)
                {
                    const bool inner = k + 1 == sp;
                    cnt[nl] = m[k];
                    ss[nl] = inner ? 1u : a.srcStrides[o0 + k + 1];
                    ds[nl++] = inner ? 1u : a.dstStrides[o0 + k + 1];
                    if (!none) base += size_t(an[o0 + k]) * (inner ? 1u : a.srcStrides[o0 + k + 1]);
                }
            }
            else
            {
                const int C = int(a.srcDims[a.numDims - 1]);
                for (int k = 0; k < sp; ++k)
                {
                    const bool inner = k + 1 == sp;
                    cnt[nl] = inner ? m[k] * C : m[k];
                    ss[nl] = inner ? 1u : a.srcStrides[1 + k];
                    ds[nl++] = inner ? 1u : a.dstStrides[1 + k];
                    if (!none) base += size_t(an[k]) * (inner ? uint32_t(C) : a.srcStrides[1 + k]);
                }
            }
            const long long writeEnd = padN ? (long long)a.dstStride0 - 1 : (long long)a.dstStride0;
            if (none && !padN) continue;
            const T* sb = s + base;
            for (long long i = i0 + threadIdx.x; i < min(iEnd, writeEnd); i += kThreads)
            {
                uint32_t rem = uint32_t(i);
                bool in = !none;
                size_t off = 0;
                for (int l = 0; l < nl; ++l)
                {
                    const uint32_t q = ds[l] == 1u ? rem : rem / ds[l];
                    rem -= q * ds[l];
                    in = in && q < uint32_t(cnt[l]);
                    off += size_t(q) * ss[l];
                }
                if (in) *RPPB_WR(d + i) = *RPPB_RD(sb + off);
                else if (padN) *RPPB_WR(d + i) = fv;
            }
        }
        else
        {
            for (long long i = i0 + threadIdx.x; i < iEnd; i += kThreads)
            {
                const uint32_t r = uint32_t(i) / a.dstStride1, c = uint32_t(i) - r * a.dstStride1;
                if (r < uint32_t(m0) && c < uint32_t(m1))
                    *RPPB_WR(d + i) = *RPPB_RD(s + ((size_t)(an[0] + r) * a.srcStride1 + an[1] + c));
                else if (pad && i < (long long)a.dstStride0 - 1) *RPPB_WR(d + i) = fv;
            }
        }
    }
}

}  // namespace

void launch_slice(Handle& h, const SliceArgs& a, const void* src, void* dst, const void* fill)
{
    if (a.n <= 0 || a.dstStride0 == 0) return;
    SliceArgs b = a;
    b.unitsPerSample = int((size_t(a.dstStride0) + kChunk - 1) / kChunk);
    const long long units = (long long)b.n * b.unitsPerSample;
    if (a.elemBytes == 1)
    {
        const int grid = int(std::min<long long>(units, persistent_grid(h, reinterpret_cast<const void*>(
                                                                              slice_kernel<unsigned char>),
                                                                          kThreads, 0)));
        slice_kernel<unsigned char><<<grid, kThreads, 0, h.stream()>>>(b, static_cast<const unsigned char*>(src),
                                                                      static_cast<unsigned char*>(dst),
                                                                      static_cast<const unsigned char*>(fill));
    }
    else
    {
        const int grid = int(std::min<long long>(
            units, persistent_grid(h, reinterpret_cast<const void*>(slice_kernel<float>), kThreads, 0)));
        slice_kernel<float><<<grid, kThreads, 0, h.stream()>>>(b, static_cast<const float*>(src),
                                                              static_cast<float*>(dst),
                                                              static_cast<const float*>(fill));
    }
    count_launch(1);
    check_cuda(cudaGetLastError(), "slice_kernel");
}

}  // namespace rppb
