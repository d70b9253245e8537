// ORACLE — test infrastructure only.  Plain-argument entry points around the reference's own
// host audio library (built from the reference sources by oracle/build_ref.sh), so that
// Python's ctypes can drive it: handle creation with an explicit thread count and the resample
// call, whose RpptResamplingWindow& argument (api/rppdefs.h:751-790) holds a std::vector and
// __m128 members that ctypes cannot build.  Compiled against the reference headers.
#include <vector>

#include "rpp.h"
#include "rppdefs.h"
#include "rppt_tensor_audio_augmentations.h"
#include "handle.hpp"
#include "host_tensor_executors.hpp"
#include "rppi_validate.hpp"

extern "C" {

// rppCreate with the host backend (api/rpp.h:132).  numThreads must be explicit: 0 means
// "batch size" threads in the reference (src/modules/handle_host.cpp:57-59).
__attribute__((visibility("default"))) void* ref_create(size_t batchSlots, unsigned numThreads)
{
    rppHandle_t h = nullptr;
    if (rppCreate(&h, batchSlots, numThreads, nullptr, RPP_HOST_BACKEND) != rppStatusSuccess) return nullptr;
    return h;
}

__attribute__((visibility("default"))) int ref_destroy(void* h)
{
    return rppDestroy(static_cast<rppHandle_t>(h), RPP_HOST_BACKEND);
}

// rppt_resample_host (api/rppt_tensor_audio_augmentations.h:292) with the window given as its
// lookup table and the scale/center/lobes/coeffs fields the reference's windowed_sinc sets
// (utilities/test_suite/rpp_test_suite_audio.h:401-430).
__attribute__((visibility("default"))) int ref_resample(float* src, RpptDesc* srcDesc, float* dst, RpptDesc* dstDesc,
                                                        float* inRate, float* outRate, int* srcDims, const float* lut,
                                                        int lutSize, float scale, float center, int lobes, int coeffs,
                                                        void* h)
{
    RpptResamplingWindow w;
    w.lookup.assign(lut, lut + lutSize);
    w.lookupSize = lutSize;
    w.scale = scale;
    w.center = center;
    w.lobes = lobes;
    w.coeffs = coeffs;
    w.pCenter = _mm_set1_ps(center);
    w.pScale = _mm_set1_ps(scale);
    return rppt_resample_host(src, srcDesc, dst, dstDesc, inRate, outRate, srcDims, w, static_cast<rppHandle_t>(h));
}

// The reference's host slice (src/modules/tensor/cpu/kernel/slice.cpp:27-238), called at the
// kernel level: rppt_slice_host lives in the geometric-augmentations dispatch file, which pulls in
// every image kernel.  The 1-D and 2-D cases read no layout parameters.
__attribute__((visibility("default"))) int ref_slice_f32(float* src, RpptGenericDesc* srcDesc, float* dst,
                                                         RpptGenericDesc* dstDesc, int* anchor, int* shape, float* fill,
                                                         bool enablePadding, unsigned* roi, void* h)
{
    RppLayoutParams lp{};
    rpp::Handle& handle = *static_cast<rpp::Handle*>(static_cast<rppHandle_t>(h));
    return slice_host_tensor<Rpp32f>(src, srcDesc, dst, dstDesc, anchor, shape, fill, enablePadding, roi, lp, handle);
}

__attribute__((visibility("default"))) int ref_slice_u8(unsigned char* src, RpptGenericDesc* srcDesc, unsigned char* dst,
                                                        RpptGenericDesc* dstDesc, int* anchor, int* shape,
                                                        unsigned char* fill, bool enablePadding, unsigned* roi, void* h)
{
    RppLayoutParams lp{};
    rpp::Handle& handle = *static_cast<rpp::Handle*>(static_cast<rppHandle_t>(h));
    return slice_host_tensor<Rpp8u>(src, srcDesc, dst, dstDesc, anchor, shape, fill, enablePadding, roi, lp, handle);
}

// The same with the layout parameters rppt_slice_host derives from the source descriptor
// (src/modules/tensor/rppt_tensor_geometric_augmentations.cpp:1074-1082), for 3-D and 4-D tensors.
static RppLayoutParams slice_layout(const RpptGenericDesc* d)
{
    RppLayoutParams lp{};
    if (d->layout == RpptLayout::NCDHW) lp = get_layout_params(d->layout, d->dims[1]);
    else if (d->layout == RpptLayout::NDHWC) lp = get_layout_params(d->layout, d->dims[4]);
    else if (d->layout == RpptLayout::NCHW) lp = get_layout_params(d->layout, d->dims[1]);
    else if (d->layout == RpptLayout::NHWC) lp = get_layout_params(d->layout, d->dims[3]);
    return lp;
}

__attribute__((visibility("default"))) int ref_slice_nd_f32(float* src, RpptGenericDesc* srcDesc, float* dst,
                                                            RpptGenericDesc* dstDesc, int* anchor, int* shape,
                                                            float* fill, bool enablePadding, unsigned* roi, void* h)
{
    rpp::Handle& handle = *static_cast<rpp::Handle*>(static_cast<rppHandle_t>(h));
    return slice_host_tensor<Rpp32f>(src, srcDesc, dst, dstDesc, anchor, shape, fill, enablePadding, roi,
                                     slice_layout(srcDesc), handle);
}

__attribute__((visibility("default"))) int ref_slice_nd_u8(unsigned char* src, RpptGenericDesc* srcDesc,
                                                           unsigned char* dst, RpptGenericDesc* dstDesc, int* anchor,
                                                           int* shape, unsigned char* fill, bool enablePadding,
                                                           unsigned* roi, void* h)
{
    rpp::Handle& handle = *static_cast<rpp::Handle*>(static_cast<rppHandle_t>(h));
    return slice_host_tensor<Rpp8u>(src, srcDesc, dst, dstDesc, anchor, shape, fill, enablePadding, roi,
                                    slice_layout(srcDesc), handle);
}

// The reference's host normalize for F32 (src/modules/tensor/cpu/kernel/normalize.cpp:507-767),
// called at the kernel level for the same reason as slice; the 2-D branch reads no layout
// parameters.
// The layout parameters rppt_normalize_host derives (src/modules/tensor/rppt_tensor_statistical_operations.cpp:
// 259-266) and the host normalize on them: F32 at any rank, and the generic path for U8 -> U8 and
// I8 (written through an unsigned pointer, as the reference dispatch does).
static RppLayoutParams normalize_layout(const RpptGenericDesc* s, const RpptGenericDesc* d)
{
    RppLayoutParams lp{};
    const unsigned tensorDim = s->numDims - 1;
    if (tensorDim == 3 && s->layout == RpptLayout::NHWC) lp = get_layout_params(s->layout, s->dims[3]);
    else if (s->layout == RpptLayout::NCDHW && d->layout == RpptLayout::NCDHW) lp = get_layout_params(s->layout, s->dims[1]);
    else if (s->layout == RpptLayout::NDHWC && d->layout == RpptLayout::NDHWC) lp = get_layout_params(s->layout, s->dims[4]);
    else if (tensorDim == 2 && s->layout == RpptLayout::NHWC) lp = get_layout_params(s->layout, s->dims[2]);
    return lp;
}

__attribute__((visibility("default"))) int ref_normalize_nd(void* src, RpptGenericDesc* srcDesc, void* dst,
                                                            RpptGenericDesc* dstDesc, unsigned axisMask, float* mean,
                                                            float* stdDev, unsigned char computeMeanStddev,
                                                            float scale, float shift, unsigned* roi, void* h)
{
    rpp::Handle& handle = *static_cast<rpp::Handle*>(static_cast<rppHandle_t>(h));
    const RppLayoutParams lp = normalize_layout(srcDesc, dstDesc);
    if (srcDesc->dataType == RpptDataType::F32)
        return normalize_f32_f32_host_tensor(static_cast<Rpp32f*>(src), srcDesc, static_cast<Rpp32f*>(dst), dstDesc,
                                             axisMask, mean, stdDev, computeMeanStddev, scale, shift, roi, lp, handle);
    if (srcDesc->dataType == RpptDataType::U8)
        return normalize_generic_host_tensor(static_cast<Rpp8u*>(src), srcDesc, static_cast<Rpp8u*>(dst), dstDesc,
                                             axisMask, mean, stdDev, computeMeanStddev, scale, shift, roi, lp, handle);
    if (srcDesc->dataType == RpptDataType::I8)
        return normalize_generic_host_tensor(static_cast<Rpp8s*>(src), srcDesc, static_cast<Rpp8u*>(dst), dstDesc,
                                             axisMask, mean, stdDev, computeMeanStddev, scale, shift, roi, lp, handle);
    return -1;
}

__attribute__((visibility("default"))) int ref_normalize_f32(float* src, RpptGenericDesc* srcDesc, float* dst,
                                                             RpptGenericDesc* dstDesc, unsigned axisMask, float* mean,
                                                             float* stdDev, unsigned char computeMeanStddev, float scale,
                                                             float shift, unsigned* roi, void* h)
{
    RppLayoutParams lp{};
    rpp::Handle& handle = *static_cast<rpp::Handle*>(static_cast<rppHandle_t>(h));
    return normalize_f32_f32_host_tensor(src, srcDesc, dst, dstDesc, axisMask, mean, stdDev, computeMeanStddev, scale,
                                         shift, roi, lp, handle);
}
}
