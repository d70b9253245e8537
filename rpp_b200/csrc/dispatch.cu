// The seven rppt_*_gpu entry points of include/rppt_tensor_audio_augmentations.h.
//
// Argument checks follow the reference's GPU dispatch
// (src/modules/tensor/rppt_tensor_audio_augmentations.cpp:332-629) in the same order and with
// the same status codes.  Beyond those, inputs on which the reference would crash, hang or write
// out of bounds return RPP_ERROR_INVALID_ARGUMENTS (null pointers, non-positive window or step,
// resetInterval 0, nfft smaller than the window).  Scalars the reference derives on the host
// (decibel minRatio and log10 factor, NSR cutoff) are derived here with the same float/double
// expressions.  Per-sample tensors are resolved to device addresses (device and pinned pointers
// are used in place; pageable ones are staged into the workspace), then the launchers of
// rpp_b200/csrc/*.cu enqueue the kernels on the handle stream.  Nothing here synchronizes the
// stream except a pageable NSR output, whose device-to-host copy is stream-ordered.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rppb_frontend.h"
#include "../../include/rppt_tensor_audio_augmentations.h"
#include "../../include/rppt_tensor_geometric_augmentations.h"
#include "../../include/rppt_tensor_statistical_operations.h"
#include "common.cuh"
#include "handle.hpp"
#include "ops.hpp"

using namespace rppb;

static_assert(sizeof(RppbFrontendParams) == 88, "RppbFrontendParams layout (rpp_b200/types.py mirrors it)");

namespace {

thread_local std::string g_last_error;

// Runs an entry point's body on its handle and turns exceptions into status codes.  In the checked build
// (check.cu) calls run one at a time, and a call's end reads its access record.
template <class F>
RppStatus guarded(rppHandle_t handle, F&& body)
{
#ifdef RPPB_CHECKED
    std::lock_guard<std::recursive_mutex> lk(check_mutex());
#endif
    Handle* hp = nullptr;
    auto abandon = [&](RppStatus st) {
#ifdef RPPB_CHECKED
        if (hp)
            try
            {
                hp->check_end(st);
            }
            catch (...)
            {
            }
#endif
        return st;
    };
    try
    {
        Handle& h = deref(handle);
        hp = &h;
        h.begin_call();
        h.check_begin();
        RppStatus st = body(h);
        hp = nullptr;
        st = h.check_end(st);
        if (st == RPP_SUCCESS) h.end_call();
        return st;
    }
    catch (const Error& e)
    {
        g_last_error = e.what;
        return abandon(e.status);
    }
    catch (const std::bad_alloc&)
    {
        g_last_error = "host allocation failed";
        return abandon(RPP_ERROR_NOT_ENOUGH_MEMORY);
    }
    catch (...)
    {
        g_last_error = "unknown error";
        return abandon(RPP_ERROR);
    }
}

inline bool is_f32(const RpptDesc* d) { return d->dataType == F32; }

void require(bool cond, const char* what)
{
    if (!cond) fail(RPP_ERROR_INVALID_ARGUMENTS, what);
}

// The bytes of a caller's tensor as its descriptor describes it (checked build: the regions of a call).
size_t elem_bytes(int dataType) { return dataType == F32 ? 4 : (dataType == F16 || dataType == I16) ? 2 : 1; }
size_t desc_bytes(const RpptDesc* d, int n)
{
    return size_t(d->offsetInBytes) + size_t(n) * d->strides.nStride * elem_bytes(d->dataType);
}
size_t desc_bytes(const RpptGenericDesc& d, int n)
{
    return size_t(d.offsetInBytes) + size_t(n) * d.strides[0] * elem_bytes(d.dataType);
}
template <class D>
void check_tensors(Handle& h, const void* src, const D& sd, const void* dst, const D& dd, int n)
{
    h.check_src(src, desc_bytes(sd, n));
    if (dst) h.check_dst(dst, desc_bytes(dd, n));
}

void build_hann(float* out, size_t count, const void*)
{
    // spectrogram.cpp:36-44: 0.5 * (1 - cos(2*pi*(t + 0.5) / W)) in FP64, rounded to float
    const double a = (2.0 * M_PI) / double(count);
    for (size_t t = 0; t < count; ++t) out[t] = float(0.5 * (1.0 - std::cos(a * (double(t) + 0.5))));
}

}  // namespace

namespace rppb {
void record_error(const std::string& what) { g_last_error = what; }
}  // namespace rppb

extern "C" SHARED_PUBLIC const char* rppbGetLastError() { return g_last_error.c_str(); }

extern "C" SHARED_PUBLIC RppStatus rppt_pre_emphasis_filter_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                                RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor,
                                                                Rpp32f* coeffTensor, RpptAudioBorderType borderType,
                                                                rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        if (srcDescPtr->numDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        Carver m(nullptr);
        m.take<int>(n);
        m.take<float>(n);
        m.take<char>(prefix_bytes(n));
        Carver cv(h.workspace(m.used()));
        int* lenStage = cv.take<int>(n);
        float* coeffStage = cv.take<float>(n);
        void* scratch = cv.take<char>(prefix_bytes(n));
        const int* len = static_cast<const int*>(h.device_view(srcLengthTensor, n * sizeof(int), lenStage));
        const float* coeff = static_cast<const float*>(h.device_view(coeffTensor, n * sizeof(float), coeffStage));
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_pre_emphasis(h, scratch, static_cast<const float*>(srcPtr), srcDescPtr->strides.nStride,
                            static_cast<float*>(dstPtr), dstDescPtr->strides.nStride, n, len, coeff, int(borderType),
                            size_t(n) * srcDescPtr->strides.nStride);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppt_down_mixing_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                        RpptDescPtr dstDescPtr, Rpp32s* srcDimsTensor,
                                                        bool normalizeWeights, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        const Rpp32u tensorDims = Rpp32u(srcDescPtr->numDims - 1);
        if (tensorDims != 1 && tensorDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        Carver m(nullptr);
        m.take<int>(2 * n);
        m.take<char>(prefix_bytes(n));
        Carver cv(h.workspace(m.used()));
        int* dimsStage = cv.take<int>(2 * n);
        void* scratch = cv.take<char>(prefix_bytes(n));
        const int* dims = static_cast<const int*>(h.device_view(srcDimsTensor, 2 * n * sizeof(int), dimsStage));
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_down_mixing(h, scratch, static_cast<const float*>(srcPtr), srcDescPtr->strides.nStride,
                           static_cast<float*>(dstPtr), dstDescPtr->strides.nStride, n, dims, normalizeWeights);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppt_to_decibels_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                        RpptDescPtr dstDescPtr, RpptImagePatchPtr srcDims,
                                                        Rpp32f cutOffDB, Rpp32f multiplier,
                                                        Rpp32f referenceMagnitude, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        const Rpp32u tensorDims = Rpp32u(srcDescPtr->numDims - 1);
        if (tensorDims != 1 && tensorDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (!multiplier) return RPP_ERROR_ZERO_DIVISION;
        if (!is_f32(srcDescPtr)) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        // to_decibels.cpp:40-45
        float minRatio = float(std::pow(10, cutOffDB / multiplier));
        if (minRatio == 0.0f) minRatio = std::nextafter(0.0f, 1.0f);
        const Rpp32f log10Factor = 0.3010299956639812;
        multiplier *= log10Factor;
        Carver m(nullptr);
        m.take<uint32_t>(2 * n);
        m.take<char>(to_decibels_scratch_bytes(n));
        Carver cv(h.workspace(m.used()));
        uint32_t* dimsStage = cv.take<uint32_t>(2 * n);
        void* scratch = cv.take<char>(to_decibels_scratch_bytes(n));
        DecibelArgs a;
        a.src = static_cast<const float*>(srcPtr);
        a.srcNStride = srcDescPtr->strides.nStride;
        a.srcHStride = srcDescPtr->strides.hStride;
        a.dst = static_cast<float*>(dstPtr);
        a.dstNStride = dstDescPtr->strides.nStride;
        a.dstHStride = dstDescPtr->strides.hStride;
        a.n = n;
        a.dims = static_cast<const uint32_t*>(h.device_view(srcDims, 2 * n * sizeof(uint32_t), dimsStage));
        a.minRatio = minRatio;
        a.multiplier = multiplier;
        a.referenceMagnitude = referenceMagnitude;
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_to_decibels(h, scratch, a);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppt_non_silent_region_detection_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr,
                                                                        Rpp32s* srcLengthTensor,
                                                                        Rpp32s* detectedIndexTensor,
                                                                        Rpp32s* detectionLengthTensor, Rpp32f cutOffDB,
                                                                        Rpp32s windowLength, Rpp32f referencePower,
                                                                        Rpp32s resetInterval, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr != nullptr, "null descriptor");
        const Rpp32u tensorDims = Rpp32u(srcDescPtr->numDims - 1);
        if (tensorDims != 1) return RPP_ERROR_INVALID_SRC_DIMS;
        if (!is_f32(srcDescPtr)) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && detectedIndexTensor && detectionLengthTensor, "null tensor");
        require(windowLength > 0, "windowLength must be positive");
        require(resetInterval == -1 || resetInterval > 0, "resetInterval must be -1 or positive");
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        const uint32_t stride = srcDescPtr->strides.nStride;
        const size_t scratchBytes = nsr_scratch_bytes(n, stride, resetInterval);
        Carver m(nullptr);
        m.take<int>(n);
        m.take<int>(2 * n);
        m.take<char>(scratchBytes);
        Carver cv(h.workspace(m.used()));
        int* lenStage = cv.take<int>(n);
        int* outStage = cv.take<int>(2 * n);
        void* scratch = cv.take<char>(scratchBytes);
        NsrArgs a;
        a.src = static_cast<const float*>(srcPtr);
        a.srcStride = stride;
        a.n = n;
        a.len = static_cast<const int*>(h.device_view(srcLengthTensor, n * sizeof(int), lenStage));
        void* dBegin = nullptr;
        void* dLength = nullptr;
        const bool directBegin = h.device_writable(detectedIndexTensor, &dBegin);
        const bool directLength = h.device_writable(detectionLengthTensor, &dLength);
        a.begin = directBegin ? static_cast<int*>(dBegin) : outStage;
        a.length = directLength ? static_cast<int*>(dLength) : outStage + n;
        a.cutOff = std::pow(10.0f, cutOffDB * 0.1f);   // non_silent_region_detection.cpp:105
        a.windowLength = windowLength;
        a.referencePower = referencePower;
        a.resetInterval = resetInterval;
        check_tensors(h, srcPtr, srcDescPtr, static_cast<const void*>(nullptr), srcDescPtr, n);
        if (directBegin) h.check_dst(a.begin, n * sizeof(int));
        if (directLength) h.check_dst(a.length, n * sizeof(int));
        launch_nsr(h, scratch, a);
        if (!directBegin)
            check_cuda(cudaMemcpyAsync(detectedIndexTensor, outStage, n * sizeof(int), cudaMemcpyDeviceToHost,
                                       h.stream()),
                       "copy NSR begin");
        if (!directLength)
            check_cuda(cudaMemcpyAsync(detectionLengthTensor, outStage + n, n * sizeof(int), cudaMemcpyDeviceToHost,
                                       h.stream()),
                       "copy NSR length");
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppt_spectrogram_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                        RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor,
                                                        bool centerWindows, bool reflectPadding,
                                                        Rpp32f* windowFunction, Rpp32s nfft, Rpp32s power,
                                                        Rpp32s windowLength, Rpp32s windowStep, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        if ((dstDescPtr->layout != NFT) && (dstDescPtr->layout != NTF)) return RPP_ERROR_INVALID_DST_LAYOUT;
        const Rpp32u srcTensorDims = Rpp32u(srcDescPtr->numDims - 1);
        const Rpp32u dstTensorDims = Rpp32u(dstDescPtr->numDims - 1);
        if (srcTensorDims != 1) return RPP_ERROR_INVALID_SRC_DIMS;
        if (dstTensorDims != 2) return RPP_ERROR_INVALID_DST_DIMS;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        require(windowLength > 0 && windowStep > 0, "windowLength and windowStep must be positive");
        if (nfft == 0) nfft = windowLength;   // spectrogram.cpp:88
        require(nfft >= windowLength, "nfft must be at least windowLength");
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        // bins must fit the destination (the reference writes them unchecked)
        const Rpp32u binsCap = dstDescPtr->layout == NFT ? dstDescPtr->h : dstDescPtr->w;
        if (binsCap < Rpp32u(nfft / 2 + 1) || dstDescPtr->strides.hStride < (dstDescPtr->layout == NFT ? dstDescPtr->w : Rpp32u(nfft / 2 + 1)))
            return RPP_ERROR_INVALID_DST_DIMS;
        Carver m(nullptr);
        m.take<int>(n);
        m.take<float>(windowFunction ? windowLength : 0);
        m.take<char>(prefix_bytes(n));
        Carver cv(h.workspace(m.used()));
        int* lenStage = cv.take<int>(n);
        float* winStage = cv.take<float>(windowFunction ? windowLength : 0);
        void* scratch = cv.take<char>(prefix_bytes(n));
        SpectrogramArgs a;
        a.src = static_cast<const float*>(srcPtr);
        a.srcStride = srcDescPtr->strides.nStride;
        a.dst = static_cast<float*>(dstPtr);
        a.dstNStride = dstDescPtr->strides.nStride;
        a.dstHStride = dstDescPtr->strides.hStride;
        a.nft = dstDescPtr->layout == NFT;
        a.n = n;
        a.len = static_cast<const int*>(h.device_view(srcLengthTensor, n * sizeof(int), lenStage));
        a.center = centerWindows;
        a.reflect = reflectPadding;
        if (windowFunction)
        {
            // the reference reads the window on the host and copies it (hip/kernel/spectrogram.cpp:264-277)
            h.upload(winStage, windowFunction, windowLength * sizeof(float));
            a.window = winStage;
        }
        else
        {
            a.window = h.table("hann" + std::to_string(windowLength), size_t(windowLength), build_hann, nullptr);
        }
        a.nfft = nfft;
        a.power = power;
        a.windowLength = windowLength;
        a.windowStep = windowStep;
        a.maxFrames = int(a.nft ? dstDescPtr->w : dstDescPtr->h);
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_spectrogram(h, scratch, a);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppt_mel_filter_bank_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                            RpptDescPtr dstDescPtr, Rpp32s* srcDimsTensor,
                                                            Rpp32f maxFreq, Rpp32f minFreq,
                                                            RpptMelScaleFormula melFormula, Rpp32s numFilter,
                                                            Rpp32f sampleRate, bool normalize, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        const Rpp32u tensorDims = Rpp32u(srcDescPtr->numDims - 1);
        if (tensorDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (srcDescPtr->layout != NFT) return RPP_ERROR_INVALID_SRC_LAYOUT;
        if (dstDescPtr->layout != NFT) return RPP_ERROR_INVALID_DST_LAYOUT;
        if (maxFreq < 0 || maxFreq > sampleRate / 2) return RPP_ERROR_INVALID_ARGUMENTS;
        if (minFreq < 0 || minFreq > sampleRate / 2) return RPP_ERROR_INVALID_ARGUMENTS;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        require(numFilter > 0, "numFilter must be positive");
        if (dstDescPtr->h < Rpp32u(numFilter)) return RPP_ERROR_INVALID_DST_DIMS;
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        Carver m(nullptr);
        m.take<int>(2 * n);
        m.take<char>(prefix_bytes(n));
        Carver cv(h.workspace(m.used()));
        int* dimsStage = cv.take<int>(2 * n);
        void* scratch = cv.take<char>(prefix_bytes(n));
        MelArgs a;
        a.src = static_cast<const float*>(srcPtr);
        a.srcNStride = srcDescPtr->strides.nStride;
        a.srcHStride = srcDescPtr->strides.hStride;
        a.dst = static_cast<float*>(dstPtr);
        a.dstNStride = dstDescPtr->strides.nStride;
        a.dstHStride = dstDescPtr->strides.hStride;
        a.n = n;
        a.dims = static_cast<const int*>(h.device_view(srcDimsTensor, 2 * n * sizeof(int), dimsStage));
        a.srcRows = srcDescPtr->h;
        a.maxFreq = maxFreq;
        a.minFreq = minFreq;
        a.htk = melFormula == HTK ? 1 : 0;
        a.numFilter = numFilter;
        a.sampleRate = sampleRate;
        a.normalize = normalize;
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_mel_filter_bank(h, scratch, a);
        return RPP_SUCCESS;
    });
}

namespace {

RppStatus resample_common(Handle& h, RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr, RpptDescPtr dstDescPtr,
                          Rpp32f* inRateTensor, Rpp32f* outRateTensor, Rpp32s* srcDimsTensor, const float* lutHost,
                          int lutSize, float scale, float center, int lobes, bool downmix, bool normalize)
{
    require(srcDescPtr && dstDescPtr, "null descriptor");
    const Rpp32u tensorDims = Rpp32u(srcDescPtr->numDims - 1);
    if (tensorDims != 1 && tensorDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
    if (!is_f32(srcDescPtr)) return RPP_ERROR_NOT_IMPLEMENTED;
    if (downmix && !is_f32(dstDescPtr)) return RPP_ERROR_NOT_IMPLEMENTED;
    require(srcPtr && dstPtr, "null tensor");
    const int n = int(srcDescPtr->n);
    if (n <= 0) return RPP_SUCCESS;
    require(lutHost != nullptr && lutSize >= 2, "resampling window has no lookup table");
    require(lobes >= 0, "negative lobes");
    require(size_t(lutSize) * sizeof(float) <= 200 * 1024, "lookup table above 200 KB");
    Carver m(nullptr);
    m.take<float>(n);
    m.take<float>(n);
    m.take<int>(2 * n);
    m.take<float>(lutSize);
    m.take<char>(prefix_bytes(n));
    Carver cv(h.workspace(m.used()));
    float* inStage = cv.take<float>(n);
    float* outStage = cv.take<float>(n);
    int* dimsStage = cv.take<int>(2 * n);
    float* lutStage = cv.take<float>(lutSize);
    void* scratch = cv.take<char>(prefix_bytes(n));
    ResampleWindowDev win;
    win.lut = static_cast<const float*>(h.device_view(lutHost, lutSize * sizeof(float), lutStage));
    win.lutSize = lutSize;
    win.scale = scale;
    win.center = center;
    win.lobes = lobes;
    check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
    launch_resample(h, scratch, static_cast<const float*>(srcPtr), srcDescPtr->strides.nStride,
                    static_cast<float*>(dstPtr), dstDescPtr->strides.nStride, n,
                    static_cast<const float*>(h.device_view(inRateTensor, n * sizeof(float), inStage)),
                    static_cast<const float*>(h.device_view(outRateTensor, n * sizeof(float), outStage)),
                    static_cast<const int*>(h.device_view(srcDimsTensor, 2 * n * sizeof(int), dimsStage)), win,
                    downmix, normalize);
    return RPP_SUCCESS;
}

}  // namespace

extern "C" SHARED_PUBLIC RppStatus rppt_resample_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                     RpptDescPtr dstDescPtr, Rpp32f* inRateTensor,
                                                     Rpp32f* outRateTensor, Rpp32s* srcDimsTensor,
                                                     RpptResamplingWindow& window, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        const float* lutHost = window.lookupPinned ? window.lookupPinned : window.lookup.data();
        require(window.lookupPinned != nullptr || int(window.lookup.size()) >= window.lookupSize,
                "lookup shorter than lookupSize");
        return resample_common(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, inRateTensor, outRateTensor, srcDimsTensor,
                               lutHost, window.lookupSize, window.scale, window.center, window.lobes, false, false);
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_downmix_resample_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                             RpptDescPtr dstDescPtr, Rpp32f* inRateTensor,
                                                             Rpp32f* outRateTensor, Rpp32s* srcDimsTensor,
                                                             bool normalizeWeights, const Rpp32f* lookup,
                                                             Rpp32s lookupSize, Rpp32f scale, Rpp32f center,
                                                             Rpp32s lobes, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        return resample_common(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, inRateTensor, outRateTensor, srcDimsTensor,
                               lookup, lookupSize, scale, center, lobes, true, normalizeWeights);
    });
}

namespace {

// Host-tensor call: default chunk count, the first/last two chunks' share of a middle chunk's samples,
// the copy kernels' CTAs per chunk and the SMs the persistent kernel leaves to them.
constexpr int kHostChunks = 16;
constexpr double kEdgeWeight[2] = {0.25, 0.5};
constexpr int kMoverCtas = 96;
constexpr int kReservedSms = 40;

// Validates the fused-front-end parameters and fills the shared fields of FrontendArgs.
RppStatus frontend_params(Handle& h, const RppbFrontendParams* params, float* winStage, FrontendArgs& a)
{
    require(params != nullptr, "null parameters");
    const RppbFrontendParams& p = *params;
    if (!p.multiplier) return RPP_ERROR_ZERO_DIVISION;
    if (p.maxFreq < 0 || p.maxFreq > p.sampleRate / 2) return RPP_ERROR_INVALID_ARGUMENTS;
    if (p.minFreq < 0 || p.minFreq > p.sampleRate / 2) return RPP_ERROR_INVALID_ARGUMENTS;
    require(p.windowLength > 0 && p.windowStep > 0, "windowLength and windowStep must be positive");
    const int nfft = p.nfft == 0 ? p.windowLength : p.nfft;
    require(nfft >= p.windowLength, "nfft must be at least windowLength");
    require(p.numFilter > 0, "numFilter must be positive");
    a.border = int(p.borderType);
    a.center = p.centerWindows;
    a.reflect = p.reflectPadding;
    if (p.windowFunction)
    {
        h.upload(winStage, p.windowFunction, p.windowLength * sizeof(float));
        a.window = winStage;
    }
    else
    {
        a.window = h.table("hann" + std::to_string(p.windowLength), size_t(p.windowLength), build_hann, nullptr);
    }
    a.nfft = nfft;
    a.W = p.windowLength;
    a.hop = p.windowStep;
    a.power = p.power;
    a.mel.minFreq = p.minFreq;
    a.mel.maxFreq = (p.maxFreq == 0) ? p.sampleRate / 2 : p.maxFreq;
    a.mel.sampleRate = p.sampleRate;
    a.mel.htk = p.melFormula == HTK ? 1 : 0;
    a.mel.numFilter = p.numFilter;
    a.mel.normalize = p.normalize;
    // to_decibels.cpp:40-45
    float minRatio = float(std::pow(10, p.cutOffDB / p.multiplier));
    if (minRatio == 0.0f) minRatio = std::nextafter(0.0f, 1.0f);
    const Rpp32f log10Factor = 0.3010299956639812;
    a.minRatio = minRatio;
    a.multiplier = p.multiplier * log10Factor;
    a.refMag = p.referenceMagnitude;
    a.lookahead = p.lookahead > 0 ? p.lookahead : 32;
    a.reserveSms = 0;
    a.tileFrames = p.tileFrames;
    a.dbFrames = p.dbFrames;
    a.ctasPerSm = p.ctasPerSm;
    a.engine = int(p.spectrumEngine);
    a.clips = nullptr;
    a.outRate = 0.f;
    a.coeffAll = 0.f;
    return RPP_SUCCESS;
}

}  // namespace

extern "C" SHARED_PUBLIC RppStatus rppb_frontend_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                     RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor,
                                                     Rpp32f* coeffTensor, const RppbFrontendParams* params,
                                                     rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr && params, "null descriptor or parameters");
        if (srcDescPtr->numDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (dstDescPtr->numDims != 3) return RPP_ERROR_INVALID_DST_DIMS;
        if (dstDescPtr->layout != NFT) return RPP_ERROR_INVALID_DST_LAYOUT;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        if (dstDescPtr->h < Rpp32u(params->numFilter) || dstDescPtr->strides.hStride < dstDescPtr->w)
            return RPP_ERROR_INVALID_DST_DIMS;
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        const int lookahead = params->lookahead > 0 ? params->lookahead : 32;
        const size_t scratchBytes = frontend_scratch_bytes(n, lookahead, params->numFilter);
        const int W = params->windowLength > 0 ? params->windowLength : 0;
        Carver m(nullptr);
        m.take<int>(n);
        m.take<float>(n);
        m.take<float>(params->windowFunction ? W : 0);
        m.take<char>(scratchBytes);
        Carver cv(h.workspace(m.used()));
        int* lenStage = cv.take<int>(n);
        float* coeffStage = cv.take<float>(n);
        float* winStage = cv.take<float>(params->windowFunction ? W : 0);
        void* scratch = cv.take<char>(scratchBytes);
        FrontendArgs a;
        RppStatus st = frontend_params(h, params, winStage, a);
        if (st != RPP_SUCCESS) return st;
        a.src = static_cast<const float*>(srcPtr);
        a.srcStride = srcDescPtr->strides.nStride;
        a.srcElems = size_t(n) * srcDescPtr->strides.nStride;
        a.dst = static_cast<float*>(dstPtr);
        a.dstNStride = dstDescPtr->strides.nStride;
        a.dstHStride = dstDescPtr->strides.hStride;
        a.n = n;
        a.len = static_cast<const int*>(h.device_view(srcLengthTensor, n * sizeof(int), lenStage));
        a.coeff = static_cast<const float*>(h.device_view(coeffTensor, n * sizeof(float), coeffStage));
        a.maxFrames = int(dstDescPtr->w);
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_frontend(h, scratch, a);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_frontend_host_gpu(const Rpp32f* srcHost, RpptDescPtr srcDescPtr,
                                                          Rpp32f* dstHost, RpptDescPtr dstDescPtr,
                                                          const Rpp32s* srcLengthHost, const Rpp32f* coeffHost,
                                                          const RppbFrontendParams* params, Rpp32s numChunks,
                                                          rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr && params, "null descriptor or parameters");
        if (srcDescPtr->numDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (dstDescPtr->numDims != 3) return RPP_ERROR_INVALID_DST_DIMS;
        if (dstDescPtr->layout != NFT) return RPP_ERROR_INVALID_DST_LAYOUT;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcHost && dstHost && srcLengthHost && coeffHost, "null tensor");
        if (dstDescPtr->h < Rpp32u(params->numFilter) || dstDescPtr->strides.hStride < dstDescPtr->w)
            return RPP_ERROR_INVALID_DST_DIMS;
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        FrontendArgs a;
        const int W = params->windowLength > 0 ? params->windowLength : 0;
        const size_t nStride = srcDescPtr->strides.nStride;
        const int maxFrames = int(dstDescPtr->w);
        const int nf = params->numFilter;

        // per-clip lengths and frame counts on the host (the call's tensors are host memory)
        std::vector<int> L(n), F(n);
        size_t total = 0;
        for (int b = 0; b < n; ++b)
        {
            L[b] = std::max(0, std::min(srcLengthHost[b], int(nStride)));
            const int len = params->centerWindows ? L[b] : L[b] - W;
            F[b] = std::min(std::max(params->windowStep > 0 ? len / params->windowStep + 1 : 0, 0), maxFrames);
            total += size_t(L[b]);
        }
        // contiguous chunks of clips; the middle ones carry about equal sample counts, the first and the
        // last two less (kEdgeWeight of a middle chunk), so that the copy-in before the first kernel and
        // the copy-out after the last one, each running with the other direction idle, are short
        const int chunks = std::max(1, std::min(n, numChunks > 0 ? numChunks : kHostChunks));
        std::vector<double> weight(chunks, 1.0);
        if (chunks >= 6)
            for (int e = 0; e < 2; ++e) weight[e] = weight[chunks - 1 - e] = kEdgeWeight[e];
        std::vector<double> cut(chunks);   // samples up to the end of chunk c
        double wsum = 0.0, run = 0.0;
        for (double w : weight) wsum += w;
        for (int c = 0; c < chunks; ++c) cut[c] = (run += weight[c]) / wsum * double(total);
        std::vector<int> bound{0};
        size_t acc = 0;
        for (int b = 0; b < n; ++b)
        {
            acc += size_t(L[b]);
            const int c = int(bound.size()) - 1;
            if (c + 1 < chunks && b + 1 < n && double(acc) >= cut[c]) bound.push_back(b + 1);
        }
        bound.push_back(n);
        const int nc = int(bound.size()) - 1;
        std::vector<uint32_t> strideC(nc);
        std::vector<int> framesC(nc);
        size_t inElems = 0, outElems = 0;
        int maxClips = 0;
        for (int c = 0; c < nc; ++c)
        {
            int ml = 2, mf = 1;
            for (int b = bound[c]; b < bound[c + 1]; ++b)
            {
                ml = std::max(ml, L[b]);
                mf = std::max(mf, F[b]);
            }
            strideC[c] = uint32_t((ml + 3) & ~3);
            framesC[c] = mf;
            const int clips = bound[c + 1] - bound[c];
            maxClips = std::max(maxClips, clips);
            inElems = std::max(inElems, size_t(clips) * strideC[c]);
            outElems = std::max(outElems, size_t(clips) * nf * size_t(mf));
        }
        const int lookahead = params->lookahead > 0 ? params->lookahead : 32;
        const size_t scratchBytes = frontend_scratch_bytes(maxClips, lookahead, params->numFilter);
        Carver m(nullptr);
        m.take<int>(2 * n);
        m.take<float>(n);
        m.take<float>(params->windowFunction ? W : 0);
        m.take<char>(scratchBytes);
        for (int i = 0; i < 2; ++i) m.take<float>(inElems);
        for (int i = 0; i < 2; ++i) m.take<float>(outElems);
        Carver cv(h.workspace(m.used()));
        int* lenDev = cv.take<int>(2 * n);   // lengths, then frame counts
        int* framesDev = lenDev + n;
        float* coeffDev = cv.take<float>(n);
        float* winStage = cv.take<float>(params->windowFunction ? W : 0);
        void* scratch = cv.take<char>(scratchBytes);
        float* in[2] = {cv.take<float>(inElems), cv.take<float>(inElems)};
        float* out[2] = {cv.take<float>(outElems), cv.take<float>(outElems)};
        RppStatus st = frontend_params(h, params, winStage, a);
        if (st != RPP_SUCCESS) return st;
        std::vector<int> LF(2 * n);
        std::copy(L.begin(), L.end(), LF.begin());
        std::copy(F.begin(), F.end(), LF.begin() + n);
        h.upload(lenDev, LF.data(), 2 * n * sizeof(int));
        h.upload(coeffDev, coeffHost, n * sizeof(float));

        // pinned (mapped) host tensors are moved by kernels; pageable ones by one DMA copy per clip
        void* srcMapped = nullptr;
        void* dstMapped = nullptr;
        const bool gatherK = h.device_writable(srcHost, &srcMapped);
        const bool scatterK = h.device_writable(dstHost, &dstMapped);
        if (gatherK || scatterK) a.reserveSms = kReservedSms;   // room for the movers next to the persistent kernel
        if (gatherK) h.check_src(srcMapped, desc_bytes(srcDescPtr, n));
        if (scatterK) h.check_dst(dstMapped, desc_bytes(dstDescPtr, n));

        cudaStream_t main = h.stream(), up = h.aux_stream(0), down = h.aux_stream(1);
        cudaEvent_t start = h.event(0);
        auto evUp = [&](int c) { return h.event(1 + 3 * c); };
        auto evComp = [&](int c) { return h.event(2 + 3 * c); };
        auto evDown = [&](int c) { return h.event(3 + 3 * c); };
        check_cuda(cudaEventRecord(start, main), "cudaEventRecord");
        check_cuda(cudaStreamWaitEvent(up, start, 0), "cudaStreamWaitEvent");
        check_cuda(cudaStreamWaitEvent(down, start, 0), "cudaStreamWaitEvent");
        for (int c = 0; c < nc; ++c)
        {
            const int c0 = bound[c], clips = bound[c + 1] - c0, buf = c & 1;
            // inputs: the valid samples of each clip (at least 2, which the REFLECT border reads)
            if (c >= 2) check_cuda(cudaStreamWaitEvent(up, evComp(c - 2), 0), "cudaStreamWaitEvent");
            if (gatherK)
                launch_host_gather(up, static_cast<const float*>(srcMapped) + size_t(c0) * nStride, nStride,
                                   lenDev + c0, clips, in[buf], strideC[c], kMoverCtas);
            else
                for (int b = c0; b < c0 + clips; ++b)
                {
                    const size_t cnt = std::min(nStride, size_t(std::max(L[b], 2)));
                    check_cuda(cudaMemcpyAsync(in[buf] + size_t(b - c0) * strideC[c], srcHost + size_t(b) * nStride,
                                               cnt * sizeof(float), cudaMemcpyHostToDevice, up),
                               "cudaMemcpyAsync(H2D clip)");
                }
            check_cuda(cudaEventRecord(evUp(c), up), "cudaEventRecord");
            // compute
            check_cuda(cudaStreamWaitEvent(main, evUp(c), 0), "cudaStreamWaitEvent");
            if (c >= 2) check_cuda(cudaStreamWaitEvent(main, evDown(c - 2), 0), "cudaStreamWaitEvent");
            a.src = in[buf];
            a.srcStride = strideC[c];
            a.srcElems = size_t(clips) * strideC[c];
            a.dst = out[buf];
            a.dstNStride = uint32_t(size_t(nf) * framesC[c]);
            a.dstHStride = uint32_t(framesC[c]);
            a.n = clips;
            a.len = lenDev + c0;
            a.coeff = coeffDev + c0;
            a.maxFrames = framesC[c];
            launch_frontend(h, scratch, a);
            check_cuda(cudaEventRecord(evComp(c), main), "cudaEventRecord");
            // outputs: numFilter rows of F frames per clip
            check_cuda(cudaStreamWaitEvent(down, evComp(c), 0), "cudaStreamWaitEvent");
            if (scatterK)
                launch_host_scatter(down, out[buf], a.dstNStride, a.dstHStride, framesDev + c0, clips, nf,
                                    static_cast<float*>(dstMapped) + size_t(c0) * dstDescPtr->strides.nStride,
                                    dstDescPtr->strides.nStride, dstDescPtr->strides.hStride, kMoverCtas);
            else
                for (int b = c0; b < c0 + clips; ++b)
                {
                    if (F[b] <= 0) continue;
                    check_cuda(cudaMemcpy2DAsync(dstHost + size_t(b) * dstDescPtr->strides.nStride,
                                                 size_t(dstDescPtr->strides.hStride) * sizeof(float),
                                                 out[buf] + size_t(b - c0) * a.dstNStride,
                                                 size_t(framesC[c]) * sizeof(float), size_t(F[b]) * sizeof(float),
                                                 size_t(nf), cudaMemcpyDeviceToHost, down),
                               "cudaMemcpy2DAsync(D2H clip)");
                }
            check_cuda(cudaEventRecord(evDown(c), down), "cudaEventRecord");
        }
        check_cuda(cudaStreamWaitEvent(main, evDown(nc - 1), 0), "cudaStreamWaitEvent");
        check_cuda(cudaStreamWaitEvent(main, evUp(nc - 1), 0), "cudaStreamWaitEvent");
        return RPP_SUCCESS;
    });
}

namespace rppb {

RppStatus frontend_clips(Handle& h, const RppbClip* clips, int numClips, float outRate, const float* lookup,
                         int lookupSize, float scale, float center, int lobes, float preemphCoeff,
                         const RppbFrontendParams* params, int reserveSms)
{
    {
        require(clips != nullptr && params != nullptr, "null clip table or parameters");
        require(lookup != nullptr && lookupSize >= 2 && lobes >= 0, "invalid resampling window");
        require(size_t(lookupSize) * sizeof(float) <= 200 * 1024, "lookup table above 200 KB");
        require(outRate > 0.f, "outRate must be positive");
        const int n = numClips;
        if (n <= 0) return RPP_SUCCESS;
        const int lookahead = params->lookahead > 0 ? params->lookahead : 32;
        const size_t scratchBytes = frontend_scratch_bytes(n, lookahead, params->numFilter);
        const int W = params->windowLength > 0 ? params->windowLength : 0;
        Carver m(nullptr);
        m.take<RppbClip>(n);
        m.take<float>(lookupSize);
        m.take<float>(params->windowFunction ? W : 0);
        m.take<char>(prefix_bytes(n));
        m.take<char>(scratchBytes);
        Carver cv(h.workspace(m.used()));
        RppbClip* clipStage = cv.take<RppbClip>(n);
        float* lutStage = cv.take<float>(lookupSize);
        float* winStage = cv.take<float>(params->windowFunction ? W : 0);
        void* resampleScratch = cv.take<char>(prefix_bytes(n));
        void* scratch = cv.take<char>(scratchBytes);
        FrontendArgs a;
        RppStatus st = frontend_params(h, params, winStage, a);
        if (st != RPP_SUCCESS) return st;
        const RppbClip* dclips = static_cast<const RppbClip*>(h.device_view(clips, n * sizeof(RppbClip), clipStage));
        ResampleWindowDev win;
        win.lut = static_cast<const float*>(h.device_view(lookup, lookupSize * sizeof(float), lutStage));
        win.lutSize = lookupSize;
        win.scale = scale;
        win.center = center;
        win.lobes = lobes;
#ifdef RPPB_CHECKED
        // the clips' buffers, as the table describes them (read back here; a captured call is not checked)
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        check_cuda(cudaStreamIsCapturing(h.stream(), &cap), "cudaStreamIsCapturing");
        if (cap == cudaStreamCaptureStatusNone)
        {
            std::vector<RppbClip> hc(n);
            check_cuda(cudaMemcpy(hc.data(), clips, n * sizeof(RppbClip), cudaMemcpyDefault), "read clip table");
            for (const RppbClip& c : hc)
            {
                if (c.length <= 0) continue;
                h.check_add(c.src, size_t(c.length) * sizeof(float), false);
                h.check_add(c.work, size_t(std::max(resampled_length(c.length, c.inRate, outRate), 0)) * sizeof(float),
                            true);
                h.check_dst(c.dst, size_t(params->numFilter) * size_t(std::max(c.dstStride, 0)) * sizeof(float));
            }
        }
        else
            h.check_suspend();
#endif
        launch_resample_clips(h, resampleScratch, dclips, n, outRate, win);
        a.src = nullptr;
        a.srcStride = 0;
        a.srcElems = 0;
        a.dst = nullptr;
        a.dstNStride = 0;
        a.dstHStride = 0;
        a.n = n;
        a.len = nullptr;
        a.coeff = nullptr;
        a.maxFrames = 0;
        a.clips = dclips;
        a.outRate = outRate;
        a.coeffAll = preemphCoeff;
        a.reserveSms = reserveSms;
        launch_frontend(h, scratch, a);
        return RPP_SUCCESS;
    }
}

}  // namespace rppb

extern "C" SHARED_PUBLIC RppStatus rppb_frontend_clips_gpu(const RppbClip* clips, Rpp32s numClips, Rpp32f outRate,
                                                           const Rpp32f* lookup, Rpp32s lookupSize, Rpp32f scale,
                                                           Rpp32f center, Rpp32s lobes, Rpp32f preemphCoeff,
                                                           const RppbFrontendParams* params, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        return frontend_clips(h, clips, numClips, outRate, lookup, lookupSize, scale, center, lobes, preemphCoeff,
                              params, 0);
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_set_wait_fault_injection(rppHandle_t rppHandle, bool enable)
{
    return guarded(rppHandle, [&](Handle& h) {
        h.set_wait_injection(enable);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_set_tc_materialized_frames(rppHandle_t rppHandle, bool materialize)
{
    return guarded(rppHandle, [&](Handle& h) {
        h.set_tc_materialize(materialize);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_get_device_error(rppHandle_t rppHandle, Rpp32s* errorCode)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(errorCode != nullptr, "null errorCode");
        int* flags = h.device_flags();
        int v = 0;
        check_cuda(cudaMemcpyAsync(&v, flags, sizeof(int), cudaMemcpyDeviceToHost, h.stream()), "read device error");
        check_cuda(cudaMemsetAsync(flags, 0, sizeof(int), h.stream()), "clear device error");
        check_cuda(cudaStreamSynchronize(h.stream()), "sync");
        *errorCode = v;
        return RPP_SUCCESS;
    });
}

namespace {

struct TcBasisKey
{
    int fmt, nfft, W, kPad;
};

void build_tc_basis(float* out, size_t, const void* ctx)
{
    const TcBasisKey k = *static_cast<const TcBasisKey*>(ctx);
    std::vector<float> win(k.W);
    build_hann(win.data(), size_t(k.W), nullptr);
    tc_build_basis(out, k.fmt, k.nfft, k.W, k.kPad, win.data());
}

}  // namespace

extern "C" SHARED_PUBLIC RppStatus rppb_spectrogram_tc_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                           RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor,
                                                           Rpp32f* coeffTensor, RpptAudioBorderType borderType,
                                                           bool centerWindows, bool reflectPadding, Rpp32s nfft,
                                                           Rpp32s power, Rpp32s windowLength, Rpp32s windowStep,
                                                           RppbTensorCorePrecision precision, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        if ((dstDescPtr->layout != NFT) && (dstDescPtr->layout != NTF)) return RPP_ERROR_INVALID_DST_LAYOUT;
        if (srcDescPtr->numDims != 2) return RPP_ERROR_INVALID_SRC_DIMS;
        if (dstDescPtr->numDims != 3) return RPP_ERROR_INVALID_DST_DIMS;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr, "null tensor");
        require(windowLength > 0 && windowStep > 0 && windowLength <= nfft, "invalid window");
        const int fmt = int(precision);
        if (fmt < kTcBf16 || fmt > kTcFp8) return RPP_ERROR_NOT_IMPLEMENTED;
        // in-place BF16 / TF32 frame rows start every hop elements and must stay 16-byte aligned
        const int granule = fmt == kTcTf32 ? 4 : fmt == kTcFp8 ? 1 : 8;
        if (nfft % 256 != 0 || windowStep % granule != 0) return RPP_ERROR_NOT_IMPLEMENTED;
        const bool nft = dstDescPtr->layout == NFT;
        const Rpp32u binsCap = nft ? dstDescPtr->h : dstDescPtr->w;
        if (binsCap < Rpp32u(nfft / 2 + 1)) return RPP_ERROR_INVALID_DST_DIMS;
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        const int maxFrames = int(nft ? dstDescPtr->w : dstDescPtr->h);
        const TcGeometry geo =
            tc_geometry(fmt, windowLength, windowStep, maxFrames, nfft,
                        !h.tc_materialize() && tc_overlap_supported(h.device_flags()));
        const size_t scratchBytes = tc_spectrogram_scratch_bytes(n, fmt, geo, maxFrames);
        Carver m(nullptr);
        m.take<int>(n);
        m.take<float>(n);
        m.take<char>(scratchBytes);
        Carver cv(h.workspace(m.used()));
        int* lenStage = cv.take<int>(n);
        float* coeffStage = cv.take<float>(n);
        void* scratch = cv.take<char>(scratchBytes);
        TcBasisKey key{fmt, nfft, windowLength, geo.kPad};
        const float* basis = h.table("tcbasis" + std::to_string(fmt) + "_" + std::to_string(nfft) + "_" +
                                         std::to_string(windowLength),
                                     geo.basisFloats, build_tc_basis, &key);
        TcSpectrogramArgs a;
        a.src = static_cast<const float*>(srcPtr);
        a.srcStride = srcDescPtr->strides.nStride;
        a.srcElems = size_t(n) * srcDescPtr->strides.nStride;
        a.len = static_cast<const int*>(h.device_view(srcLengthTensor, n * sizeof(int), lenStage));
        a.coeff = coeffTensor ? static_cast<const float*>(h.device_view(coeffTensor, n * sizeof(float), coeffStage))
                              : nullptr;
        a.border = int(borderType);
        a.center = centerWindows;
        a.reflect = reflectPadding;
        a.windowLength = windowLength;
        a.windowStep = windowStep;
        a.nfft = nfft;
        a.fmt = fmt;
        a.geo = geo;
        a.maxFrames = maxFrames;
        a.basis = basis;
        a.dst = static_cast<float*>(dstPtr);
        a.dstNStride = dstDescPtr->strides.nStride;
        a.dstHStride = dstDescPtr->strides.hStride;
        a.nft = nft;
        a.power = power;
        a.n = n;
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_tc_spectrogram(h, scratch, a);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppt_slice_gpu(RppPtr_t srcPtr, RpptGenericDescPtr srcGenericDescPtr,
                                                  RppPtr_t dstPtr, RpptGenericDescPtr dstGenericDescPtr,
                                                  Rpp32s* anchorTensor, Rpp32s* shapeTensor, RppPtr_t fillValue,
                                                  bool enablePadding, Rpp32u* roiTensor, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcGenericDescPtr && dstGenericDescPtr, "null descriptor");
        const RpptGenericDesc& sd = *srcGenericDescPtr;
        const RpptGenericDesc& dd = *dstGenericDescPtr;
        // rppt_tensor_geometric_augmentations.cpp:2520-2522
        if (sd.dataType != F32 && sd.dataType != U8) return RPP_ERROR_INVALID_SRC_DATATYPE;
        if (dd.dataType != F32 && dd.dataType != U8) return RPP_ERROR_INVALID_DST_DATATYPE;
        if (sd.layout != dd.layout) return RPP_ERROR_LAYOUT_MISMATCH;
        if (sd.dataType != dd.dataType) return RPP_ERROR_NOT_IMPLEMENTED;
        // 1-D signals and 2-D spectra in any layout; 3-D images (NCHW, NHWC) and 4-D volumes (NCDHW,
        // NDHWC), the layouts the reference slices (cpu/kernel/slice.cpp:61-199)
        if (sd.numDims < 2 || sd.numDims > 5 || dd.numDims != sd.numDims) return RPP_ERROR_NOT_IMPLEMENTED;
        int layoutKind = 0;
        if (sd.numDims == 4) layoutKind = sd.layout == NCHW ? 1 : sd.layout == NHWC ? 2 : 0;
        if (sd.numDims == 5) layoutKind = sd.layout == NCDHW ? 1 : sd.layout == NDHWC ? 2 : 0;
        if (sd.numDims >= 4 && layoutKind == 0) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr && anchorTensor && shapeTensor && roiTensor, "null tensor");
        require(!enablePadding || fillValue, "null fill value");
        const int n = int(dd.dims[0]);
        if (n <= 0) return RPP_SUCCESS;
        require(sd.dims[0] >= dd.dims[0], "source batch smaller than destination batch");
        const int nd = int(sd.numDims) - 1;
        const int eb = sd.dataType == U8 ? 1 : 4;
        Carver m(nullptr);
        m.take<int>(size_t(n) * nd);
        m.take<int>(size_t(n) * nd);
        m.take<uint32_t>(size_t(n) * nd * 2);
        m.take<float>(1);
        Carver cv(h.workspace(m.used()));
        int* aStage = cv.take<int>(size_t(n) * nd);
        int* sStage = cv.take<int>(size_t(n) * nd);
        uint32_t* rStage = cv.take<uint32_t>(size_t(n) * nd * 2);
        float* fStage = cv.take<float>(1);
        SliceArgs a;
        a.n = n;
        a.numDims = nd;
        a.elemBytes = eb;
        a.srcStride0 = sd.strides[0];
        a.srcStride1 = nd == 2 ? sd.strides[1] : 0;
        a.dstStride0 = dd.strides[0];
        a.dstStride1 = nd == 2 ? dd.strides[1] : 0;
        a.srcDim0 = sd.dims[1];
        a.srcDim1 = nd == 2 ? sd.dims[2] : 1;
        if (nd == 2 && (a.dstStride1 == 0 || a.srcStride1 < a.srcDim1)) return RPP_ERROR_INVALID_ARGUMENTS;
        a.layoutKind = layoutKind;
        for (int k = 0; k <= nd; ++k)
        {
            a.srcStrides[k] = sd.strides[k];
            a.dstStrides[k] = dd.strides[k];
            if (k < nd)
            {
                a.srcDims[k] = sd.dims[k + 1];
                a.dstDims[k] = dd.dims[k + 1];
            }
        }
        if (nd >= 3)
        {
            // rows are contiguous, both tensors hold the same channels, and the destination's strides
            // nest (each level at least the next level's extent), so that every destination element
            // belongs to one box position
            if (sd.strides[nd] != 1 || dd.strides[nd] != 1) return RPP_ERROR_INVALID_ARGUMENTS;
            const int ch = layoutKind == 1 ? 0 : nd - 1;
            if (sd.dims[ch + 1] != dd.dims[ch + 1]) return RPP_ERROR_INVALID_ARGUMENTS;
            // channel-last rows are width x channels contiguous elements
            if (layoutKind == 2 && (sd.strides[nd - 1] != sd.dims[nd] || dd.strides[nd - 1] != dd.dims[nd]))
                return RPP_ERROR_INVALID_ARGUMENTS;
            // destination levels, outermost first: (stride, extent of one step of the next level)
            std::vector<std::pair<size_t, size_t>> lv;
            if (layoutKind == 1)
            {
                lv.push_back({sd.strides[1], size_t(dd.dims[2]) * dd.strides[2]});   // channels step by the source's stride
                for (int k = 2; k < nd; ++k) lv.push_back({dd.strides[k], size_t(dd.dims[k + 1]) * dd.strides[k + 1]});
            }
            else
                for (int k = 1; k < nd - 1; ++k)
                    lv.push_back({dd.strides[k], size_t(dd.dims[k + 1]) * dd.strides[k + 1]});
            for (const auto& l : lv)
                if (l.first < l.second) return RPP_ERROR_INVALID_ARGUMENTS;
            if (size_t(sd.dims[ch + 1]) * (layoutKind == 1 ? sd.strides[1] : 1) > size_t(UINT32_MAX))
                return RPP_ERROR_INVALID_ARGUMENTS;
        }
        a.anchor = static_cast<const int*>(h.device_view(anchorTensor, size_t(n) * nd * sizeof(int), aStage));
        a.shape = static_cast<const int*>(h.device_view(shapeTensor, size_t(n) * nd * sizeof(int), sStage));
        a.roi = static_cast<const uint32_t*>(h.device_view(roiTensor, size_t(n) * nd * 2 * sizeof(uint32_t), rStage));
        a.enablePadding = enablePadding;
        const void* fill = enablePadding ? h.device_view(fillValue, size_t(eb), fStage) : nullptr;
        const size_t off = sd.offsetInBytes, doff = dd.offsetInBytes;
        check_tensors(h, srcPtr, sd, dstPtr, dd, n);
        launch_slice(h, a, static_cast<const char*>(srcPtr) + off, static_cast<char*>(dstPtr) + doff, fill);
        return RPP_SUCCESS;
    });
}

namespace {

// The caller's roi tensor on the host (parameter counts and plans are built there).  Memory the
// device can write (device, managed, pinned) may still be written by earlier work on the handle
// stream, so the stream is synchronized before the host reads it; pageable memory is read as it is.
std::vector<uint32_t> roi_to_host(Handle& h, const Rpp32u* roiTensor, size_t count)
{
    std::vector<uint32_t> roi(count);
    cudaPointerAttributes attr{};
    const bool known = cudaPointerGetAttributes(&attr, roiTensor) == cudaSuccess;
    if (!known) cudaGetLastError();
    const cudaMemoryType mt = known ? attr.type : cudaMemoryTypeUnregistered;
    if (mt == cudaMemoryTypeDevice)
    {
        check_cuda(cudaMemcpyAsync(roi.data(), roiTensor, count * 4, cudaMemcpyDeviceToHost, h.stream()),
                   "cudaMemcpyAsync(roi)");
        check_cuda(cudaStreamSynchronize(h.stream()), "cudaStreamSynchronize(roi)");
    }
    else
    {
        if (mt == cudaMemoryTypeHost || mt == cudaMemoryTypeManaged)
            check_cuda(cudaStreamSynchronize(h.stream()), "cudaStreamSynchronize(roi)");
        std::memcpy(roi.data(), roiTensor, count * 4);
    }
    return roi;
}

int norm_type(RpptDataType t)
{
    return t == F32 ? kNormF32 : t == F16 ? kNormF16 : t == U8 ? kNormU8 : t == I8 ? kNormI8 : -1;
}

// Largest element offset a set of (count, stride) levels reaches; false if some count is 0.
bool reach(const uint32_t* count, const uint32_t* stride, int levels, size_t& out)
{
    out = 0;
    for (int l = 0; l < levels; ++l)
    {
        if (count[l] == 0) return false;
        out += size_t(count[l] - 1) * stride[l];
    }
    return true;
}

// Plan of one sample for the F32 3-D branch (normalize.cpp:592-730).
bool plan_3d(const RpptGenericDesc& sd, const RpptGenericDesc& dd, unsigned axisMask, const uint32_t* begin,
             const uint32_t* length, NormNdSample& s, uint32_t& params)
{
    const uint32_t L0 = length[0], L1 = length[1], L2 = length[2];
    if (uint64_t(L0) * L1 * L2 > UINT32_MAX) return false;   // the reduction counts stay 32-bit
    const uint32_t S1 = sd.strides[1], S2 = sd.strides[2], S3 = sd.strides[3];
    uint32_t rd[3], rs[3];
    bool ps[3] = {false, false, false};
    bool consecutive = true;
    switch (axisMask)
    {
    case 1: rd[0] = L1; rd[1] = L2; rd[2] = L0; rs[0] = S1; rs[1] = S3; rs[2] = S2; ps[1] = ps[2] = true; break;
    case 2: rd[0] = L0; rd[1] = L2; rd[2] = L1; rs[0] = S2; rs[1] = S3; rs[2] = S1; ps[0] = ps[2] = true; break;
    case 3: rd[0] = 1; rd[1] = L2; rd[2] = L0 * L1; rs[0] = S2; rs[1] = S3; rs[2] = S3; ps[2] = true; break;
    case 4: rd[0] = L0; rd[1] = L1; rd[2] = L2; rs[0] = S3; rs[1] = S2; rs[2] = S1; ps[0] = ps[1] = true; break;
    case 5: rd[0] = L1; rd[1] = L0; rd[2] = L2; rs[0] = S3; rs[1] = S1; rs[2] = S2; ps[1] = true; consecutive = false;
        break;
    case 6: rd[0] = 1; rd[1] = L0; rd[2] = L1 * L2; rs[0] = S3; rs[1] = S1; rs[2] = S3; ps[0] = true; break;
    default: rd[0] = 1; rd[1] = 1; rd[2] = L0 * L1 * L2; rs[0] = rs[1] = rs[2] = S3; break;
    }
    s.srcBase = size_t(begin[0]) * S1 + size_t(begin[1]) * S2;
    s.accumulate = 0;
    s.lineStride = rs[0];
    s.lineCount = rd[2];
    if (consecutive)
    {
        s.pLevels = 2;
        s.pCount[0] = rd[0];
        s.pStride[0] = rs[2];
        s.pCount[1] = rd[1];
        s.pStride[1] = rs[1];
        s.oLevels = 0;
        s.normFactor = float(1.0 / double(rd[2]));
        params = rd[0] * rd[1];
    }
    else
    {
        s.pLevels = 1;
        s.pCount[0] = rd[0];
        s.pStride[0] = rs[2];
        s.oLevels = 1;
        s.oCount[0] = rd[1];
        s.oStride[0] = rs[1];
        s.normFactor = float(1.0 / double(rd[1] * rd[2]));
        params = rd[0];
    }
    // output (normalize.cpp:717-723): NHWC -> NHWC (the 16-channel mask-3 case over whole rows of 16
    // channels), NHWC -> NCHW for mask 3, otherwise nothing
    s.levels = 0;
    s.zeroFrom = 0;
    if (axisMask == 3 && sd.layout == NHWC && dd.layout == NHWC && sd.dims[3] == 16)
    {
        if (L2 != 16) return false;   // the 16 channel parameters must all exist
        s.lv[0] = {L0, S1, dd.strides[1], 0};
        s.lv[1] = {L1, 16, 16, 0};
        s.lv[2] = {16, 1, 1, 1};
        s.levels = 3;
    }
    else if (sd.layout == NHWC && dd.layout == NHWC)
    {
        const uint32_t m2 = ps[2] ? 1 : 0, m1 = ps[1] ? (ps[2] ? L2 : 1) : 0;
        const uint32_t m0 = ps[0] ? (ps[1] ? L1 : 1) * (ps[2] ? L2 : 1) : 0;
        s.lv[0] = {L0, S1, dd.strides[1], m0};
        s.lv[1] = {L1, S2, dd.strides[2], m1};
        s.lv[2] = {L2, 1, 1, m2};
        s.levels = 3;
    }
    else if (axisMask == 3 && sd.layout == NHWC && dd.layout == NCHW)
    {
        s.lv[0] = {L0, S1, dd.strides[2], 0};
        s.lv[1] = {L1, S2, dd.strides[3], 0};
        s.lv[2] = {L2, 1, dd.strides[1], 1};
        s.levels = 3;
    }
    return true;
}

// Plan of one sample for the N-D branch (normalize.cpp:731-868): collapse_axis, dense addressing.
bool plan_nd(const RpptGenericDesc& sd, int T, unsigned axisMask, const uint32_t* begin, const uint32_t* length,
             NormNdSample& s, uint32_t& params)
{
    uint32_t axis[4], newAxis[4] = {0, 0, 0, 0}, newDims[4] = {0, 0, 0, 0}, size = 1, total = 1;
    uint64_t volume = 1;
    for (int i = 0; i < T; ++i) volume *= length[i];
    if (volume > UINT32_MAX) return false;   // dense strides and counts stay 32-bit
    s.srcBase = 0;
    for (int i = 0; i < T; ++i)
    {
        axis[i] = (axisMask >> i) & 1u;
        size *= axis[i] ? 1 : length[i];
        total *= axis[i] ? length[i] : 1;
        s.srcBase += size_t(begin[i]) * sd.strides[i + 1];
    }
    // collapse_axis as the reference runs it: a normalized axis merges into the previous one only
    // while no axis has been merged before it
    int skipped = 0, prev = -2, k = 0;
    for (int i = 0; i < T; ++i)
    {
        if (axis[i])
        {
            if (i - skipped != prev + 1)
            {
                newAxis[k] = 1;
                newDims[k] = length[i];
                prev = i;
                ++k;
            }
            else if (prev >= 0)
            {
                newDims[prev] *= length[i];
                ++skipped;
            }
        }
        else
            newDims[k++] = length[i];
    }
    const int nT = T - skipped;
    int lastNorm = 0;
    for (int i = 0; i < nT; ++i)
        if (newAxis[i]) lastNorm = i;
    uint32_t st[4];
    uint32_t v = 1;
    for (int i = nT - 1; i >= 0; --i)
    {
        st[i] = v;
        v *= newDims[i];
    }
    s.accumulate = 1;
    s.normFactor = float(1.0 / double(total));
    s.pLevels = s.oLevels = 0;
    for (int l = 0; l < nT; ++l)
    {
        if (!newAxis[l])
        {
            s.pCount[s.pLevels] = newDims[l];
            s.pStride[s.pLevels++] = st[l];
        }
        else if (l != lastNorm)
        {
            s.oCount[s.oLevels] = newDims[l];
            s.oStride[s.oLevels++] = st[l];
        }
    }
    s.lineStride = st[lastNorm];
    s.lineCount = newDims[lastNorm];
    params = size;
    s.levels = nT;
    s.elems = 1;
    for (int l = 0; l < nT; ++l)
    {
        uint32_t pm = 0;
        if (!newAxis[l])
        {
            pm = 1;
            for (int m = l + 1; m < nT; ++m)
                if (!newAxis[m]) pm *= newDims[m];
        }
        s.lv[l] = {newDims[l], st[l], st[l], pm};
        s.elems *= newDims[l];
    }
    return true;
}

// normalize for every type and rank but the 2-D F32 one.
RppStatus normalize_nd(Handle& h, const void* srcPtr, const RpptGenericDesc& sd, void* dstPtr,
                       const RpptGenericDesc& dd, Rpp32u axisMask, Rpp32f* meanTensor, Rpp32f* stdDevTensor,
                       int compute, Rpp32f scale, Rpp32f shift, const Rpp32u* roiTensor)
{
    const int ts = norm_type(RpptDataType(sd.dataType)), td = norm_type(RpptDataType(dd.dataType));
    if (ts < 0 || ts != td) return RPP_ERROR_NOT_IMPLEMENTED;   // U8, F16, F32, I8, source type = destination type
    if (sd.numDims < 2 || sd.numDims > 5 || dd.numDims != sd.numDims) return RPP_ERROR_NOT_IMPLEMENTED;
    const int T = int(sd.numDims) - 1;
    if (axisMask == 0 || axisMask >= (1u << T)) return RPP_ERROR_INVALID_ARGUMENTS;
    require(srcPtr && dstPtr && roiTensor && meanTensor && stdDevTensor, "null tensor");
    const int n = int(dd.dims[0]);
    if (n <= 0) return RPP_SUCCESS;
    require(sd.dims[0] >= dd.dims[0], "source batch smaller than destination batch");
    const std::vector<uint32_t> roi = roi_to_host(h, roiTensor, size_t(n) * T * 2);
    int maxSize = 1;
    for (int b = 0; b < n; ++b)
    {
        size_t size = 1;
        for (int i = 0; i < T; ++i) size *= ((axisMask >> i) & 1u) ? 1 : roi[size_t(b) * 2 * T + T + i];
        if (size > size_t(INT32_MAX)) return RPP_ERROR_INVALID_ARGUMENTS;
        maxSize = std::max(maxSize, int(size));
    }
    const bool is3d = ts == kNormF32 && T == 3;
    std::vector<NormNdSample> samples(n);
    std::vector<int4> tasks;
    size_t maxElems = 0, maxZero = 0;
    for (int b = 0; b < n; ++b)
    {
        const uint32_t* begin = &roi[size_t(b) * 2 * T];
        const uint32_t* length = begin + T;
        NormNdSample& s = samples[b];
        std::memset(&s, 0, sizeof s);
        uint32_t params = 0;
        if (!(is3d ? plan_3d(sd, dd, axisMask, begin, length, s, params)
                   : plan_nd(sd, T, axisMask, begin, length, s, params)))
            return RPP_ERROR_INVALID_ARGUMENTS;
        // every read inside the source sample, every write inside the destination sample
        uint32_t lc[4], lst[4], ld_[4];
        for (int l = 0; l < s.levels; ++l)
        {
            lc[l] = s.lv[l].count;
            lst[l] = s.lv[l].srcStride;
            ld_[l] = s.lv[l].dstStride;
        }
        size_t r1 = 0, r2 = 0, r3 = 0, w = 0;
        if (compute && params > 0 && s.lineCount > 0 && reach(s.pCount, s.pStride, s.pLevels, r1) &&
            reach(s.oCount, s.oStride, s.oLevels, r2))
        {
            r3 = size_t(s.lineCount - 1) * s.lineStride;
            if (s.srcBase + r1 + r2 + r3 >= sd.strides[0]) return RPP_ERROR_INVALID_ARGUMENTS;
        }
        if (s.levels > 0 && reach(lc, lst, s.levels, r1) && reach(lc, ld_, s.levels, w))
        {
            if (s.srcBase + r1 >= sd.strides[0] || w >= dd.strides[0]) return RPP_ERROR_INVALID_ARGUMENTS;
        }
        else
            s.elems = 0;
        if (!is3d) s.zeroFrom = std::min<size_t>(s.elems, dd.strides[0]);
        else s.elems = s.levels > 0 ? size_t(s.lv[0].count) * s.lv[1].count * s.lv[2].count : 0;
        if (s.levels == 0) s.elems = 0;
        maxElems = std::max(maxElems, s.elems);
        maxZero = std::max<size_t>(maxZero, dd.strides[0] - s.zeroFrom);
        if (compute && params > 0)
        {
            if (s.lineCount >= uint32_t(kNormalizeWarpMinElems))
                for (uint32_t p = 0; p < params; ++p) tasks.push_back(make_int4(b, int(p), 1, 1));
            else
                for (uint32_t p = 0; p < params; p += 32)
                    tasks.push_back(make_int4(b, int(p), int(std::min<uint32_t>(32, params - p)), 0));
        }
    }
    const size_t perAll = size_t(n) * maxSize;
    const size_t meanInCount = compute == 0 ? size_t(maxSize) : perAll;
    Carver m(nullptr);
    m.take<NormNdSample>(n);
    m.take<int4>(tasks.size());
    m.take<float>(perAll);
    m.take<float>(perAll);
    m.take<float>(maxSize);
    m.take<float>(meanInCount);
    m.take<float>(meanInCount);
    Carver cv(h.workspace(m.used()));
    NormNdSample* dSamples = cv.take<NormNdSample>(n);
    int4* dTasks = cv.take<int4>(tasks.size());
    float* meanOut = cv.take<float>(perAll);
    float* invOut = cv.take<float>(perAll);
    float* inverted = cv.take<float>(maxSize);
    float* meanStage = cv.take<float>(meanInCount);
    float* stdStage = cv.take<float>(meanInCount);
    h.upload(dSamples, samples.data(), samples.size() * sizeof(NormNdSample));
    if (!tasks.empty()) h.upload(dTasks, tasks.data(), tasks.size() * sizeof(int4));
    NormNdArgs a;
    a.src = static_cast<const char*>(srcPtr) + sd.offsetInBytes;
    a.dst = static_cast<char*>(dstPtr) + dd.offsetInBytes;
    a.type = ts;
    a.srcElem = a.dstElem = ts == kNormF32 ? 4 : ts == kNormF16 ? 2 : 1;
    a.n = n;
    a.srcStride0 = sd.strides[0];
    a.dstStride0 = dd.strides[0];
    a.compute = compute;
    a.scale = scale;
    a.shift = shift;
    a.maxSize = maxSize;
    a.samples = dSamples;
    a.meanIn = (compute & 1) ? nullptr
                             : static_cast<const float*>(h.device_view(meanTensor, meanInCount * 4, meanStage));
    a.meanOut = meanOut;
    a.invOut = invOut;
    const float* stdIn =
        (compute & 2) ? nullptr : static_cast<const float*>(h.device_view(stdDevTensor, meanInCount * 4, stdStage));
    const float* meanEff = (compute & 1) ? meanOut : a.meanIn;
    const float* invEff = (compute & 2) ? invOut : compute == 0 ? inverted : stdIn;
    // the caller's values: where the N-D branch starts its sums, and what entries past a sample's
    // parameter count keep
    if (compute & 1)
        check_cuda(cudaMemcpyAsync(meanOut, meanTensor, perAll * 4, cudaMemcpyDefault, h.stream()),
                   "cudaMemcpyAsync(mean in)");
    if (compute & 2)
        check_cuda(cudaMemcpyAsync(invOut, stdDevTensor, perAll * 4, cudaMemcpyDefault, h.stream()),
                   "cudaMemcpyAsync(stdDev in)");
    check_tensors(h, srcPtr, sd, dstPtr, dd, n);
    launch_normalize_nd(h, a, dTasks, int(tasks.size()), meanEff, invEff, compute == 0 ? 0 : maxSize, maxElems,
                        maxZero, stdIn, inverted, compute == 0 ? maxSize : 0);
    if (compute & 1)
        check_cuda(cudaMemcpyAsync(meanTensor, meanOut, perAll * 4, cudaMemcpyDefault, h.stream()),
                   "cudaMemcpyAsync(mean)");
    if (compute & 2)
        check_cuda(cudaMemcpyAsync(stdDevTensor, invOut, perAll * 4, cudaMemcpyDefault, h.stream()),
                   "cudaMemcpyAsync(stdDev)");
    return RPP_SUCCESS;
}

}  // namespace

extern "C" SHARED_PUBLIC RppStatus rppt_normalize_gpu(RppPtr_t srcPtr, RpptGenericDescPtr srcGenericDescPtr,
                                                      RppPtr_t dstPtr, RpptGenericDescPtr dstGenericDescPtr,
                                                      Rpp32u axisMask, Rpp32f* meanTensor, Rpp32f* stdDevTensor,
                                                      Rpp8u computeMeanStddev, Rpp32f scale, Rpp32f shift,
                                                      Rpp32u* roiTensor, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcGenericDescPtr && dstGenericDescPtr, "null descriptor");
        const RpptGenericDesc& sd = *srcGenericDescPtr;
        const RpptGenericDesc& dd = *dstGenericDescPtr;
        // the 2-D F32 tensors of the audio path (normalize.cpp's tensorDims == 2 branch) here; every
        // other type and rank in normalize_nd
        if (!(sd.dataType == F32 && dd.dataType == F32 && sd.numDims == 3 && dd.numDims == 3))
            return normalize_nd(h, srcPtr, sd, dstPtr, dd, axisMask, meanTensor, stdDevTensor, computeMeanStddev & 3,
                                scale, shift, roiTensor);
        if (axisMask < 1 || axisMask > 3) return RPP_ERROR_INVALID_ARGUMENTS;
        require(srcPtr && dstPtr && roiTensor && meanTensor && stdDevTensor, "null tensor");
        const int n = int(dd.dims[0]);
        if (n <= 0) return RPP_SUCCESS;
        const int compute = computeMeanStddev & 3;
        // roi lengths are needed on the host (parameter counts, work list)
        const std::vector<uint32_t> roi = roi_to_host(h, roiTensor, size_t(n) * 4);
        int maxSize = 1;
        std::vector<NormalizeSample> samples(n);
        std::vector<int4> tasks;
        for (int b = 0; b < n; ++b)
        {
            const uint32_t l0 = roi[4 * b + 2], l1 = roi[4 * b + 3];
            int size = 1;
            if (!(axisMask & 1)) size *= int(l0);
            if (!(axisMask & 2)) size *= int(l1);
            maxSize = std::max(maxSize, size);
            NormalizeSample& s = samples[b];
            s.len0 = int(std::min(l0, sd.dims[1]));
            s.len1 = int(std::min(l1, sd.dims[2]));
            int params;
            if (axisMask == 3)
            {
                s.count = s.len0 * s.len1;
                s.elemStride = int(sd.strides[2]);
                s.paramStride = 0;
                params = 1;
            }
            else if (axisMask == 1)
            {
                s.count = s.len0;
                s.elemStride = int(sd.strides[1]);
                s.paramStride = int(sd.strides[2]);
                params = s.len1;
            }
            else
            {
                s.count = s.len1;
                s.elemStride = int(sd.strides[2]);
                s.paramStride = int(sd.strides[1]);
                params = s.len0;
            }
            s.normFactor = float(1.0 / double(s.count));
            if (compute)
            {
                if (s.count >= kNormalizeWarpMinElems)
                    for (int p = 0; p < params; ++p) tasks.push_back(make_int4(b, p, 1, 1));
                else
                    for (int p = 0; p < params; p += 32) tasks.push_back(make_int4(b, p, std::min(32, params - p), 0));
            }
        }
        const size_t perAll = size_t(n) * maxSize;
        const size_t meanInCount = compute == 0 ? size_t(maxSize) : perAll;
        Carver m(nullptr);
        m.take<NormalizeSample>(n);
        m.take<int4>(tasks.size());
        m.take<float>(perAll);
        m.take<float>(perAll);
        m.take<float>(maxSize);
        m.take<float>(meanInCount);
        m.take<float>(meanInCount);
        Carver cv(h.workspace(m.used()));
        NormalizeSample* dSamples = cv.take<NormalizeSample>(n);
        int4* dTasks = cv.take<int4>(tasks.size());
        float* meanOut = cv.take<float>(perAll);
        float* invOut = cv.take<float>(perAll);
        float* inverted = cv.take<float>(maxSize);
        float* meanStage = cv.take<float>(meanInCount);
        float* stdStage = cv.take<float>(meanInCount);
        h.upload(dSamples, samples.data(), samples.size() * sizeof(NormalizeSample));
        if (!tasks.empty()) h.upload(dTasks, tasks.data(), tasks.size() * sizeof(int4));
        NormalizeArgs a;
        a.src = reinterpret_cast<const float*>(static_cast<const char*>(srcPtr) + sd.offsetInBytes);
        a.dst = reinterpret_cast<float*>(static_cast<char*>(dstPtr) + dd.offsetInBytes);
        a.n = n;
        a.srcStride0 = sd.strides[0];
        a.srcStride1 = sd.strides[1];
        a.srcStride2 = sd.strides[2];
        a.dstStride0 = dd.strides[0];
        a.dstStride1 = dd.strides[1];
        if (a.dstStride1 == 0) return RPP_ERROR_INVALID_ARGUMENTS;
        a.axisMask = axisMask;
        a.compute = compute;
        a.scale = scale;
        a.shift = shift;
        a.maxSize = maxSize;
        a.samples = dSamples;
        a.meanIn = (compute & 1) ? nullptr
                                 : static_cast<const float*>(h.device_view(meanTensor, meanInCount * 4, meanStage));
        a.meanOut = meanOut;
        a.invOut = invOut;
        const float* stdIn = (compute & 2) ? nullptr
                                           : static_cast<const float*>(h.device_view(stdDevTensor, meanInCount * 4,
                                                                                     stdStage));
        const float* meanEff = (compute & 1) ? meanOut : a.meanIn;
        const float* invEff = (compute & 2) ? invOut : compute == 0 ? inverted : stdIn;
        // entries past a sample's parameter count keep the caller's values, as in the reference
        if (compute & 1)
            check_cuda(cudaMemcpyAsync(meanOut, meanTensor, perAll * 4, cudaMemcpyDefault, h.stream()),
                       "cudaMemcpyAsync(mean in)");
        if (compute & 2)
            check_cuda(cudaMemcpyAsync(invOut, stdDevTensor, perAll * 4, cudaMemcpyDefault, h.stream()),
                       "cudaMemcpyAsync(stdDev in)");
        check_tensors(h, srcPtr, sd, dstPtr, dd, n);
        launch_normalize(h, a, dTasks, int(tasks.size()), meanEff, invEff, compute == 0 ? 0 : maxSize, stdIn,
                         inverted, compute == 0 ? maxSize : 0);
        // computed statistics go back to the caller's arrays, as the reference writes them
        if (compute & 1)
            check_cuda(cudaMemcpyAsync(meanTensor, meanOut, perAll * 4, cudaMemcpyDefault, h.stream()),
                       "cudaMemcpyAsync(mean)");
        if (compute & 2)
            check_cuda(cudaMemcpyAsync(stdDevTensor, invOut, perAll * 4, cudaMemcpyDefault, h.stream()),
                       "cudaMemcpyAsync(stdDev)");
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_pcm16_to_f32_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                         RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor,
                                                         rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        if (srcDescPtr->dataType != I16) return RPP_ERROR_INVALID_SRC_DATATYPE;
        if (dstDescPtr->dataType != F32) return RPP_ERROR_INVALID_DST_DATATYPE;
        if (srcDescPtr->c != dstDescPtr->c || srcDescPtr->c == 0) return RPP_ERROR_INVALID_ARGUMENTS;
        require(srcPtr && dstPtr, "null tensor");
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        Carver m(nullptr);
        m.take<int>(n);
        Carver cv(h.workspace(m.used()));
        int* lenStage = cv.take<int>(n);
        const int* len = static_cast<const int*>(h.device_view(srcLengthTensor, n * sizeof(int), lenStage));
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_pcm16(h, reinterpret_cast<const short*>(static_cast<const char*>(srcPtr) + srcDescPtr->offsetInBytes),
                     srcDescPtr->strides.nStride,
                     reinterpret_cast<float*>(static_cast<char*>(dstPtr) + dstDescPtr->offsetInBytes),
                     dstDescPtr->strides.nStride, len, int(srcDescPtr->c), n);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_mel_filter_bank_tc_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                               RpptDescPtr dstDescPtr, Rpp32s* srcDimsTensor,
                                                               Rpp32f maxFreq, Rpp32f minFreq,
                                                               RpptMelScaleFormula melFormula, Rpp32s numFilter,
                                                               Rpp32f sampleRate, bool normalize,
                                                               RppbTensorCorePrecision precision, rppHandle_t rppHandle)
{
    return guarded(rppHandle, [&](Handle& h) {
        require(srcDescPtr && dstDescPtr, "null descriptor");
        if (srcDescPtr->numDims != 3) return RPP_ERROR_INVALID_SRC_DIMS;
        if (srcDescPtr->layout != NFT) return RPP_ERROR_INVALID_SRC_LAYOUT;
        if (dstDescPtr->layout != NFT) return RPP_ERROR_INVALID_DST_LAYOUT;
        if (maxFreq < 0 || maxFreq > sampleRate / 2) return RPP_ERROR_INVALID_ARGUMENTS;
        if (minFreq < 0 || minFreq > sampleRate / 2) return RPP_ERROR_INVALID_ARGUMENTS;
        if (!(is_f32(srcDescPtr) && is_f32(dstDescPtr))) return RPP_ERROR_NOT_IMPLEMENTED;
        require(srcPtr && dstPtr && srcDimsTensor, "null tensor");
        require(numFilter > 0, "numFilter must be positive");
        const int fmt = int(precision);
        if (fmt < kTcBf16 || fmt > kTcFp8 || numFilter > 256) return RPP_ERROR_NOT_IMPLEMENTED;
        if (dstDescPtr->h < Rpp32u(numFilter)) return RPP_ERROR_INVALID_DST_DIMS;
        const int bins = int(srcDescPtr->h);
        if (bins < 2) return RPP_ERROR_INVALID_SRC_DIMS;
        const int n = int(srcDescPtr->n);
        if (n <= 0) return RPP_SUCCESS;
        const int maxFrames = int(std::min(dstDescPtr->w, srcDescPtr->strides.hStride));
        const size_t scratchBytes = tc_mel_scratch_bytes(n, fmt, bins, maxFrames);
        Carver m(nullptr);
        m.take<int>(2 * n);
        m.take<char>(scratchBytes);
        Carver cv(h.workspace(m.used()));
        int* dimsStage = cv.take<int>(2 * n);
        void* scratch = cv.take<char>(scratchBytes);
        TcMelArgs a;
        a.src = static_cast<const float*>(srcPtr);
        a.srcNStride = srcDescPtr->strides.nStride;
        a.srcHStride = srcDescPtr->strides.hStride;
        a.bins = bins;
        a.dims = static_cast<const int*>(h.device_view(srcDimsTensor, 2 * n * sizeof(int), dimsStage));
        a.n = n;
        a.maxFrames = maxFrames;
        a.fmt = fmt;
        a.mel.minFreq = minFreq;
        a.mel.maxFreq = (maxFreq == 0) ? sampleRate / 2 : maxFreq;
        a.mel.sampleRate = sampleRate;
        a.mel.htk = melFormula == HTK ? 1 : 0;
        a.mel.numFilter = numFilter;
        a.mel.normalize = normalize;
        a.dst = static_cast<float*>(dstPtr);
        a.dstNStride = dstDescPtr->strides.nStride;
        a.dstHStride = dstDescPtr->strides.hStride;
        check_tensors(h, srcPtr, srcDescPtr, dstPtr, dstDescPtr, n);
        launch_tc_mel(h, scratch, a);
        return RPP_SUCCESS;
    });
}
