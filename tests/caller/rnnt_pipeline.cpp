// A C++ caller of the audio path written the way an augmentation pipeline (MIVisionX / rocAL style)
// binds RPP: it includes only include/*.h, links librppb.so, creates one handle on its own CUDA
// stream, keeps the per-sample tensors in pinned host memory and runs the RNN-T speech front end
//
//   int16 PCM -> float (rppb_pcm16_to_f32_gpu)
//   -> non_silent_region_detection (-60 dB, window 2048, reset 8192) -> slice to the detected region
//   -> pre_emphasis (0.97, ZERO) -> spectrogram (512, Hann 400, hop 160, centred, reflect, power 2)
//   -> mel_filter_bank (128, 0-8 kHz, Slaney, normalized) -> to_decibels (x10, -80 dB, per-clip max)
//   -> normalize (per filter over time, computed mean and std dev)
//
// reading NSR's results back on the host to size the later stages, as such pipelines do.  Every
// stage's output is written to <outdir>/<stage>.bin (raw, the shapes the caller's descriptors give)
// for the test that checks each stage against the oracle.
//
//   rnnt_pipeline <input.bin> <outdir>
//   input.bin: int32 n, int32 w (samples per clip slot), int32 lengths[n], int16 pcm[n][w]
//
// Exit status 0 on success; on the first failing call it prints the call and its status and
// returns 1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rpp.h"
#include "rppb_frontend.h"
#include "rppt_tensor_audio_augmentations.h"
#include "rppt_tensor_geometric_augmentations.h"
#include "rppt_tensor_statistical_operations.h"

namespace {

constexpr int kNfft = 512, kWin = 400, kHop = 160, kBins = kNfft / 2 + 1, kMel = 128;

#define CHECK_CUDA(call)                                                                      \
    do                                                                                        \
    {                                                                                         \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
        {                                                                                     \
            std::fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));           \
            return 1;                                                                         \
        }                                                                                     \
    } while (0)
#define CHECK_RPP(call)                                                                       \
    do                                                                                        \
    {                                                                                         \
        int s_ = int(call);                                                                   \
        if (s_ != 0)                                                                          \
        {                                                                                     \
            std::fprintf(stderr, "%s returned %d\n", #call, s_);                              \
            return 1;                                                                         \
        }                                                                                     \
    } while (0)

// 1-D signals: numDims 2, [n][w], one channel
RpptDesc signal_desc(Rpp32u n, Rpp32u w, RpptDataType type)
{
    RpptDesc d{};
    d.numDims = 2;
    d.dataType = type;
    d.n = n;
    d.c = 1;
    d.h = 1;
    d.w = w;
    d.strides.nStride = w;
    d.strides.hStride = w;
    d.strides.wStride = 1;
    d.strides.cStride = 1;
    d.layout = NFT;
    return d;
}

// 2-D spectra: numDims 3, [n][rows][cols], frequency-major
RpptDesc spectra_desc(Rpp32u n, Rpp32u rows, Rpp32u cols)
{
    RpptDesc d{};
    d.numDims = 3;
    d.dataType = F32;
    d.n = n;
    d.c = 1;
    d.h = rows;
    d.w = cols;
    d.strides.nStride = rows * cols;
    d.strides.hStride = cols;
    d.strides.wStride = 1;
    d.strides.cStride = 1;
    d.layout = NFT;
    return d;
}

RpptGenericDesc generic_desc(std::vector<Rpp32u> dims)
{
    RpptGenericDesc d{};
    d.numDims = dims.size();
    d.dataType = F32;
    Rpp32u stride = 1;
    for (int i = int(dims.size()) - 1; i >= 0; --i)
    {
        d.dims[i] = dims[i];
        d.strides[i] = stride;
        stride *= dims[i];
    }
    d.layout = NCHW;
    return d;
}

template <class T>
T* pinned(size_t count)
{
    void* p = nullptr;
    if (cudaMallocHost(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    std::memset(p, 0, std::max<size_t>(count, 1) * sizeof(T));
    return static_cast<T*>(p);
}

bool write_file(const std::string& path, const void* data, size_t bytes)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

// device buffer -> <dir>/<name>.bin
int dump(const std::string& dir, const char* name, const void* dev, size_t bytes)
{
    std::vector<char> h(bytes);
    CHECK_CUDA(cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost));
    if (!write_file(dir + "/" + name + ".bin", h.data(), bytes))
    {
        std::fprintf(stderr, "cannot write %s\n", name);
        return 1;
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3)
    {
        std::fprintf(stderr, "usage: %s <input.bin> <outdir>\n", argv[0]);
        return 2;
    }
    const std::string outDir = argv[2];
    FILE* f = std::fopen(argv[1], "rb");
    if (!f)
    {
        std::fprintf(stderr, "cannot open %s\n", argv[1]);
        return 1;
    }
    int32_t hdr[2] = {0, 0};
    if (std::fread(hdr, sizeof(int32_t), 2, f) != 2 || hdr[0] <= 0 || hdr[1] <= 0)
    {
        std::fclose(f);
        std::fprintf(stderr, "bad header\n");
        return 1;
    }
    const Rpp32u n = Rpp32u(hdr[0]), w = Rpp32u(hdr[1]);
    std::vector<int32_t> lengths(n);
    std::vector<int16_t> pcm(size_t(n) * w);
    const bool readOk = std::fread(lengths.data(), sizeof(int32_t), n, f) == n &&
                        std::fread(pcm.data(), sizeof(int16_t), pcm.size(), f) == pcm.size();
    std::fclose(f);
    if (!readOk)
    {
        std::fprintf(stderr, "short input\n");
        return 1;
    }

    cudaStream_t stream;
    CHECK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    rppHandle_t handle = nullptr;
    CHECK_RPP(rppCreate(&handle, n, 0, stream, RPP_HIP_BACKEND));

    // per-sample tensors in pinned memory, as the pipeline's graph keeps them
    Rpp32s* len = pinned<Rpp32s>(n);
    Rpp32s* begin = pinned<Rpp32s>(n);
    Rpp32s* detected = pinned<Rpp32s>(n);
    Rpp32f* coeff = pinned<Rpp32f>(n);
    Rpp32u* sliceRoi = pinned<Rpp32u>(2 * n);
    Rpp32f* fill = pinned<Rpp32f>(1);
    Rpp32s* melDims = pinned<Rpp32s>(2 * n);
    RpptImagePatch* patches = pinned<RpptImagePatch>(n);
    Rpp32u* normRoi = pinned<Rpp32u>(4 * n);
    if (!len || !begin || !detected || !coeff || !sliceRoi || !fill || !melDims || !patches || !normRoi)
    {
        std::fprintf(stderr, "cudaMallocHost failed\n");
        return 1;
    }
    for (Rpp32u b = 0; b < n; ++b)
    {
        len[b] = lengths[b];
        coeff[b] = 0.97f;
    }

    // ---- ingest and voice-activity trim
    int16_t* dPcm = nullptr;
    float *dSig = nullptr, *dTrim = nullptr, *dPre = nullptr;
    CHECK_CUDA(cudaMalloc(&dPcm, pcm.size() * sizeof(int16_t)));
    CHECK_CUDA(cudaMalloc(&dSig, size_t(n) * w * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dTrim, size_t(n) * w * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dPre, size_t(n) * w * sizeof(float)));
    CHECK_CUDA(cudaMemsetAsync(dSig, 0, size_t(n) * w * sizeof(float), stream));
    CHECK_CUDA(cudaMemsetAsync(dTrim, 0, size_t(n) * w * sizeof(float), stream));
    CHECK_CUDA(cudaMemsetAsync(dPre, 0, size_t(n) * w * sizeof(float), stream));
    CHECK_CUDA(cudaMemcpyAsync(dPcm, pcm.data(), pcm.size() * sizeof(int16_t), cudaMemcpyHostToDevice, stream));

    RpptDesc pcmDesc = signal_desc(n, w, I16), sigDesc = signal_desc(n, w, F32);
    CHECK_RPP(rppb_pcm16_to_f32_gpu(dPcm, &pcmDesc, dSig, &sigDesc, len, handle));
    CHECK_RPP(rppt_non_silent_region_detection_gpu(dSig, &sigDesc, len, begin, detected, -60.0f, 2048, 0.0f, 8192,
                                                   handle));
    CHECK_CUDA(cudaStreamSynchronize(stream));   // the host sizes the later stages from NSR's results

    RpptGenericDesc slDesc = generic_desc({n, w});
    for (Rpp32u b = 0; b < n; ++b)
    {
        sliceRoi[2 * b] = 0;
        sliceRoi[2 * b + 1] = Rpp32u(lengths[b]);
    }
    fill[0] = 0.f;
    CHECK_RPP(rppt_slice_gpu(dSig, &slDesc, dTrim, &slDesc, begin, detected, fill, false, sliceRoi, handle));

    // ---- spectral front end on the trimmed clips
    int maxFrames = 1;
    for (Rpp32u b = 0; b < n; ++b) maxFrames = std::max(maxFrames, detected[b] / kHop + 1);
    CHECK_RPP(rppt_pre_emphasis_filter_gpu(dTrim, &sigDesc, dPre, &sigDesc, detected, coeff, ZERO, handle));

    float *dSpec = nullptr, *dMel = nullptr, *dDb = nullptr, *dNorm = nullptr, *dMean = nullptr, *dStd = nullptr;
    const size_t specElems = size_t(n) * kBins * maxFrames, melElems = size_t(n) * kMel * maxFrames;
    CHECK_CUDA(cudaMalloc(&dSpec, specElems * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dMel, melElems * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dDb, melElems * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dNorm, melElems * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dMean, size_t(n) * kMel * sizeof(float)));
    CHECK_CUDA(cudaMalloc(&dStd, size_t(n) * kMel * sizeof(float)));
    CHECK_CUDA(cudaMemsetAsync(dSpec, 0, specElems * sizeof(float), stream));
    CHECK_CUDA(cudaMemsetAsync(dMel, 0, melElems * sizeof(float), stream));
    CHECK_CUDA(cudaMemsetAsync(dDb, 0, melElems * sizeof(float), stream));
    CHECK_CUDA(cudaMemsetAsync(dNorm, 0, melElems * sizeof(float), stream));

    RpptDesc specDesc = spectra_desc(n, kBins, Rpp32u(maxFrames)), melDesc = spectra_desc(n, kMel, Rpp32u(maxFrames));
    CHECK_RPP(rppt_spectrogram_gpu(dPre, &sigDesc, dSpec, &specDesc, detected, true, true, nullptr, kNfft, 2, kWin,
                                   kHop, handle));
    for (Rpp32u b = 0; b < n; ++b)
    {
        const int frames = detected[b] / kHop + 1;
        melDims[2 * b] = kBins;
        melDims[2 * b + 1] = frames;
        patches[b].width = Rpp32u(frames);
        patches[b].height = kMel;
        normRoi[4 * b] = 0;
        normRoi[4 * b + 1] = 0;
        normRoi[4 * b + 2] = kMel;
        normRoi[4 * b + 3] = Rpp32u(frames);
    }
    CHECK_RPP(rppt_mel_filter_bank_gpu(dSpec, &specDesc, dMel, &melDesc, melDims, 8000.0f, 0.0f, SLANEY, kMel,
                                       16000.0f, true, handle));
    CHECK_RPP(rppt_to_decibels_gpu(dMel, &melDesc, dDb, &melDesc, patches, -80.0f, 10.0f, 0.0f, handle));
    RpptGenericDesc featDesc = generic_desc({n, Rpp32u(kMel), Rpp32u(maxFrames)});
    CHECK_RPP(rppt_normalize_gpu(dDb, &featDesc, dNorm, &featDesc, 2, dMean, dStd, 3, 1.0f, 0.0f, normRoi, handle));
    CHECK_CUDA(cudaStreamSynchronize(stream));
    Rpp32s devErr = 0;
    CHECK_RPP(rppb_get_device_error(handle, &devErr));
    if (devErr != 0)
    {
        std::fprintf(stderr, "device error word %d\n", devErr);
        return 1;
    }

    // ---- outputs of every stage
    const int32_t meta[3] = {int32_t(n), int32_t(w), maxFrames};
    if (!write_file(outDir + "/meta.bin", meta, sizeof(meta)) ||
        !write_file(outDir + "/nsr_begin.bin", begin, n * sizeof(Rpp32s)) ||
        !write_file(outDir + "/nsr_length.bin", detected, n * sizeof(Rpp32s)))
    {
        std::fprintf(stderr, "cannot write outputs\n");
        return 1;
    }
    if (dump(outDir, "signal", dSig, size_t(n) * w * 4) || dump(outDir, "trimmed", dTrim, size_t(n) * w * 4) ||
        dump(outDir, "preemph", dPre, size_t(n) * w * 4) || dump(outDir, "spectrogram", dSpec, specElems * 4) ||
        dump(outDir, "mel", dMel, melElems * 4) || dump(outDir, "decibels", dDb, melElems * 4) ||
        dump(outDir, "normalized", dNorm, melElems * 4) || dump(outDir, "mean", dMean, size_t(n) * kMel * 4) ||
        dump(outDir, "inv_std", dStd, size_t(n) * kMel * 4))
        return 1;

    for (void* p : {static_cast<void*>(dPcm), static_cast<void*>(dSig), static_cast<void*>(dTrim),
                    static_cast<void*>(dPre), static_cast<void*>(dSpec), static_cast<void*>(dMel),
                    static_cast<void*>(dDb), static_cast<void*>(dNorm), static_cast<void*>(dMean),
                    static_cast<void*>(dStd)})
        CHECK_CUDA(cudaFree(p));
    for (void* p : {static_cast<void*>(len), static_cast<void*>(begin), static_cast<void*>(detected),
                    static_cast<void*>(coeff), static_cast<void*>(sliceRoi), static_cast<void*>(fill),
                    static_cast<void*>(melDims), static_cast<void*>(patches), static_cast<void*>(normRoi)})
        CHECK_CUDA(cudaFreeHost(p));
    CHECK_RPP(rppDestroy(handle, RPP_HIP_BACKEND));
    CHECK_CUDA(cudaStreamDestroy(stream));
    std::printf("ok %u clips, %d frames max\n", n, maxFrames);
    return 0;
}
