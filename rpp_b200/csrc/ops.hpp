// Launchers of the audio kernels.  Every pointer is a device address (per-sample tensors are
// already resolved by the dispatch layer); every launch goes on h.stream().  Each launcher takes
// a device `scratch` region of at least <op>_scratch_bytes(...) bytes, carved by the dispatch
// layer out of the handle workspace.
#pragma once

#include "../../include/rppb_frontend.h"
#include "handle.hpp"

namespace rppb {

inline size_t prefix_bytes(int n) { return size_t(n + 1) * sizeof(long long); }

void launch_pre_emphasis(Handle& h, void* scratch, const float* src, uint32_t srcStride, float* dst,
                         uint32_t dstStride, int n, const int* len, const float* coeff, int border, size_t srcElems);

void launch_down_mixing(Handle& h, void* scratch, const float* src, uint32_t srcStride, float* dst,
                        uint32_t dstStride, int n, const int* dims, bool normalize);

struct ResampleWindowDev
{
    const float* lut;
    int lutSize;
    float scale, center;
    int lobes;
    int padLeft = 0, padRight = 0;   // set by the resample launchers (shared-memory pair table padding)
    // set by the resample launchers: outputs whose phase has a binary exponent in [exactMinE, exactMaxE]
    // take the exact walk (every tap position exact in float; resample.cu)
    int exactMinE = 1 << 30, exactMaxE = -(1 << 30);
};
// downmix: the input is interleaved {length, channels} and is down-mixed to mono while resampling
// (equal to rppt_down_mixing_gpu followed by a mono rppt_resample_gpu).
void launch_resample(Handle& h, void* scratch, const float* src, uint32_t srcStride, float* dst, uint32_t dstStride, int n,
                     const float* inRate, const float* outRate, const int* dims, const ResampleWindowDev& win,
                     bool downmix = false, bool normalize = false);
// Mono resample of a clip table: clips[b].src (length at inRate) -> clips[b].work at outRate.
void launch_resample_clips(Handle& h, void* scratch, const RppbClip* clips, int n, float outRate,
                           const ResampleWindowDev& win);

struct SpectrogramArgs
{
    const float* src;
    uint32_t srcStride;
    float* dst;
    uint32_t dstNStride, dstHStride;
    bool nft;
    int n;
    const int* len;
    bool center, reflect;
    const float* window;   // device, windowLength floats
    int nfft, power, windowLength, windowStep;
    int maxFrames;         // frames the dst descriptor holds per sample
};
void launch_spectrogram(Handle& h, void* scratch, const SpectrogramArgs& a);

struct MelArgs
{
    const float* src;
    uint32_t srcNStride, srcHStride;
    float* dst;
    uint32_t dstNStride, dstHStride;
    int n;
    const int* dims;       // {bins, frames} per sample
    uint32_t srcRows;      // bins the src descriptor holds per sample
    float maxFreq, minFreq;
    int htk;
    int numFilter;
    float sampleRate;
    bool normalize;
};
void launch_mel_filter_bank(Handle& h, void* scratch, const MelArgs& a);

struct DecibelArgs
{
    const float* src;
    uint32_t srcNStride, srcHStride;
    float* dst;
    uint32_t dstNStride, dstHStride;
    int n;
    const uint32_t* dims;  // {width, height} per sample
    float minRatio;        // pow(10, cutOffDB / multiplier), denorm-min when 0
    float multiplier;      // multiplier * log10(2)
    float referenceMagnitude;
};
inline size_t to_decibels_scratch_bytes(int n) { return prefix_bytes(n) + 256 + size_t(n) * sizeof(unsigned); }
void launch_to_decibels(Handle& h, void* scratch, const DecibelArgs& a);

struct NsrArgs
{
    const float* src;
    uint32_t srcStride;
    int n;
    const int* len;
    int* begin;            // device-writable
    int* length;
    float cutOff;          // powf(10, cutOffDB * 0.1f)
    int windowLength;
    float referencePower;
    int resetInterval;
};
// Moving-mean-square buffer (srcStride floats per sample), per-reset-block maxima and the prefix.
size_t nsr_scratch_bytes(int n, uint32_t srcStride, int resetInterval);
void launch_nsr(Handle& h, void* scratch, const NsrArgs& a);

// Mel filter placement parameters (maxFreq already resolved: 0 -> sampleRate / 2).
struct MelParams
{
    float minFreq, maxFreq;
    float sampleRate;
    int htk;
    int numFilter;
    bool normalize;
};

// Twiddle table W_nfft^e = (cos, sin)(2*pi*e/nfft), e < nfft, cached on the handle.
const float2* spectrogram_twiddles(Handle& h, int nfft);

struct FrontendArgs
{
    const float* src;
    uint32_t srcStride;
    size_t srcElems;
    float* dst;
    uint32_t dstNStride, dstHStride;
    int n;
    const int* len;
    const float* coeff;
    int border;
    bool center, reflect;
    const float* window;     // device, W floats
    int nfft, W, hop, maxFrames, power;
    MelParams mel;
    float minRatio, multiplier, refMag;
    int lookahead;
    // clip-table mode (clips != nullptr): clip b reads clips[b].work (clips[b].length resampled from
    // inRate to outRate), writes clips[b].dst with hStride clips[b].dstStride, pre-emphasis coeffAll
    const RppbClip* clips;
    float outRate;
    float coeffAll;
    int reserveSms;          // SMs' worth of CTA slots left to kernels on other streams
    // schedule (never the arithmetic): frames per spectrum item (0: the plan's tile; else 1, 2 or
    // 4 tiles), frames per decibel item (0: 128), CTAs per SM (0: as many as fit)
    int tileFrames, dbFrames, ctasPerSm;
    int subTiles;            // set by launch_frontend: tiles per spectrum item
    // set by launch_frontend from the handle's wait fault injection (test only): tiles a decibel
    // item waits for beyond its clip's, and the poll limit of that wait (0: the default)
    int waitExtra;
    long long waitLimit;
    // spectrum engine: 0 the FP32 register FFT (bit-identical to the plain calls), 1 the factored DFT
    // on tensor cores in BF16 hi/lo x3 (fused_tc.cu; nfft 512 only)
    int engine;
};
size_t frontend_scratch_bytes(int n, int lookahead, int numFilter);
void launch_frontend(Handle& h, void* scratch, const FrontendArgs& a);
// The tensor-core engine (fused_tc.cu): launched by launch_frontend for engine 1; `melScratch` holds the
// mel tables when the handle's cache cannot provide them (stream capture with new parameters).
// rppb_frontend_clips_gpu on a handle, leaving `reserveSms` SMs' worth of CTA slots of the fused kernel
// to kernels on other streams (the server's copy movers).
RppStatus frontend_clips(Handle& h, const RppbClip* clips, int numClips, float outRate, const float* lookup,
                         int lookupSize, float scale, float center, int lobes, float preemphCoeff,
                         const RppbFrontendParams* params, int reserveSms);
bool frontend_tc_supported(const FrontendArgs& a);
void launch_frontend_tc(Handle& h, const FrontendArgs& a, void* scratch, uint4* melScratch);

// slice (slice.cu): 1-D or 2-D boxes per sample, strides in elements.
struct SliceArgs
{
    int n, numDims, elemBytes;
    uint32_t srcStride0, srcStride1, dstStride0, dstStride1;
    uint32_t srcDim0, srcDim1;   // extents of a sample (lengths are clamped to them)
    const int* anchor;           // device views, n * numDims
    const int* shape;
    const uint32_t* roi;         // n * numDims * 2: begins (unused), then lengths
    bool enablePadding;
    int unitsPerSample;          // set by launch_slice
    // 3-D and 4-D boxes
    int layoutKind;              // 1: channel-first (NCHW, NCDHW), 2: channel-last (NHWC, NDHWC)
    uint32_t srcStrides[5], dstStrides[5];   // the descriptors' strides[0 .. numDims]
    uint32_t srcDims[4], dstDims[4];         // the descriptors' dims[1 .. numDims]
};
void launch_slice(Handle& h, const SliceArgs& a, const void* src, void* dst, const void* fill);

// normalize (normalize.cu): 2-D F32, per-sample roi lengths.
// Reductions of at least this many elements run one warp per parameter (normalize.cu).
constexpr int kNormalizeWarpMinElems = 544;

struct NormalizeSample
{
    int len0, len1;          // roi lengths (rows, columns)
    int count;               // elements per parameter
    int elemStride;          // stride between a parameter's elements
    int paramStride;         // stride between consecutive parameters
    float normFactor;        // float(1.0 / count)
};
struct NormalizeArgs
{
    const float* src;
    float* dst;
    int n;
    uint32_t srcStride0, srcStride1, srcStride2, dstStride0, dstStride1;
    unsigned axisMask;
    int compute;             // computeMeanStddev
    float scale, shift;
    int maxSize;             // parameters per sample in the mean / std arrays
    const NormalizeSample* samples;   // device, n
    const float* meanIn;     // caller's means (device view) when not computed
    float* meanOut;          // computed means, n * maxSize
    float* invOut;           // computed inverse std devs, n * maxSize
};
void launch_normalize(Handle& h, const NormalizeArgs& a, const int4* tasks, int numTasks, const float* meanEff,
                      const float* invEff, int paramOffsetPerSample, const float* stdToInvert, float* invertOut,
                      int invertCount);

// normalize, every other type and rank (normalize_nd.cu): per-sample plans built by the dispatch.
constexpr int kNormF32 = 0, kNormF16 = 1, kNormU8 = 2, kNormI8 = 3;
struct NormNdLevel
{
    uint32_t count, srcStride, dstStride, paramMult;
};
struct NormNdSample
{
    // statistics: parameter p = row-major over pLevels (count, source stride); its lines row-major
    // over oLevels; each line lineCount elements lineStride apart
    int pLevels, oLevels;
    uint32_t pCount[4], pStride[4], oCount[4], oStride[4];
    uint32_t lineStride, lineCount;
    float normFactor;
    int accumulate;          // sums start from the caller's mean / std-dev value (the N-D branch)
    // output: elems elements row-major over `levels`
    int levels;
    NormNdLevel lv[4];
    size_t elems;
    size_t srcBase;          // source element offset of the roi start within the sample
    size_t zeroFrom;         // destination elements [zeroFrom, dstStride0) are cleared
};
struct NormNdArgs
{
    const void* src;
    void* dst;
    int type, srcElem, dstElem;   // kNorm*, element sizes in bytes
    int n;
    size_t srcStride0, dstStride0;
    int compute;
    float scale, shift;
    int maxSize;
    const NormNdSample* samples;  // device, n
    const float* meanIn;
    float* meanOut;
    float* invOut;
};
void launch_normalize_nd(Handle& h, const NormNdArgs& a, const int4* tasks, int numTasks, const float* meanEff,
                         const float* invEff, int paramOffsetPerSample, size_t maxElems, size_t maxZero,
                         const float* stdToInvert, float* invertOut, int invertCount);

// 16-bit PCM ingest (pcm.cu).
void launch_pcm16(Handle& h, const short* src, uint32_t srcStride, float* dst, uint32_t dstStride, const int* len,
                  int channels, int n);

// PCIe movers over mapped pinned host memory (host_io.cu).
// A contiguous copy of `count` floats for launch_copy_jobs (host_io.cu); unit0 = the segments of the
// jobs before it (copy_job_segments per job, scanned).
struct CopyJob
{
    const float* src;
    float* dst;
    long long count;
    long long unit0;
};
long long copy_job_segments(long long count);
// One launch that performs every job of `jobs` (device-visible memory: device, or pinned host).
void launch_copy_jobs(cudaStream_t stream, const CopyJob* jobs, int njobs, long long units, int ctas);
void launch_host_gather(cudaStream_t stream, const float* src, size_t nStride, const int* len, int clips, float* dst,
                        uint32_t dstStride, int ctas);
void launch_host_scatter(cudaStream_t stream, const float* src, uint32_t srcNStride, uint32_t srcHStride,
                         const int* frames, int clips, int rows, float* dst, size_t dstNStride, size_t dstHStride,
                         int ctas);

// Tensor-core spectrogram (tc_dft.cu).
enum TcFormat
{
    kTcBf16 = 0,       // BF16 operands, one pass
    kTcBf16x3 = 1,     // BF16 hi + lo split, three passes (hi*hi + hi*lo + lo*hi)
    kTcTf32 = 2,       // TF32 operands (FP32 rounded to 10 mantissa bits)
    kTcFp8 = 3,        // FP8 E4M3 operands, frames scaled to the format's range one by one
};
struct TcGeometry
{
    int kPad;            // window length rounded up to one 128-byte row of operand elements
    uint32_t rowStep;    // elements between consecutive frames' rows of the A operand
    uint32_t clipStride; // elements per clip of the A operand
    size_t basisFloats;  // size of the cached basis table, in floats
    bool materialized;   // frame rows written out [frame][kPad] (FP8, or no overlapping-row tensor map)
};
// Whether the driver encodes a tensor map whose rows overlap (frame rows hop elements apart);
// anyDevicePtr: any 16-byte aligned device allocation (only encoded, never accessed).
bool tc_overlap_supported(const void* anyDevicePtr);
TcGeometry tc_geometry(int fmt, int windowLength, int windowStep, int maxFrames, int nfft, bool overlapRows);
// Window-folded DFT basis [nfft][kPad] in the format's element type (hi then lo for kTcBf16x3).
void tc_build_basis(float* out, int fmt, int nfft, int windowLength, int kPad, const float* window);
struct TcSpectrogramArgs
{
    const float* src;
    uint32_t srcStride;
    size_t srcElems;
    const int* len;
    const float* coeff;       // pre-emphasis coefficients, nullptr: none
    int border;
    bool center, reflect;
    int windowLength, windowStep, nfft;
    int fmt;
    TcGeometry geo;
    int maxFrames;
    const void* basis;
    float* dst;
    uint32_t dstNStride, dstHStride;
    bool nft;
    int power;
    int n;
};
size_t tc_spectrogram_scratch_bytes(int n, int fmt, const TcGeometry& g, int maxFrames);
// Mel projection on tensor cores (tc_dft.cu): NFT spectra -> NFT mel, numFilter <= 256.
struct TcMelArgs
{
    const float* src;
    uint32_t srcNStride, srcHStride;
    int bins;                 // spectrum rows (nfft / 2 + 1)
    const int* dims;          // device: per sample {bins, frames}
    int n, maxFrames, fmt;
    MelParams mel;
    float* dst;
    uint32_t dstNStride, dstHStride;
};
size_t tc_mel_scratch_bytes(int n, int fmt, int bins, int maxFrames);
void launch_tc_mel(Handle& h, void* scratch, const TcMelArgs& a);
void launch_tc_spectrogram(Handle& h, void* scratch, const TcSpectrogramArgs& a);

}  // namespace rppb
