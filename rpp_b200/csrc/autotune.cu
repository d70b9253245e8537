// Autotuner of the fused front end's schedule (rppb_frontend_tune_gpu, include/rppb_frontend.h).
//
// The schedule knobs of RppbFrontendParams -- frames per spectrum item, frames per decibel item,
// the decibel lookahead in clips and CTAs per SM -- change which CTA does what and when, never the
// arithmetic of a frame, so every candidate writes the same bits.  The tuner times each candidate
// on the caller's own batch (one untimed call, then the fastest of `reps` timed calls, CUDA events
// on the handle stream), writes the winner into the caller's parameters and remembers it per
// (device, shape of the call) for the life of the process.  With RPPB_TUNE_CACHE naming a file, the
// winners are also read from and appended to that file, one line per key:
//   <key> <tileFrames> <dbFrames> <lookahead> <ctasPerSm> <ms>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rppb_frontend.h"
#include "handle.hpp"

namespace rppb {
namespace {

struct Choice
{
    int tileFrames, dbFrames, lookahead, ctasPerSm;
    float ms;
};

std::mutex g_tuneMu;
std::map<std::string, Choice> g_tuned;
bool g_fileLoaded = false;

int plan_tile_frames(int nfft) { return nfft >= 512 ? 16 : 32; }   // Plan<NFFT>::TF of stft.cuh

std::string tune_key(int device, const RpptDesc* sd, const RpptDesc* dd, const Rpp32s* lenHost,
                     const RppbFrontendParams& p)
{
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    std::ostringstream k;
    std::string name(prop.name);
    for (char& c : name)
        if (c == ' ') c = '_';
    // the shape of the work: clips, longest clip (power-of-two bucket) and the front-end geometry
    k << name << "/n" << sd->n << "/L" << (sd->strides.nStride ? 1u << (31 - __builtin_clz(sd->strides.nStride)) : 0)
      << "/nfft" << p.nfft << "/W" << p.windowLength << "/hop" << p.windowStep << "/mel" << p.numFilter << "/F"
      << dd->w << "/engine" << p.spectrumEngine;
    (void)lenHost;
    return k.str();
}

void load_file_locked()
{
    if (g_fileLoaded) return;
    g_fileLoaded = true;
    const char* path = std::getenv("RPPB_TUNE_CACHE");
    if (!path) return;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line))
    {
        std::istringstream ls(line);
        std::string key;
        Choice c{};
        if (ls >> key >> c.tileFrames >> c.dbFrames >> c.lookahead >> c.ctasPerSm >> c.ms) g_tuned[key] = c;
    }
}

void append_file(const std::string& key, const Choice& c)
{
    const char* path = std::getenv("RPPB_TUNE_CACHE");
    if (!path) return;
    std::ofstream out(path, std::ios::app);
    out << key << ' ' << c.tileFrames << ' ' << c.dbFrames << ' ' << c.lookahead << ' ' << c.ctasPerSm << ' ' << c.ms
        << '\n';
}

}  // namespace
}  // namespace rppb

using namespace rppb;

extern "C" SHARED_PUBLIC RppStatus rppb_frontend_tune_gpu(RppPtr_t srcPtr, RpptDescPtr srcDescPtr, RppPtr_t dstPtr,
                                                          RpptDescPtr dstDescPtr, Rpp32s* srcLengthTensor,
                                                          Rpp32f* coeffTensor, RppbFrontendParams* params,
                                                          Rpp32s reps, Rpp32f* bestMs, rppHandle_t rppHandle)
{
    try
    {
        if (!srcDescPtr || !dstDescPtr || !params) fail(RPP_ERROR_INVALID_ARGUMENTS, "null descriptor or parameters");
        Handle& h = deref(rppHandle);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        check_cuda(cudaStreamIsCapturing(h.stream(), &cap), "cudaStreamIsCapturing");
        if (cap != cudaStreamCaptureStatusNone) fail(RPP_ERROR_INVALID_ARGUMENTS, "tuning needs an uncaptured stream");
        const std::string key = tune_key(h.device(), srcDescPtr, dstDescPtr, srcLengthTensor, *params);
        {
            std::lock_guard<std::mutex> lk(g_tuneMu);
            load_file_locked();
            auto it = g_tuned.find(key);
            if (it != g_tuned.end())
            {
                params->tileFrames = it->second.tileFrames;
                params->dbFrames = it->second.dbFrames;
                params->lookahead = it->second.lookahead;
                params->ctasPerSm = it->second.ctasPerSm;
                if (bestMs) *bestMs = it->second.ms;
                return RPP_SUCCESS;
            }
        }
        const int t0 = plan_tile_frames(params->nfft);
        std::vector<Choice> cands;
        for (int tf : {t0, 2 * t0, 4 * t0})
            for (int db : {32, 64, 128})
                for (int la : {8, 32, 96})
                    // CTAs per SM: all that fit (3 for the FP32 engine, 2 for the tensor-core one) or fewer
                    for (int cps : {0, params->spectrumEngine == 1 ? 1 : 2}) cands.push_back(Choice{tf, db, la, cps, 0.f});
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        Choice best{0, 0, 0, 0, -1.f};
        RppStatus lastErr = RPP_SUCCESS;
        const int r = reps > 0 ? reps : 3;
        for (Choice& c : cands)
        {
            RppbFrontendParams p = *params;
            p.tileFrames = c.tileFrames;
            p.dbFrames = c.dbFrames;
            p.lookahead = c.lookahead;
            p.ctasPerSm = c.ctasPerSm;
            RppStatus st = rppb_frontend_gpu(srcPtr, srcDescPtr, dstPtr, dstDescPtr, srcLengthTensor, coeffTensor, &p,
                                             rppHandle);
            if (st != RPP_SUCCESS)
            {
                lastErr = st;   // e.g. a tile too large for shared memory: not a candidate here
                continue;
            }
            float fastest = -1.f;
            for (int i = 0; i < r; ++i)
            {
                check_cuda(cudaEventRecord(e0, h.stream()), "cudaEventRecord");
                st = rppb_frontend_gpu(srcPtr, srcDescPtr, dstPtr, dstDescPtr, srcLengthTensor, coeffTensor, &p,
                                       rppHandle);
                check_cuda(cudaEventRecord(e1, h.stream()), "cudaEventRecord");
                check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
                if (st != RPP_SUCCESS) break;
                float ms = 0.f;
                check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                if (fastest < 0.f || ms < fastest) fastest = ms;
            }
            if (st != RPP_SUCCESS) continue;
            c.ms = fastest;
            if (best.ms < 0.f || fastest < best.ms) best = c;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (best.ms < 0.f) return lastErr != RPP_SUCCESS ? lastErr : RPP_ERROR;
        params->tileFrames = best.tileFrames;
        params->dbFrames = best.dbFrames;
        params->lookahead = best.lookahead;
        params->ctasPerSm = best.ctasPerSm;
        if (bestMs) *bestMs = best.ms;
        std::lock_guard<std::mutex> lk(g_tuneMu);
        g_tuned[key] = best;
        append_file(key, best);
        return RPP_SUCCESS;
    }
    catch (const Error& e)
    {
        record_error(e.what);
        return e.status;
    }
    catch (...)
    {
        record_error("unknown error");
        return RPP_ERROR;
    }
}
