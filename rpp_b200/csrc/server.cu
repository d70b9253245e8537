// Continuous-batching server of the multi-rate front end (include/rppb_server.h): arena admission,
// upload / compute / download streams, one captured graph per clip table, and a scheduler thread.
//
// Scheduler round (repeated until stopped):
//   finish  - requests whose output copies ended: stamp, free their arena blocks, report;
//   retire  - steps whose graph ended: queue the clips' output copies on the download stream (one copy
//             kernel over every pinned output of the round's steps, a DMA copy per pageable one);
//   admit   - FIFO: allocate every clip's block (input, outRate signal, decibels) or wait; queue the
//             clips' copies on the upload stream (one copy kernel over the round's pinned clips, a DMA
//             copy per pageable one);
//   step    - while a table is free and uploaded clips wait: fill the pinned table, replay its graph.
// The copy kernels read their job lists from pinned rings (a slot is reused once its kernel ended) and
// leave the fused kernel's CTA slots on kServerReserveSms SMs to run beside it.  Steps run either the
// fused front end or, with plainChain, the plain four-call path on a batch buffer (plain_step below).
// All CUDA state lives on the scheduler thread except creation and destruction.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/rppb_server.h"
#include "../../include/rppt_tensor_audio_augmentations.h"
#include "common.cuh"
#include "handle.hpp"
#include "ops.hpp"

namespace rppb {
namespace {

constexpr size_t kAlign = 256;
constexpr int kJobCap = 4096;        // copy jobs per mover launch
constexpr int kJobRing = 8;          // mover job lists in flight per direction
constexpr int kMoverCtas = 32;
constexpr int kServerReserveSms = 8; // SMs left to the movers beside the fused kernel
constexpr int kSeg = 8192;           // floats per work unit of the plain path's copy kernels

// Plain path, step input: clip b of the table (resampled into clips[b].work) -> row b of the batch
// buffer, with the per-sample tensors of the four plain calls (length, coefficient, {bins, frames},
// {frames, numFilter}).  Empty slots get length 0 and no frames.
__global__ void clips_to_batch_kernel(const RppbClip* __restrict__ clips, int n, float outRate, int S, int Fmax,
                                      float* __restrict__ xb, int* __restrict__ len, float* __restrict__ coeff,
                                      float c, int* __restrict__ dims, uint32_t* __restrict__ patches, int bins,
                                      int nf, int W, int hop, bool center)
{
    const int segs = (S + kSeg - 1) / kSeg;
    for (long long u = blockIdx.x; u < (long long)n * segs; u += gridDim.x)
    {
        const int b = int(u / segs), sg = int(u % segs);
        const RppbClip cl = clips[b];
        const int L = cl.length <= 0 ? 0 : min(resampled_length(cl.length, cl.inRate, outRate), S);
        if (sg == 0 && threadIdx.x == 0)
        {
            const int F = L <= 0 ? 0 : max(0, min(num_windows(L, W, hop, center), min(Fmax, cl.dstStride)));
            len[b] = L;
            coeff[b] = c;
            dims[2 * b] = bins;
            dims[2 * b + 1] = F;
            patches[2 * b] = uint32_t(F);
            patches[2 * b + 1] = uint32_t(nf);
        }
        const int i0 = sg * kSeg, i1 = min(L, i0 + kSeg);
        for (int i = i0 + int(threadIdx.x); i < i1; i += blockDim.x) xb[size_t(b) * S + i] = cl.work[i];
    }
}

// Plain path, step output: rows [numFilter][frames] of each clip's decibels -> the clip's dst (row
// stride dstStride), a warp per (clip, row).
__global__ void batch_to_clips_kernel(const float* __restrict__ db, int n, int nf, int Fmax,
                                      const RppbClip* __restrict__ clips, const int* __restrict__ dims)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    for (long long w = blockIdx.x * (long long)(blockDim.x / 32) + (threadIdx.x >> 5); w < (long long)n * nf;
         w += warps)
    {
        const int b = int(w / nf), r = int(w % nf);
        const RppbClip cl = clips[b];
        const int F = dims[2 * b + 1];
        if (cl.dst == nullptr || F <= 0) continue;
        const float* s = db + (size_t(b) * nf + r) * Fmax;
        float* d = cl.dst + size_t(r) * cl.dstStride;
        for (int f = lane; f < F; f += 32) d[f] = s[f];
    }
}

// Device address of a pinned (mapped) host buffer, or null for pageable memory.
const void* mapped_address(const void* p)
{
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess)
    {
        cudaGetLastError();
        return nullptr;
    }
    if (attr.type == cudaMemoryTypeHost) return attr.devicePointer;
    return nullptr;
}

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

long long now_ns()
{
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// First-fit allocator over [0, size) in kAlign units; free ranges keyed by offset.
class Arena
{
  public:
    explicit Arena(size_t size) : size_(size) { free_[0] = size; }
    bool alloc(size_t bytes, size_t* off)
    {
        bytes = align_up(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= bytes)
            {
                *off = it->first;
                const size_t rest = it->second - bytes, o = it->first + bytes;
                free_.erase(it);
                if (rest) free_[o] = rest;
                used_ += bytes;
                return true;
            }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        bytes = align_up(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first)
        {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin())
        {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first)
            {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t used() const { return used_; }
    size_t size() const { return size_; }

  private:
    size_t size_;
    size_t used_ = 0;
    std::map<size_t, size_t> free_;
};

struct Request
{
    uint64_t id;
    long long submitNs;
    std::vector<const float*> src;
    std::vector<int> len;
    std::vector<float> rate;
    std::vector<float*> out;
    std::vector<const float*> srcMapped;          // device address of a pinned clip (null: DMA copy)
    std::vector<float*> outMapped;                // device address of a pinned output (null: DMA copy)
    std::vector<int> lr, frames;                  // outRate length and frames per clip
    std::vector<size_t> off, bytes;               // arena block per clip
    cudaEvent_t uploaded = nullptr, downloaded = nullptr;
    bool uploadDone = false;
    int retired = 0;
};

struct Step
{
    cudaEvent_t done;
    int table;
    std::vector<std::pair<Request*, int>> clips;
};

}  // namespace
}  // namespace rppb

using namespace rppb;

extern "C" const char* rppbGetLastError();

struct RppbServer
{
    RppbServerConfig cfg{};
    int device = 0;
    cudaStream_t compute = nullptr, up = nullptr, down = nullptr;
    rppHandle_t handle = nullptr;
    char* arenaBase = nullptr;
    Arena* arena = nullptr;
    float* lut = nullptr;
    std::vector<RppbClip*> hostTables, devTables;
    std::vector<cudaGraphExec_t> graphs;
    std::vector<cudaEvent_t> tableBusy;
    std::vector<bool> tableUsed;
    std::vector<cudaEvent_t> eventPool;
    // copy-kernel job lists (pinned rings) per direction
    struct JobRing
    {
        std::vector<CopyJob*> lists;
        std::vector<cudaEvent_t> free;
        std::vector<bool> used;
        int next = 0;
        CopyJob* cur = nullptr;
        int slot = -1, count = 0;
        long long units = 0;
    } upRing, downRing;
    // plain path buffers (plainChain)
    int plainS = 0, plainF = 0, plainBins = 0;
    float *xb = nullptr, *pb = nullptr, *spec = nullptr, *mel = nullptr, *db = nullptr, *pcoeff = nullptr;
    int *plen = nullptr, *pdims = nullptr;
    uint32_t* ppatches = nullptr;
    void* rsScratch = nullptr;

    std::mutex mu;
    std::deque<Request*> submitted;
    std::deque<RppbCompletion> completions;
    std::atomic<uint64_t> nextId{1};
    std::atomic<bool> stop{false};
    std::atomic<size_t> arenaUsed{0};
    std::string error;
    RppStatus errorStatus = RPP_SUCCESS;
    std::thread worker;

    // scheduler-thread state
    std::deque<Request*> pending;
    std::deque<std::pair<Request*, int>> ready;
    std::deque<Step> inflight;
    std::vector<Request*> finishing;
    std::vector<Request*> admitted;
    int nextTable = 0;

    int frames_of(int length, float rate, int* lr) const
    {
        const RppbFrontendParams& p = cfg.params;
        const int l = length <= 0 ? 0 : resampled_length(length, rate, cfg.outRate);
        if (lr) *lr = l;
        return std::max(0, num_windows(l, p.windowLength, p.windowStep, p.centerWindows));
    }
    cudaEvent_t take_event()
    {
        if (!eventPool.empty())
        {
            cudaEvent_t e = eventPool.back();
            eventPool.pop_back();
            return e;
        }
        cudaEvent_t e;
        check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate(server)");
        return e;
    }
    void give_event(cudaEvent_t e) { eventPool.push_back(e); }

    // Adds a copy of `count` floats to the ring's current job list (launching the list first when full).
    void add_job(JobRing& ring, cudaStream_t st, const float* src, float* dst, long long count)
    {
        if (count <= 0) return;
        if (ring.cur && ring.count == kJobCap) flush_jobs(ring, st);
        if (!ring.cur)
        {
            const int t = ring.next;
            if (ring.used[t]) check_cuda(cudaEventSynchronize(ring.free[t]), "cudaEventSynchronize(job list)");
            ring.cur = ring.lists[t];
            ring.slot = t;
            ring.count = 0;
            ring.units = 0;
        }
        ring.cur[ring.count++] = CopyJob{src, dst, count, ring.units};
        ring.units += copy_job_segments(count);
    }
    // Launches the ring's current job list on `st` (one kernel for all of its copies).
    void flush_jobs(JobRing& ring, cudaStream_t st)
    {
        if (!ring.cur) return;
        launch_copy_jobs(st, ring.cur, ring.count, ring.units, kMoverCtas);
        check_cuda(cudaEventRecord(ring.free[ring.slot], st), "cudaEventRecord(job list)");
        ring.used[ring.slot] = true;
        ring.next = (ring.slot + 1) % int(ring.lists.size());
        ring.cur = nullptr;
        ring.count = 0;
    }

    bool finish_round()
    {
        bool work = false;
        for (size_t i = 0; i < finishing.size();)
        {
            Request* r = finishing[i];
            const cudaError_t q = cudaEventQuery(r->downloaded);
            if (q == cudaErrorNotReady)
            {
                ++i;
                continue;
            }
            check_cuda(q, "cudaEventQuery(download)");
            const long long t = now_ns();
            for (size_t c = 0; c < r->off.size(); ++c) arena->release(r->off[c], r->bytes[c]);
            arenaUsed = arena->used();
            give_event(r->uploaded);
            give_event(r->downloaded);
            {
                std::lock_guard<std::mutex> lk(mu);
                completions.push_back(RppbCompletion{r->id, r->submitNs, t});
            }
            delete r;
            finishing[i] = finishing.back();
            finishing.pop_back();
            work = true;
        }
        return work;
    }

    bool retire_round()
    {
        bool work = false;
        const int nf = cfg.params.numFilter;
        std::vector<Request*> completing;
        while (!inflight.empty())
        {
            Step& s = inflight.front();
            const cudaError_t q = cudaEventQuery(s.done);
            if (q == cudaErrorNotReady) break;
            check_cuda(q, "cudaEventQuery(step)");
            check_cuda(cudaStreamWaitEvent(down, s.done, 0), "cudaStreamWaitEvent(download)");
            for (auto& [r, i] : s.clips)
            {
                const size_t outOff = r->off[i] + align_up(size_t(r->len[i]) * 4) + align_up(size_t(r->lr[i] + 4) * 4);
                const long long count = (long long)nf * std::max(r->frames[i], 1);
                const float* src = reinterpret_cast<const float*>(arenaBase + outOff);
                if (r->outMapped[i]) add_job(downRing, down, src, r->outMapped[i], count);
                else
                    check_cuda(cudaMemcpyAsync(r->out[i], src, size_t(count) * 4, cudaMemcpyDeviceToHost, down),
                               "cudaMemcpyAsync(output)");
                if (++r->retired == int(r->src.size())) completing.push_back(r);
            }
            give_event(s.done);
            inflight.pop_front();
            work = true;
        }
        flush_jobs(downRing, down);
        for (Request* r : completing)
        {
            check_cuda(cudaEventRecord(r->downloaded, down), "cudaEventRecord(download)");
            finishing.push_back(r);
        }
        return work;
    }

    bool admit_round()
    {
        bool work = false;
        const int nf = cfg.params.numFilter;
        while (!pending.empty())
        {
            Request* r = pending.front();
            const size_t k = r->src.size();
            r->off.assign(k, 0);
            r->bytes.assign(k, 0);
            size_t got = 0;
            for (; got < k; ++got)
            {
                const size_t b = align_up(size_t(r->len[got]) * 4) + align_up(size_t(r->lr[got] + 4) * 4) +
                                 align_up(size_t(nf) * std::max(r->frames[got], 1) * 4);
                if (!arena->alloc(b, &r->off[got])) break;
                r->bytes[got] = b;
            }
            if (got < k)
            {
                for (size_t c = 0; c < got; ++c) arena->release(r->off[c], r->bytes[c]);
                break;   // first come, first served: wait for memory
            }
            arenaUsed = arena->used();
            pending.pop_front();
            for (size_t c = 0; c < k; ++c)
            {
                if (r->len[c] <= 0) continue;
                float* dst = reinterpret_cast<float*>(arenaBase + r->off[c]);
                if (r->srcMapped[c]) add_job(upRing, up, r->srcMapped[c], dst, r->len[c]);
                else
                    check_cuda(cudaMemcpyAsync(dst, r->src[c], size_t(r->len[c]) * 4, cudaMemcpyHostToDevice, up),
                               "cudaMemcpyAsync(clip)");
            }
            admitted.push_back(r);
            work = true;
        }
        // one copy kernel for the round's pinned clips, then each request's upload event after it
        flush_jobs(upRing, up);
        for (Request* r : admitted)
        {
            r->uploaded = take_event();
            r->downloaded = take_event();
            check_cuda(cudaEventRecord(r->uploaded, up), "cudaEventRecord(upload)");
            for (size_t c = 0; c < r->src.size(); ++c) ready.emplace_back(r, int(c));
        }
        admitted.clear();
        return work;
    }

    bool step_round()
    {
        bool work = false;
        while (!ready.empty())
        {
            const int t = nextTable;
            if (tableUsed[t])
            {
                const cudaError_t q = cudaEventQuery(tableBusy[t]);
                if (q == cudaErrorNotReady) break;
                check_cuda(q, "cudaEventQuery(table)");
            }
            Step s;
            s.table = t;
            while (!ready.empty() && int(s.clips.size()) < cfg.maxClipsPerStep)
            {
                Request* r = ready.front().first;
                if (!r->uploadDone)
                {
                    const cudaError_t q = cudaEventQuery(r->uploaded);
                    if (q == cudaErrorNotReady) break;
                    check_cuda(q, "cudaEventQuery(upload)");
                    r->uploadDone = true;
                }
                s.clips.push_back(ready.front());
                ready.pop_front();
            }
            if (s.clips.empty()) break;
            RppbClip* tab = hostTables[t];
            std::memset(tab, 0, sizeof(RppbClip) * cfg.maxClipsPerStep);
            for (size_t e = 0; e < s.clips.size(); ++e)
            {
                Request* r = s.clips[e].first;
                const int i = s.clips[e].second;
                char* a0 = arenaBase + r->off[i];
                char* a1 = a0 + align_up(size_t(r->len[i]) * 4);
                char* a2 = a1 + align_up(size_t(r->lr[i] + 4) * 4);
                tab[e].src = reinterpret_cast<const float*>(a0);
                tab[e].work = reinterpret_cast<float*>(a1);
                tab[e].dst = reinterpret_cast<float*>(a2);
                tab[e].length = r->len[i];
                tab[e].inRate = r->rate[i];
                tab[e].dstStride = std::max(r->frames[i], 1);
            }
            check_cuda(cudaGraphLaunch(graphs[t], compute), "cudaGraphLaunch(step)");
            check_cuda(cudaEventRecord(tableBusy[t], compute), "cudaEventRecord(table)");
            tableUsed[t] = true;
            s.done = take_event();
            check_cuda(cudaEventRecord(s.done, compute), "cudaEventRecord(step)");
            inflight.push_back(std::move(s));
            nextTable = (t + 1) % int(graphs.size());
            work = true;
        }
        return work;
    }

    static RpptDesc desc(int n, int h, int w, int numDims)
    {
        RpptDesc d{};
        d.numDims = numDims;
        d.offsetInBytes = 0;
        d.dataType = F32;
        d.n = Rpp32u(n);
        d.c = 1;
        d.h = Rpp32u(h);
        d.w = Rpp32u(w);
        d.strides.nStride = Rpp32u(h) * Rpp32u(w);
        d.strides.hStride = Rpp32u(w);
        d.strides.wStride = 1;
        d.strides.cStride = 1;
        d.layout = NFT;
        return d;
    }

    // The plain FP32 path of one step on the compute stream: resample the table's clips, copy them into
    // the batch buffer, the four plain calls (pre-emphasis, spectrogram, mel filter bank, decibels) on it,
    // then copy each clip's decibels to its output block.  Captured once per table.
    void plain_step(const RppbClip* table)
    {
        Handle& h = deref(handle);
        const RppbFrontendParams& p = cfg.params;
        const int n = cfg.maxClipsPerStep, nf = p.numFilter;
        ResampleWindowDev win;
        win.lut = lut;
        win.lutSize = cfg.lookupSize;
        win.scale = cfg.scale;
        win.center = cfg.center;
        win.lobes = cfg.lobes;
        launch_resample_clips(h, rsScratch, table, n, cfg.outRate, win);
        const int grid = 2 * h.num_sms();
        clips_to_batch_kernel<<<grid, 256, 0, compute>>>(table, n, cfg.outRate, plainS, plainF, xb, plen, pcoeff,
                                                         cfg.preemphCoeff, pdims, ppatches, plainBins, nf,
                                                         p.windowLength, p.windowStep, p.centerWindows);
        count_launch(1);
        check_cuda(cudaGetLastError(), "clips_to_batch_kernel");
        RpptDesc sd = desc(n, 1, plainS, 2), spd = desc(n, plainBins, plainF, 3), md = desc(n, nf, plainF, 3);
        auto ok = [](RppStatus st, const char* what) {
            if (st != RPP_SUCCESS) fail(st, std::string(what) + ": " + rppbGetLastError());
        };
        ok(rppt_pre_emphasis_filter_gpu(xb, &sd, pb, &sd, plen, pcoeff, p.borderType, handle), "pre_emphasis");
        ok(rppt_spectrogram_gpu(pb, &sd, spec, &spd, plen, p.centerWindows, p.reflectPadding, nullptr,
                                p.nfft ? p.nfft : p.windowLength, p.power, p.windowLength, p.windowStep, handle),
           "spectrogram");
        ok(rppt_mel_filter_bank_gpu(spec, &spd, mel, &md, pdims, p.maxFreq, p.minFreq, p.melFormula, nf, p.sampleRate,
                                    p.normalize, handle),
           "mel_filter_bank");
        ok(rppt_to_decibels_gpu(mel, &md, db, &md, reinterpret_cast<RpptImagePatch*>(ppatches), p.cutOffDB,
                                p.multiplier, p.referenceMagnitude, handle),
           "to_decibels");
        batch_to_clips_kernel<<<grid, 256, 0, compute>>>(db, n, nf, plainF, table, pdims);
        count_launch(1);
        check_cuda(cudaGetLastError(), "batch_to_clips_kernel");
    }

    void run()
    {
        cudaSetDevice(device);
        try
        {
            while (true)
            {
                bool work = false;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    while (!submitted.empty())
                    {
                        pending.push_back(submitted.front());
                        submitted.pop_front();
                        work = true;
                    }
                }
                work |= finish_round();
                work |= retire_round();
                work |= admit_round();
                work |= step_round();
                if (!work)
                {
                    if (stop && pending.empty() && ready.empty() && inflight.empty() && finishing.empty()) break;
                    std::this_thread::yield();
                }
            }
        }
        catch (const Error& e)
        {
            std::lock_guard<std::mutex> lk(mu);
            error = e.what;
            errorStatus = e.status;
        }
    }
};

namespace {

RppStatus server_guard(const std::function<RppStatus()>& body)
{
    try
    {
        return body();
    }
    catch (const Error& e)
    {
        record_error(e.what);
        return e.status;
    }
    catch (const std::bad_alloc&)
    {
        record_error("host allocation failed");
        return RPP_ERROR_NOT_ENOUGH_MEMORY;
    }
    catch (...)
    {
        record_error("unknown error");
        return RPP_ERROR;
    }
}

void release(RppbServer* s)
{
    if (s->worker.joinable())
    {
        s->stop = true;
        s->worker.join();
    }
    for (cudaStream_t st : {s->compute, s->up, s->down})
        if (st) cudaStreamSynchronize(st);
    for (auto g : s->graphs)
        if (g) cudaGraphExecDestroy(g);
    for (auto e : s->tableBusy)
        if (e) cudaEventDestroy(e);
    for (auto e : s->eventPool) cudaEventDestroy(e);
    for (auto p : s->hostTables)
        if (p) cudaFreeHost(p);
    for (auto* ring : {&s->upRing, &s->downRing})
    {
        for (auto p : ring->lists)
            if (p) cudaFreeHost(p);
        for (auto e : ring->free)
            if (e) cudaEventDestroy(e);
    }
    for (void* p : {static_cast<void*>(s->xb), static_cast<void*>(s->pb), static_cast<void*>(s->spec),
                    static_cast<void*>(s->mel), static_cast<void*>(s->db), static_cast<void*>(s->pcoeff),
                    static_cast<void*>(s->plen), static_cast<void*>(s->pdims), static_cast<void*>(s->ppatches),
                    s->rsScratch})
        if (p) cudaFree(p);
    for (auto p : s->devTables)
        if (p) cudaFree(p);
    if (s->handle) rppDestroy(s->handle, RPP_HIP_BACKEND);
    if (s->lut) cudaFree(s->lut);
    if (s->arenaBase) cudaFree(s->arenaBase);
    delete s->arena;
    for (cudaStream_t st : {s->compute, s->up, s->down})
        if (st) cudaStreamDestroy(st);
    delete s;
}

}  // namespace

extern "C" SHARED_PUBLIC RppStatus rppb_server_create(rppbServer_t* server, const RppbServerConfig* config)
{
    RppbServer* s = nullptr;
    const RppStatus st = server_guard([&]() -> RppStatus {
        if (!server || !config) fail(RPP_ERROR_INVALID_ARGUMENTS, "null server or config");
        const RppbServerConfig& c = *config;
        if (c.maxClipsPerStep <= 0 || c.tables <= 0 || c.budgetBytes == 0 || !(c.outRate > 0.f))
            fail(RPP_ERROR_INVALID_ARGUMENTS, "invalid server configuration");
        if (!c.lookup || c.lookupSize < 2 || c.lobes < 0) fail(RPP_ERROR_INVALID_ARGUMENTS, "invalid resampling window");
        if (c.params.windowFunction) fail(RPP_ERROR_NOT_IMPLEMENTED, "the server uses the Hann window");
        s = new RppbServer();
        s->cfg = c;
        check_cuda(cudaGetDevice(&s->device), "cudaGetDevice");
        check_cuda(cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking), "cudaStreamCreate");
        void* base = nullptr;
        check_cuda(cudaMalloc(&base, c.budgetBytes), "cudaMalloc(arena)");
        s->arenaBase = static_cast<char*>(base);
        s->arena = new Arena(c.budgetBytes);
        check_cuda(cudaMalloc(&s->lut, size_t(c.lookupSize) * 4), "cudaMalloc(lut)");
        check_cuda(cudaMemcpy(s->lut, c.lookup, size_t(c.lookupSize) * 4, cudaMemcpyHostToDevice), "cudaMemcpy(lut)");
        if (rppCreate(&s->handle, size_t(c.maxClipsPerStep), 0, s->compute, RPP_HIP_BACKEND) != rppStatusSuccess)
            fail(RPP_ERROR, "rppCreate failed");
        for (auto* ring : {&s->upRing, &s->downRing})
            for (int t = 0; t < kJobRing; ++t)
            {
                void* hp = nullptr;
                check_cuda(cudaMallocHost(&hp, sizeof(CopyJob) * kJobCap), "cudaMallocHost(job list)");
                ring->lists.push_back(static_cast<CopyJob*>(hp));
                cudaEvent_t e;
                check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
                ring->free.push_back(e);
                ring->used.push_back(false);
            }
        if (c.plainChain)
        {
            const RppbFrontendParams& p = c.params;
            const int n = c.maxClipsPerStep, nf = p.numFilter;
            const int nfft = p.nfft ? p.nfft : p.windowLength;
            s->plainS = ((c.maxSamples > 0 ? c.maxSamples : int(30.0f * c.outRate) + 8) + 3) & ~3;
            s->plainF = std::max(1, num_windows(s->plainS, p.windowLength, p.windowStep, p.centerWindows));
            s->plainBins = nfft / 2 + 1;
            auto dalloc = [](auto*& ptr, size_t bytes) {
                void* q = nullptr;
                check_cuda(cudaMalloc(&q, bytes), "cudaMalloc(plain path)");
                ptr = static_cast<std::remove_reference_t<decltype(ptr)>>(q);
            };
            const size_t sig = size_t(n) * s->plainS * 4;
            dalloc(s->xb, sig);
            dalloc(s->pb, sig);
            dalloc(s->spec, size_t(n) * s->plainBins * s->plainF * 4);
            dalloc(s->mel, size_t(n) * nf * s->plainF * 4);
            dalloc(s->db, size_t(n) * nf * s->plainF * 4);
            dalloc(s->pcoeff, size_t(n) * 4);
            dalloc(s->plen, size_t(n) * 4);
            dalloc(s->pdims, size_t(n) * 8);
            dalloc(s->ppatches, size_t(n) * 8);
            dalloc(s->rsScratch, size_t(n + 1) * 8 + 4096);
        }
        const size_t tableBytes = sizeof(RppbClip) * c.maxClipsPerStep;
        for (int t = 0; t < c.tables; ++t)
        {
            void* hp = nullptr;
            void* dp = nullptr;
            check_cuda(cudaMallocHost(&hp, tableBytes), "cudaMallocHost(table)");
            s->hostTables.push_back(static_cast<RppbClip*>(hp));
            std::memset(hp, 0, tableBytes);
            check_cuda(cudaMalloc(&dp, tableBytes), "cudaMalloc(table)");
            s->devTables.push_back(static_cast<RppbClip*>(dp));
            check_cuda(cudaMemsetAsync(dp, 0, tableBytes, s->compute), "cudaMemset(table)");
            cudaEvent_t e;
            check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            s->tableBusy.push_back(e);
            s->tableUsed.push_back(false);
        }
        auto call = [&](int t) {
            if (c.plainChain)
            {
                s->plain_step(s->devTables[t]);
                return;
            }
            frontend_clips(deref(s->handle), s->devTables[t], c.maxClipsPerStep, c.outRate, s->lut, c.lookupSize,
                           c.scale, c.center, c.lobes, c.preemphCoeff, &s->cfg.params, kServerReserveSms);
        };
        // one uncaptured call (empty table) sizes the handle workspace and builds the cached tables
        call(0);
        check_cuda(cudaStreamSynchronize(s->compute), "cudaStreamSynchronize");
        for (int t = 0; t < c.tables; ++t)
        {
            cudaGraph_t g;
            check_cuda(cudaStreamBeginCapture(s->compute, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            check_cuda(cudaMemcpyAsync(s->devTables[t], s->hostTables[t], tableBytes, cudaMemcpyHostToDevice,
                                       s->compute),
                       "cudaMemcpyAsync(table)");
            call(t);
            check_cuda(cudaStreamEndCapture(s->compute, &g), "cudaStreamEndCapture");
            cudaGraphExec_t ex;
            const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            check_cuda(ie, "cudaGraphInstantiate");
            s->graphs.push_back(ex);
        }
        s->worker = std::thread([s] { s->run(); });
        *server = s;
        return RPP_SUCCESS;
    });
    if (st != RPP_SUCCESS && s) release(s);
    return st;
}

extern "C" SHARED_PUBLIC RppStatus rppb_server_destroy(rppbServer_t server)
{
    return server_guard([&]() -> RppStatus {
        if (!server) fail(RPP_ERROR_INVALID_ARGUMENTS, "null server");
        release(server);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC Rpp32s rppb_server_frames(rppbServer_t server, Rpp32s length, Rpp32f rate)
{
    return server ? server->frames_of(length, rate, nullptr) : -1;
}

extern "C" SHARED_PUBLIC RppStatus rppb_server_submit(rppbServer_t server, const Rpp32f* const* clips,
                                                      const Rpp32s* lengths, const Rpp32f* rates,
                                                      Rpp32f* const* outputs, Rpp32s numClips, Rpp64u* requestId)
{
    return server_guard([&]() -> RppStatus {
        if (!server || !clips || !lengths || !rates || !outputs || numClips <= 0)
            fail(RPP_ERROR_INVALID_ARGUMENTS, "invalid request");
        {
            std::lock_guard<std::mutex> lk(server->mu);
            if (server->errorStatus != RPP_SUCCESS) fail(server->errorStatus, "server stopped: " + server->error);
        }
        auto* r = new Request();
        r->submitNs = now_ns();
        const int nf = server->cfg.params.numFilter;
        size_t total = 0;
        for (int i = 0; i < numClips; ++i)
        {
            if (!(rates[i] > 0.f) || lengths[i] < 0 || (lengths[i] > 0 && !clips[i]) || !outputs[i])
            {
                delete r;
                fail(RPP_ERROR_INVALID_ARGUMENTS, "invalid clip");
            }
            int lr = 0;
            const int f = server->frames_of(lengths[i], rates[i], &lr);
            if (server->cfg.plainChain && lr > server->plainS)
            {
                delete r;
                fail(RPP_ERROR_NOT_ENOUGH_MEMORY, "clip longer than the plain path's maxSamples");
            }
            r->srcMapped.push_back(lengths[i] > 0 ? static_cast<const float*>(mapped_address(clips[i])) : nullptr);
            r->outMapped.push_back(const_cast<float*>(static_cast<const float*>(mapped_address(outputs[i]))));
            r->src.push_back(clips[i]);
            r->len.push_back(lengths[i]);
            r->rate.push_back(rates[i]);
            r->out.push_back(outputs[i]);
            r->lr.push_back(lr);
            r->frames.push_back(f);
            total += align_up(size_t(lengths[i]) * 4) + align_up(size_t(lr + 4) * 4) +
                     align_up(size_t(nf) * std::max(f, 1) * 4);
        }
        if (total > server->arena->size())
        {
            delete r;
            fail(RPP_ERROR_NOT_ENOUGH_MEMORY, "request larger than the server's device budget");
        }
        r->id = server->nextId++;
        if (requestId) *requestId = r->id;
        std::lock_guard<std::mutex> lk(server->mu);
        server->submitted.push_back(r);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC RppStatus rppb_server_poll(rppbServer_t server, RppbCompletion* done, Rpp32s capacity,
                                                    Rpp32s* count)
{
    return server_guard([&]() -> RppStatus {
        if (!server || !count || (capacity > 0 && !done)) fail(RPP_ERROR_INVALID_ARGUMENTS, "invalid poll");
        std::lock_guard<std::mutex> lk(server->mu);
        int k = 0;
        while (k < capacity && !server->completions.empty())
        {
            done[k++] = server->completions.front();
            server->completions.pop_front();
        }
        *count = k;
        if (server->errorStatus != RPP_SUCCESS) fail(server->errorStatus, "server stopped: " + server->error);
        return RPP_SUCCESS;
    });
}

extern "C" SHARED_PUBLIC Rpp64u rppb_server_arena_used(rppbServer_t server)
{
    return server ? Rpp64u(server->arenaUsed.load()) : 0;
}
