// Continuous-batching server of the multi-rate front end (include/rppb_server.h): arena admission,
// upload / compute / download streams, one captured graph per clip table, and a scheduler thread.
//
// Scheduler round (repeated until stopped):
//   finish  - requests whose output copies ended: stamp, free their arena blocks, report;
//   retire  - steps whose graph ended: queue each clip's output copy on the download stream;
//   admit   - FIFO: allocate every clip's block (input, outRate signal, decibels) or wait;
//             queue the clip copies on the upload stream;
//   step    - while a table is free and uploaded clips wait: fill the pinned table, replay its graph.
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
#include <vector>

#include "../../include/rppb_server.h"
#include "common.cuh"
#include "handle.hpp"

namespace rppb {
namespace {

constexpr size_t kAlign = 256;

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
                check_cuda(cudaMemcpyAsync(r->out[i], arenaBase + outOff, size_t(nf) * std::max(r->frames[i], 1) * 4,
                                           cudaMemcpyDeviceToHost, down),
                           "cudaMemcpyAsync(output)");
                if (++r->retired == int(r->src.size()))
                {
                    check_cuda(cudaEventRecord(r->downloaded, down), "cudaEventRecord(download)");
                    finishing.push_back(r);
                }
            }
            give_event(s.done);
            inflight.pop_front();
            work = true;
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
                if (r->len[c] > 0)
                    check_cuda(cudaMemcpyAsync(arenaBase + r->off[c], r->src[c], size_t(r->len[c]) * 4,
                                               cudaMemcpyHostToDevice, up),
                               "cudaMemcpyAsync(clip)");
            r->uploaded = take_event();
            r->downloaded = take_event();
            check_cuda(cudaEventRecord(r->uploaded, up), "cudaEventRecord(upload)");
            for (size_t c = 0; c < k; ++c) ready.emplace_back(r, int(c));
            work = true;
        }
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
            const RppStatus r = rppb_frontend_clips_gpu(s->devTables[t], c.maxClipsPerStep, c.outRate, s->lut,
                                                        c.lookupSize, c.scale, c.center, c.lobes, c.preemphCoeff,
                                                        &s->cfg.params, s->handle);
            if (r != RPP_SUCCESS) fail(r, std::string("rppb_frontend_clips_gpu: ") + rppbGetLastError());
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
