// The checked build's device-side record (common.cuh: RPPB_RD / RPPB_WR).
//
// librppb_checked.so is compiled with -DRPPB_CHECKED and relocatable device code, so the one region
// table and violation record below serve the kernels of every file.  A call's regions are uploaded by a
// one-thread kernel launched on the handle stream before the call's first kernel (and again when the
// call adds regions after that): the kernel parameters carry the table, so a call captured into a CUDA
// graph replays its own table.  The call ends with a second upload that switches checking off (kernels
// launched outside a call, such as the serving thread's, are not checked), then (outside stream
// capture) synchronizes, reads the record and turns a violation into a status code: a stray read into
// RPP_ERROR_OUT_OF_BOUND_SRC_ROI, a stray write into RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH.
//
// In the library (no RPPB_CHECKED) this file only defines rppb_check_shrink_next_tensors, which returns
// RPP_ERROR_NOT_IMPLEMENTED there.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rppb_frontend.h"
#include "common.cuh"
#include "handle.hpp"

#ifdef RPPB_CHECKED
namespace rppb {

struct CheckRegion
{
    unsigned long long lo, hi;   // [lo, hi)
    int writable;
    int pad;
};
constexpr int kCheckRegions = 256;
struct CheckTable
{
    int enabled;
    int count;
    CheckRegion r[kCheckRegions];
};
struct CheckRecord
{
    unsigned long long violations;
    unsigned long long addr, bytes;
    unsigned site;
    int write;
};

__device__ CheckTable g_checkTable;
__device__ CheckRecord g_checkRecord;
__device__ __align__(16) unsigned char g_checkDummy[256];

__device__ static bool check_inside(unsigned long long a, unsigned long long e, bool write)
{
    const int n = g_checkTable.count;
    for (int i = 0; i < n; ++i)
    {
        const CheckRegion& r = g_checkTable.r[i];
        if (a >= r.lo && e <= r.hi && (r.writable || !write)) return true;
    }
    return false;
}

__device__ static void check_record(unsigned long long a, unsigned long long bytes, bool write, unsigned site)
{
    if (atomicAdd(&g_checkRecord.violations, 1ull) == 0ull)
    {
        g_checkRecord.addr = a;
        g_checkRecord.bytes = bytes;
        g_checkRecord.site = site;
        g_checkRecord.write = write ? 1 : 0;
    }
}

__device__ void* check_addr(const void* p, unsigned bytes, bool write, unsigned site)
{
    if (!g_checkTable.enabled || !__isGlobal(p)) return const_cast<void*>(p);
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    if (check_inside(a, a + bytes, write)) return const_cast<void*>(p);
    check_record(a, bytes, write, site);
    return g_checkDummy;
}

__device__ bool check_range(const void* p, unsigned long long bytes, bool write, unsigned site)
{
    if (!g_checkTable.enabled || bytes == 0 || !__isGlobal(p)) return true;
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    if (check_inside(a, a + bytes, write)) return true;
    check_record(a, bytes, write, site);
    return false;
}

namespace {

__global__ void check_table_kernel(CheckTable t) { g_checkTable = t; }

// The checked sources, for naming a violation's file from its site (common.cuh: RPPB_SITE).
const char* const kCheckFiles[] = {"common.cuh", "preemph.cu", "downmix.cu", "downmix.cuh", "resample.cu",
                                   "spectrogram.cu", "stft.cuh", "fft.cuh", "mel.cu", "mel_tables.cuh",
                                   "to_decibels.cu", "nsr.cu", "fused.cu", "fused_queue.cuh", "fused_tc.cu",
                                   "tc_dft.cu", "tcgen05.cuh", "host_io.cu", "server.cu", "slice.cu",
                                   "normalize.cu", "normalize_nd.cu", "pcm.cu", "autotune.cu", "check.cu"};

std::string site_name(unsigned site)
{
    const unsigned h = site >> 16;
    for (const char* f : kCheckFiles)
        if (check_file_hash(f) == h) return std::string(f) + ":" + std::to_string(site & 0xffffu);
    return "file " + std::to_string(h) + ":" + std::to_string(site & 0xffffu);
}

unsigned long long g_shrink[2] = {0, 0};   // rppb_check_shrink_next_tensors: source, destination

}  // namespace

std::recursive_mutex& check_mutex()
{
    static std::recursive_mutex m;
    return m;
}

unsigned long long check_take_shrink(bool destination)
{
    const unsigned long long s = g_shrink[destination ? 1 : 0];
    g_shrink[destination ? 1 : 0] = 0;
    return s;
}

void check_upload(cudaStream_t s, bool enabled, std::vector<CheckSpan> spans)
{
    std::vector<CheckSpan> keep;
    for (const CheckSpan& x : spans)
        if (x.p && x.bytes) keep.push_back(x);
    std::sort(keep.begin(), keep.end(), [](const CheckSpan& a, const CheckSpan& b) {
        return a.writable != b.writable ? a.writable < b.writable
                                        : reinterpret_cast<uintptr_t>(a.p) < reinterpret_cast<uintptr_t>(b.p);
    });
    std::vector<CheckRegion> rs;
    for (const CheckSpan& x : keep)
    {
        const unsigned long long lo = reinterpret_cast<uintptr_t>(x.p), hi = lo + x.bytes;
        if (!rs.empty() && rs.back().writable == int(x.writable) && lo <= rs.back().hi)   // overlapping or adjacent
            rs.back().hi = std::max(rs.back().hi, hi);
        else
            rs.push_back(CheckRegion{lo, hi, int(x.writable), 0});
    }
    // more regions than the table holds (a clip table of many separate buffers): merge the two neighbours
    // of equal access with the smallest gap until they fit, so the checks only widen
    while (rs.size() > size_t(kCheckRegions))
    {
        size_t best = rs.size();
        unsigned long long gap = ~0ull;
        for (size_t i = 0; i + 1 < rs.size(); ++i)
            if (rs[i].writable == rs[i + 1].writable && rs[i + 1].lo - rs[i].hi < gap)
            {
                gap = rs[i + 1].lo - rs[i].hi;
                best = i;
            }
        if (best == rs.size()) fail(RPP_ERROR, "checked build: more device regions than the table holds");
        rs[best].hi = std::max(rs[best].hi, rs[best + 1].hi);
        rs.erase(rs.begin() + best + 1);
    }
    CheckTable t{};
    t.enabled = enabled ? 1 : 0;
    t.count = int(rs.size());
    std::copy(rs.begin(), rs.end(), t.r);
    check_table_kernel<<<1, 1, 0, s>>>(t);
    check_cuda(cudaGetLastError(), "check_table_kernel");
}

RppStatus check_collect(RppStatus st)
{
    CheckRecord rec{};
    check_cuda(cudaMemcpyFromSymbol(&rec, g_checkRecord, sizeof rec), "cudaMemcpyFromSymbol(check record)");
    if (rec.violations == 0) return st;
    const CheckRecord zero{};
    check_cuda(cudaMemcpyToSymbol(g_checkRecord, &zero, sizeof zero), "cudaMemcpyToSymbol(check record)");
    char buf[96];
    std::snprintf(buf, sizeof buf, "%llu bytes at 0x%llx", rec.bytes, rec.addr);
    record_error(std::string("checked build: ") + (rec.write ? "write of " : "read of ") + buf +
                 " outside the call's regions at " + site_name(rec.site) + " (" + std::to_string(rec.violations) +
                 " accesses)");
    return rec.write ? RPP_ERROR_INSUFFICIENT_DST_BUFFER_LENGTH : RPP_ERROR_OUT_OF_BOUND_SRC_ROI;
}

void check_reset()
{
    const CheckRecord zero{};
    check_cuda(cudaMemcpyToSymbol(g_checkRecord, &zero, sizeof zero), "cudaMemcpyToSymbol(check record)");
}

}  // namespace rppb

extern "C" SHARED_PUBLIC RppStatus rppb_check_shrink_next_tensors(Rpp64u sourceBytes, Rpp64u destinationBytes)
{
    std::lock_guard<std::recursive_mutex> lk(rppb::check_mutex());
    rppb::g_shrink[0] = sourceBytes;
    rppb::g_shrink[1] = destinationBytes;
    return RPP_SUCCESS;
}

#else

extern "C" SHARED_PUBLIC RppStatus rppb_check_shrink_next_tensors(Rpp64u, Rpp64u) { return RPP_ERROR_NOT_IMPLEMENTED; }

#endif
