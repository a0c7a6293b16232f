// pipeline.cu -- one `ff_sieve <sumStart> <sumLimit>` run as a library call (ffb_run):
// the prime map sieved on the device (the reference's, extended to every value the search
// probes), every sum of ff_seg's schedule searched
// on the device, the packed records copied back once, and the text emitted on the host
// in ff_seg's order (reference/segmentedSieve.C:829-925).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ffb200.h"
#include "ffb_internal.h"
#include "../host/plan.h"

struct FfbContext {
    int dev = 0;
    cudaStream_t stream = nullptr;
    uint8_t* d_map = nullptr;
    uint64_t map_cap = 0;
    uint64_t* d_rec = nullptr;
    uint64_t rec_cap = 0;
    uint64_t* h_rec = nullptr;  // pinned
    uint64_t hrec_cap = 0;
    uint64_t map_budget = 0;    // cap on the map's bytes (0: the device's free memory)
};

namespace ffb {
namespace {

int grow(FfbContext* c, uint64_t map_bytes, uint64_t nrec)
{
    map_bytes = (map_bytes + 255) & ~255ull;
    if (map_bytes > c->map_cap) {
        if (c->d_map) cudaFree(c->d_map);
        c->d_map = nullptr;
        c->map_cap = 0;
        FFB_CUDA(cudaMalloc(&c->d_map, map_bytes));
        c->map_cap = map_bytes;
    }
    if (nrec > c->rec_cap) {
        if (c->d_rec) cudaFree(c->d_rec);
        c->d_rec = nullptr;
        c->rec_cap = 0;
        FFB_CUDA(cudaMalloc(&c->d_rec, 8 * nrec));
        c->rec_cap = nrec;
    }
    if (nrec > c->hrec_cap) {
        if (c->h_rec) cudaFreeHost(c->h_rec);
        c->h_rec = nullptr;
        c->hrec_cap = 0;
        FFB_CUDA(cudaMallocHost(&c->h_rec, 8 * nrec));
        c->hrec_cap = nrec;
    }
    return 0;
}

// The map bound of a job: `want` (every value the job may probe) when that map fits the
// device-memory budget (the reference's computeBudget on the free memory, source/budget.cpp:
// 15-42, less the job's records), else the largest map that fits; the search answers the
// probes above it by Miller-Rabin, which is exact, so the output is the same either way
// (the reference likewise caps its own map, reference/segmentedSieve.C:148-176). 0: no room.
uint64_t fit_map_mpv(FfbContext* c, uint64_t want, uint64_t nrec)
{
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(c->dev) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
    }
    // Memory grow() can reuse: the map buffer (freed when the new map is larger; a map that
    // fits in it needs nothing new) and the record buffer only when the job's records do not
    // fit in it (grow() keeps it otherwise, and then the records need nothing new).
    const bool rec_grows = nrec > c->rec_cap;
    const uint64_t own = c->map_cap + (rec_grows ? 8 * c->rec_cap : 0);
    FfbBudget b{};
    ffb_compute_budget(free_b + own, 0.90, 0, 0, 0, &b);
    const uint64_t rec_need = rec_grows ? 16 * nrec : 0;
    uint64_t avail = b.backing > rec_need ? b.backing - rec_need : 0;
    if (c->map_budget && c->map_budget < avail) avail = c->map_budget;
    const uint64_t want_bytes = (want + 1 + 15) >> 4;
    if (want_bytes + 256 <= avail) return want;
    const uint64_t bytes = (avail > 256 ? avail - 256 : 0) & ~255ull;
    return bytes >= 4096 ? bytes * 16 - 1 : 0;
}

// Text of the solution lines of the schedule, numbered from 1 in emission order.
// Ranges are formatted in parallel after a prefix count of their solutions.
std::string emit(const std::vector<Range>& ranges, const uint64_t* rec, uint32_t lo)
{
    const size_t nr = ranges.size();
    std::vector<uint32_t> cnt(nr, 0), first(nr, 0);
    for (size_t r = 0; r < nr; ++r)
        for (uint32_t s = ranges[r].first | 1u; s <= ranges[r].last; s += 2)
            cnt[r] += rec[(s - lo) >> 1] != 0;
    uint32_t total = 0;
    for (size_t r = 0; r < nr; ++r) {
        first[r] = total;
        total += cnt[r];
    }
    std::vector<std::string> parts(nr);
    auto work = [&](size_t r) {
        std::string& out = parts[r];
        out.resize((size_t)cnt[r] * kMaxLine);
        char* p = &out[0];
        uint32_t count = first[r];
        for (uint32_t s = ranges[r].first | 1u; s <= ranges[r].last; s += 2) {
            const uint64_t v = rec[(s - lo) >> 1];
            if (!v) continue;
            p = format_line(p, ++count, s, rec_low(v), rec_high(v), rec_low_prime(v),
                            rec_high_prime(v));
        }
        out.resize((size_t)(p - &out[0]));
    };
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt, 16u));
    if (total < 4096) nt = 1;
    if (nt == 1) {
        for (size_t r = 0; r < nr; ++r) work(r);
    } else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (size_t r = t; r < nr; r += nt) work(r);
            });
        for (auto& t : th) t.join();
    }
    size_t bytes = 0;
    for (auto& s : parts) bytes += s.size();
    std::string all;
    all.reserve(bytes);
    for (auto& s : parts) all += s;
    return all;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" FfbContext* ffb_context_create(int deviceIndex)
{
    if (!device_state(deviceIndex)) return nullptr;
    FfbContext* c = new FfbContext;
    c->dev = deviceIndex;
    if (cudaSetDevice(deviceIndex) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return nullptr;
    }
    return c;
}

extern "C" void ffb_context_destroy(FfbContext* c)
{
    if (!c) return;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->d_map) cudaFree(c->d_map);
    if (c->d_rec) cudaFree(c->d_rec);
    if (c->h_rec) cudaFreeHost(c->h_rec);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int ffb_context_set_map_budget(FfbContext* ctx, uint64_t bytes)
{
    if (!ctx) return -1;
    ctx->map_budget = bytes;
    return 0;
}

extern "C" void ffb_free(void* p) { std::free(p); }

extern "C" int ffb_run(FfbContext* ctx, int nargs, int32_t a1, int32_t a2, char** text, size_t* len)
{
    using clk = std::chrono::steady_clock;
    *text = nullptr;
    *len = 0;
    uint32_t start, limit;
    parse_args(nargs, a1, a2, &start, &limit);
    char hdr[2048];
    Geometry g;
    const int hn = plan_geometry(start, limit, &g, hdr, sizeof hdr);
    if (hn < 0) {
        std::fprintf(stderr, "ffb_run: %s", g.too_big ? hdr : "header overflow\n");
        return -1;
    }
    std::vector<Range> ranges;
    if (!plan_schedule(start, limit, g.mpv, kThreads, ranges)) {
        std::fprintf(stderr, "ffb_run: range [%u, %u] outside what the reference can run\n", start,
                     limit);
        return -1;
    }
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    for (const Range& r : ranges) {
        const uint32_t f = r.first | 1u;
        if (f > r.last) continue;
        lo = std::min(lo, f);
        hi = std::max(hi, r.last - !(r.last & 1));
    }
    if (hi > kMaxSum) {
        std::fprintf(stderr, "ffb_run: sums above 2^25 are outside the exact domain\n");
        return -1;
    }
    // The device map: the reference's (values up to mpv) or, when larger, one covering every
    // value the search probes, so that no probe falls back to Miller-Rabin, as far as device
    // memory allows (fit_map_mpv). IsPrime is exact either way, so the output does not
    // depend on this choice.
    uint64_t want = g.mpv;
    if (lo <= hi) want = std::max(want, ffb_probe_bound(hi));
    FfbContext* c = ctx ? ctx : ffb_context_create(0);
    if (!c) return -1;
    const uint64_t nrec = lo <= hi ? ((uint64_t)hi - lo) / 2 + 1 : 1;
    const uint64_t map_mpv = fit_map_mpv(c, want, nrec);
    const uint64_t map_bytes = (map_mpv + 1 + 15) >> 4;
    int rc = 0;
    std::string body;
    double prime_us = 0, freud_us = 0;
    do {
        if (!map_mpv) {
            std::fprintf(stderr, "ffb_run: no device memory left for a prime map\n");
            rc = -1;
            break;
        }
        if ((rc = grow(c, map_bytes, nrec))) break;
        cudaSetDevice(c->dev);
        const auto t0 = clk::now();
        if ((rc = ffb_sieve_map_async(c->dev, map_mpv, c->d_map, c->stream))) break;
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) { rc = -1; break; }
        const auto t1 = clk::now();
        if (lo <= hi) {
            if ((rc = ffb_search_async(c->dev, c->d_map, map_mpv, lo, hi, c->d_rec, c->stream))) break;
            if (cudaMemcpyAsync(c->h_rec, c->d_rec, 8 * nrec, cudaMemcpyDeviceToHost, c->stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess) {
                rc = -1;
                break;
            }
            uint32_t flags = 0;
            if ((rc = ffb_take_errors(c->dev, &flags))) break;
            if (flags) {
                std::fprintf(stderr, "ffb_run: device error flags 0x%x\n", flags);
                rc = -1;
                break;
            }
            body = emit(ranges, c->h_rec, lo);
        }
        const auto t2 = clk::now();
        prime_us = std::chrono::duration<double, std::micro>(t1 - t0).count();
        freud_us = std::chrono::duration<double, std::micro>(t2 - t1).count();
    } while (0);
    if (!ctx) ffb_context_destroy(c);
    if (rc) {
        std::fprintf(stderr, "ffb_run: failed: %s\n", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    char tail[160];
    const int tn = std::snprintf(tail, sizeof tail, "Prime time: %llu \xce\xbcs\nFreudenthal time: %llu \xce\xbcs\n",
                                 (unsigned long long)prime_us, (unsigned long long)freud_us);
    const size_t n = (size_t)hn + body.size() + (size_t)tn;
    char* out = (char*)std::malloc(n + 1);
    if (!out) return -1;
    std::memcpy(out, hdr, (size_t)hn);
    std::memcpy(out + hn, body.data(), body.size());
    std::memcpy(out + hn + body.size(), tail, (size_t)tn);
    out[n] = 0;
    *text = out;
    *len = n;
    return 0;
}

extern "C" int ffb_emit(int nargs, int32_t a1, int32_t a2, const uint64_t* h_rec, uint32_t recLo,
                        uint64_t nrec, double primeUs, double freudUs, char** text, size_t* len)
{
    if (!text || !len) return -1;
    *text = nullptr;
    *len = 0;
    uint32_t start, limit;
    parse_args(nargs, a1, a2, &start, &limit);
    char hdr[2048];
    Geometry g;
    const int hn = plan_geometry(start, limit, &g, hdr, sizeof hdr);
    std::vector<Range> ranges;
    if (hn < 0 || !plan_schedule(start, limit, g.mpv, kThreads, ranges)) {
        std::fprintf(stderr, "ffb_emit: arguments (%d, %d) cannot be run\n", a1, a2);
        return -1;
    }
    const uint64_t rec_hi = (uint64_t)recLo + 2 * (nrec ? nrec - 1 : 0);
    for (const Range& r : ranges) {
        const uint32_t f = r.first | 1u;
        if (f > r.last) continue;
        const uint32_t l = r.last - !(r.last & 1);
        if (!(recLo & 1) || nrec == 0 || !h_rec || f < recLo || l > rec_hi) {
            std::fprintf(stderr, "ffb_emit: the records (odd sums %u..%llu) do not cover sums "
                         "%u..%u of the schedule\n", recLo, (unsigned long long)rec_hi, f, l);
            return -1;
        }
    }
    const std::string body = emit(ranges, h_rec, recLo);
    char tail[160];
    const int tn = std::snprintf(tail, sizeof tail, "Prime time: %llu \xce\xbcs\nFreudenthal time: %llu \xce\xbcs\n",
                                 (unsigned long long)primeUs, (unsigned long long)freudUs);
    const size_t n = (size_t)hn + body.size() + (size_t)tn;
    char* out = (char*)std::malloc(n + 1);
    if (!out) return -1;
    std::memcpy(out, hdr, (size_t)hn);
    std::memcpy(out + hn, body.data(), body.size());
    std::memcpy(out + hn + body.size(), tail, (size_t)tn);
    out[n] = 0;
    *text = out;
    *len = n;
    return 0;
}

extern "C" int ffb_map_dump(int deviceIndex, int nargs, int32_t a1, int32_t a2, uint8_t** map,
                            uint64_t* bytes, char* hdr, size_t hdrCap)
{
    if (!map || !bytes) return -1;
    *map = nullptr;
    *bytes = 0;
    uint32_t start, limit;
    parse_args(nargs, a1, a2, &start, &limit);
    char h[2048];
    Geometry g;
    const int hn = plan_geometry(start, limit, &g, h, sizeof h);
    if (hn < 0) {
        std::fprintf(stderr, "ffb_map_dump: %s", g.too_big ? h : "header overflow\n");
        return -1;
    }
    if (hdr && hdrCap) {
        const size_t n = std::min((size_t)hn, hdrCap - 1);
        std::memcpy(hdr, h, n);
        hdr[n] = 0;
    }
    // Prime::PrimeMapSize(): (maxPrimeMapValue + 15) >> 4 bytes; the device map covers
    // (maxPrimeMapValue + 1 + 15) >> 4 bytes, at most one more
    const uint64_t size = (g.mpv + 15) >> 4;
    const uint64_t dev_bytes = (((g.mpv + 1 + 15) >> 4) + 255) & ~255ull;
    uint8_t* d = nullptr;
    uint8_t* out = (uint8_t*)std::malloc(size ? size : 1);
    if (!out) return -1;
    cudaStream_t st = nullptr;
    int rc = 0;
    if (cudaSetDevice(deviceIndex) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&d, dev_bytes) != cudaSuccess) {
        rc = -1;
    } else if (ffb_sieve_map_async(deviceIndex, g.mpv, d, st) != 0 ||
               cudaMemcpyAsync(out, d, size, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
               cudaStreamSynchronize(st) != cudaSuccess) {
        rc = -1;
    }
    if (d) cudaFree(d);
    if (st) cudaStreamDestroy(st);
    if (rc) {
        std::fprintf(stderr, "ffb_map_dump: failed: %s\n", cudaGetErrorString(cudaGetLastError()));
        std::free(out);
        return -1;
    }
    *map = out;
    *bytes = size;
    return 0;
}
