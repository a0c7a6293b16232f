// batch.cu -- many `ff_sieve <sumStart> <sumLimit>` ranges in one launch (ffb_batch_*).
//
// Every range keeps its own output exactly as ff_seg prints it (its own header lines, its
// own 62-way schedule and numbering). The device work is shared:
//   * one prime map, sieved once up to the probe bound of the largest sum of the batch (by
//     the exactness of IsPrime, one map serves every range whatever its own limit);
//   * the sums every range's schedule evaluates, merged into disjoint intervals and handed
//     to ONE persistent search launch as its work queue (largest sums first), each sum
//     evaluated once however many ranges share it;
//   * the sieve and the search launches captured once into a CUDA graph and replayed;
//   * the sieve's tile size, the search's block size (warps per block), the warps that share
//     one sum (1, 2 or 4) and the sums taken per pull of the work queue (sums per chunk;
//     sums per block = warps x chunk / warps per sum) picked by a small autotuner that times
//     the candidates on the batch itself.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ffb200.h"
#include "ffb_internal.h"
#include "../host/plan.h"

namespace ffb {
namespace {

struct RangeJob {
    uint32_t start, limit;
    std::string header;
    std::vector<Range> schedule;
};

struct Interval {
    uint32_t lo, hi;  // odd sums lo..hi
};

struct Tuned {
    uint32_t tile_bytes, warps, chunk, group;
};
std::mutex g_tune_mu;
std::map<std::pair<uint64_t, uint64_t>, Tuned> g_tuned;  // (map bytes, sums) -> choice

}  // namespace
}  // namespace ffb

using namespace ffb;

struct FfbBatch {
    int dev = 0;
    int sms = 0;
    std::vector<RangeJob> jobs;
    std::vector<Interval> iv;        // ascending, disjoint
    std::vector<uint64_t> rec_base;  // per interval (ascending order)
    uint64_t nrec = 0;
    uint64_t map_mpv = 0, map_bytes = 0;
    uint32_t tile_bytes = 0, warps = 8, chunk = 32, group = 1;
    int tuned = 0;
    // device
    uint8_t* d_map = nullptr;
    uint64_t* d_rec = nullptr;
    uint4* d_seg = nullptr;
    uint32_t nseg = 0, nchunks = 0;
    uint32_t* d_words = nullptr;  // [0] work counter, [1] error flags
    SievePlan* sieve = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    uint64_t* h_rec = nullptr;
    bool launched = false;
};

namespace {

int build_sieve(FfbBatch* b)
{
    if (b->sieve) destroy_sieve_plan(b->sieve);
    SieveArgs a;
    a.out = b->d_map;
    a.seg_lo = 0;
    a.seg_hi = b->map_mpv + 1;
    a.tile_bytes = b->tile_bytes;
    a.clear_one = 1;
    a.true_map = 1;
    b->sieve = create_sieve_plan(a, b->sms, b->d_words + 1);
    return b->sieve ? 0 : -1;
}

SearchArgs search_args(const FfbBatch* b, const DeviceState* s)
{
    SearchArgs a;
    a.map = b->d_map;
    a.bound = b->map_mpv;
    a.lo = b->iv.empty() ? 1 : b->iv.front().lo;
    a.hi = b->iv.empty() ? 1 : b->iv.back().hi;
    a.nsums = (uint32_t)b->nrec;
    a.rec = b->d_rec;
    a.grec = nullptr;
    a.grec_base = 0;
    a.gcount = nullptr;
    a.tdiv = s->tdiv;
    a.ntdiv = s->ntdiv;
    a.spf = s->spf;
    a.spf_limit = s->spf_limit;
    a.sched = b->d_words;
    a.err = b->d_words + 1;
    a.stats = nullptr;
    a.seg = b->d_seg;
    a.nseg = b->nseg;
    a.nchunks = b->nchunks;
    a.warps = b->warps;
    a.chunk = b->chunk;
    a.group = b->group;
    return a;
}

// The work queue for b->chunk sums per chunk: the intervals largest first, each entry
// {lo, count, record base, first chunk}, uploaded to d_seg (synchronously).
int build_queue(FfbBatch* b)
{
    std::vector<uint4> seg;
    b->nchunks = 0;
    for (size_t k = b->iv.size(); k-- > 0;) {
        const Interval& x = b->iv[k];
        const uint32_t cnt = (x.hi - x.lo) / 2 + 1;
        seg.push_back(make_uint4(x.lo, cnt, (uint32_t)b->rec_base[k], b->nchunks));
        b->nchunks += (cnt + b->chunk - 1) / b->chunk;
    }
    b->nseg = (uint32_t)seg.size();
    if (!seg.empty())
        FFB_CUDA(cudaMemcpy(b->d_seg, seg.data(), sizeof(uint4) * seg.size(), cudaMemcpyHostToDevice));
    return 0;
}

// sieve + search on b->stream, for capture: the events are recorded as nodes of the graph
// (cudaEventRecordExternal), so every replay timestamps the sieve and the search
int enqueue_all(FfbBatch* b)
{
    DeviceState* s = device_state(b->dev);
    if (!s) return -1;
    FFB_CUDA(cudaEventRecordWithFlags(b->ev[0], b->stream, cudaEventRecordExternal));
    if (enqueue_sieve_plan(b->sieve, b->stream)) return -1;
    FFB_CUDA(cudaEventRecordWithFlags(b->ev[1], b->stream, cudaEventRecordExternal));
    FFB_CUDA(cudaMemsetAsync(b->d_words, 0, 8, b->stream));
    FFB_CUDA(cudaMemsetAsync(b->d_rec, 0, 8 * b->nrec, b->stream));
    if (b->nseg && launch_search(search_args(b, s), b->sms, b->stream)) return -1;
    FFB_CUDA(cudaEventRecordWithFlags(b->ev[2], b->stream, cudaEventRecordExternal));
    return 0;
}

float elapsed(cudaEvent_t a, cudaEvent_t c)
{
    float ms = 0;
    cudaEventElapsedTime(&ms, a, c);
    return ms;
}

// Times each candidate on this batch: sieve tile sizes first (the sieve alone), then the
// search block sizes with the best tile. Results are kept per (map size, sum count).
int autotune(FfbBatch* b)
{
    const std::pair<uint64_t, uint64_t> key(b->map_bytes >> 24, b->nrec >> 12);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            b->tile_bytes = it->second.tile_bytes;
            b->warps = it->second.warps;
            b->chunk = it->second.chunk;
            b->group = it->second.group;
            b->tuned = 2;
            return build_queue(b) || build_sieve(b);
        }
    }
    // the tile shares the CTA's 227 KB of shared memory with ~9 KB of pre-sieve patterns
    const uint32_t tiles[] = {64 * 1024, 96 * 1024, 128 * 1024, 160 * 1024, 192 * 1024, 216 * 1024};
    float best = 1e30f;
    uint32_t best_tile = 216 * 1024;
    for (uint32_t t : tiles) {
        b->tile_bytes = t;
        if (build_sieve(b)) continue;  // a tile that does not fit is skipped
        float ms = 1e30f;
        for (int r = 0; r < 2; ++r) {
            FFB_CUDA(cudaEventRecord(b->ev[0], b->stream));
            if (enqueue_sieve_plan(b->sieve, b->stream)) return -1;
            FFB_CUDA(cudaEventRecord(b->ev[1], b->stream));
            FFB_CUDA(cudaStreamSynchronize(b->stream));
            ms = std::min(ms, elapsed(b->ev[0], b->ev[1]));
        }
        if (ms < best) { best = ms; best_tile = t; }
    }
    b->tile_bytes = best_tile;
    if (build_sieve(b)) return -1;
    if (enqueue_sieve_plan(b->sieve, b->stream)) return -1;  // the map the search reads
    DeviceState* s = device_state(b->dev);
    if (!s) return -1;
    // (warps per sum, sums per chunk): one warp per sum with 16, 32 or 64 sums per pull, or
    // 2 / 4 warps per sum with 32 sums per warp of the group; each with 4, 8, 16 warps a block
    const uint32_t shapes[][2] = {{1, 16}, {1, 32}, {1, 64}, {2, 64}, {4, 128}};
    best = 1e30f;
    uint32_t best_w = 8, best_c = 32, best_g = 1;
    for (const auto& sh : shapes) {
        b->group = sh[0];
        b->chunk = sh[1];
        if (build_queue(b)) return -1;
        for (uint32_t w : {4u, 8u, 16u}) {
            b->warps = w;
            FFB_CUDA(cudaMemsetAsync(b->d_words, 0, 8, b->stream));
            FFB_CUDA(cudaEventRecord(b->ev[1], b->stream));
            if (b->nseg && launch_search(search_args(b, s), b->sms, b->stream)) return -1;
            FFB_CUDA(cudaEventRecord(b->ev[2], b->stream));
            FFB_CUDA(cudaStreamSynchronize(b->stream));
            const float ms = elapsed(b->ev[1], b->ev[2]);
            if (ms < best) { best = ms; best_w = w; best_c = b->chunk; best_g = b->group; }
        }
    }
    b->warps = best_w;
    b->chunk = best_c;
    b->group = best_g;
    if (build_queue(b)) return -1;
    b->tuned = 1;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = {b->tile_bytes, b->warps, b->chunk, b->group};
    return 0;
}

int capture(FfbBatch* b)
{
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    FFB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_all(b);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        std::fprintf(stderr, "ffb_batch: graph capture failed: %s\n", cudaGetErrorString(e));
        cudaGetLastError();
        return -1;
    }
    b->graph = g;
    FFB_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    return 0;
}

// record index of odd sum s (which some interval contains)
inline uint64_t rec_index(const FfbBatch* b, uint32_t s)
{
    size_t a = 0, c = b->iv.size() - 1;
    while (a < c) {
        const size_t m = (a + c + 1) / 2;
        if (b->iv[m].lo <= s) a = m; else c = m - 1;
    }
    return b->rec_base[a] + ((s - b->iv[a].lo) >> 1);
}

std::string emit_job(const FfbBatch* b, const RangeJob& j, double prime_us, double freud_us)
{
    std::string out = j.header;
    char line[kMaxLine];
    uint32_t count = 0;
    for (const Range& r : j.schedule)
        for (uint32_t s = r.first | 1u; s <= r.last; s += 2) {
            const uint64_t v = b->h_rec[rec_index(b, s)];
            if (!v) continue;
            char* e = format_line(line, ++count, s, rec_low(v), rec_high(v), rec_low_prime(v),
                                  rec_high_prime(v));
            out.append(line, (size_t)(e - line));
        }
    char tail[160];
    const int n = std::snprintf(tail, sizeof tail,
                                "Prime time: %llu \xce\xbcs\nFreudenthal time: %llu \xce\xbcs\n",
                                (unsigned long long)prime_us, (unsigned long long)freud_us);
    out.append(tail, (size_t)n);
    return out;
}

}  // namespace

extern "C" void ffb_batch_destroy(FfbBatch* b)
{
    if (!b) return;
    cudaSetDevice(b->dev);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    destroy_sieve_plan(b->sieve);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->d_map) cudaFree(b->d_map);
    if (b->d_rec) cudaFree(b->d_rec);
    if (b->d_seg) cudaFree(b->d_seg);
    if (b->d_words) cudaFree(b->d_words);
    if (b->h_rec) cudaFreeHost(b->h_rec);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

extern "C" FfbBatch* ffb_batch_create(int deviceIndex, uint32_t n, const int32_t* starts,
                                      const int32_t* limits, int autotune_flag)
{
    DeviceState* st = device_state(deviceIndex);
    if (!st || n == 0 || !starts || !limits) return nullptr;
    FfbBatch* b = new FfbBatch;
    b->dev = deviceIndex;
    b->sms = st->sms;
    // ---- host plan: every range's header and schedule, the merged intervals ----
    std::vector<Interval> all;
    uint32_t top = 0;
    for (uint32_t i = 0; i < n; ++i) {
        RangeJob j;
        parse_args(2, starts[i], limits[i], &j.start, &j.limit);
        char hdr[2048];
        Geometry g;
        const int hn = plan_geometry(j.start, j.limit, &g, hdr, sizeof hdr);
        if (hn < 0 || !plan_schedule(j.start, j.limit, g.mpv, kThreads, j.schedule)) {
            std::fprintf(stderr, "ffb_batch: range %u (%d, %d) cannot be run\n", i, starts[i],
                         limits[i]);
            delete b;
            return nullptr;
        }
        j.header.assign(hdr, (size_t)hn);
        for (const Range& r : j.schedule) {
            const uint32_t f = r.first | 1u;
            if (f > r.last) continue;
            const uint32_t l = r.last - !(r.last & 1);
            all.push_back({f, l});
            top = std::max(top, l);
        }
        b->jobs.push_back(std::move(j));
    }
    if (top > kMaxSum) {
        std::fprintf(stderr, "ffb_batch: sums above 2^25 are outside the exact domain\n");
        delete b;
        return nullptr;
    }
    std::sort(all.begin(), all.end(), [](const Interval& x, const Interval& y) { return x.lo < y.lo; });
    for (const Interval& x : all) {
        if (!b->iv.empty() && x.lo <= b->iv.back().hi + 2) b->iv.back().hi = std::max(b->iv.back().hi, x.hi);
        else b->iv.push_back(x);
    }
    for (const Interval& x : b->iv) {
        b->rec_base.push_back(b->nrec);
        b->nrec += (x.hi - x.lo) / 2 + 1;
    }
    b->map_mpv = std::max<uint64_t>(ffb_probe_bound(std::max(top, 5u)), 15);
    b->map_bytes = (b->map_mpv + 1 + 15) >> 4;
    // ---- device buffers ----
    bool ok = cudaSetDevice(deviceIndex) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&b->d_map, (b->map_bytes + 255) & ~255ull) == cudaSuccess &&
              cudaMalloc(&b->d_rec, 8 * std::max<uint64_t>(b->nrec, 1)) == cudaSuccess &&
              cudaMalloc(&b->d_seg, sizeof(uint4) * std::max<size_t>(b->iv.size(), 1)) == cudaSuccess &&
              cudaMalloc(&b->d_words, 256) == cudaSuccess &&
              cudaMallocHost(&b->h_rec, 8 * std::max<uint64_t>(b->nrec, 1)) == cudaSuccess;
    for (cudaEvent_t& e : b->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    b->chunk = 32;
    ok = ok && build_queue(b) == 0;
    if (!ok) {
        std::fprintf(stderr, "ffb_batch: device allocation failed (map %llu bytes): %s\n",
                     (unsigned long long)b->map_bytes, cudaGetErrorString(cudaGetLastError()));
        ffb_batch_destroy(b);
        return nullptr;
    }
    b->tile_bytes = 216 * 1024;
    b->warps = 8;
    if ((autotune_flag ? autotune(b) : build_sieve(b)) || capture(b)) {
        ffb_batch_destroy(b);
        return nullptr;
    }
    return b;
}

extern "C" int ffb_batch_launch(FfbBatch* b, void* stream)
{
    if (!b) return -1;
    FFB_CUDA(cudaSetDevice(b->dev));
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    FFB_CUDA(cudaGraphLaunch(b->exec, st));
    b->launched = true;
    return 0;
}

extern "C" int ffb_batch_collect(FfbBatch* b, char** text, size_t* offsets)
{
    using clk = std::chrono::steady_clock;
    if (!b || !b->launched) return -1;
    *text = nullptr;
    FFB_CUDA(cudaSetDevice(b->dev));
    FFB_CUDA(cudaMemcpyAsync(b->h_rec, b->d_rec, 8 * b->nrec, cudaMemcpyDeviceToHost, b->stream));
    FFB_CUDA(cudaStreamSynchronize(b->stream));
    uint32_t flags = 0;
    FFB_CUDA(cudaMemcpy(&flags, b->d_words + 1, 4, cudaMemcpyDeviceToHost));
    if (flags) {
        std::fprintf(stderr, "ffb_batch: device error flags 0x%x\n", flags);
        return -1;
    }
    const auto t0 = clk::now();
    const double prime_us = 1e3 * elapsed(b->ev[0], b->ev[1]);
    const double search_us = 1e3 * elapsed(b->ev[1], b->ev[2]);
    const size_t n = b->jobs.size();
    std::vector<std::string> parts(n);
    unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (size_t i = t; i < n; i += nt)
                parts[i] = emit_job(b, b->jobs[i], prime_us, search_us);
        });
    for (auto& t : th) t.join();
    (void)t0;
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) {
        offsets[i] = total;
        total += parts[i].size();
    }
    offsets[n] = total;
    char* out = (char*)std::malloc(total + 1);
    if (!out) return -1;
    for (size_t i = 0; i < n; ++i) std::memcpy(out + offsets[i], parts[i].data(), parts[i].size());
    out[total] = 0;
    *text = out;
    b->launched = false;
    return 0;
}

extern "C" int ffb_batch_info(const FfbBatch* b, FfbBatchInfo* info)
{
    if (!b || !info) return -1;
    info->ranges = (uint32_t)b->jobs.size();
    info->intervals = b->nseg;
    info->sums = b->nrec;
    info->mapMaxValue = b->map_mpv;
    info->mapBytes = b->map_bytes;
    info->sieveTileBytes = b->tile_bytes;
    info->searchWarps = b->warps;
    info->searchChunk = b->chunk;
    info->searchGroup = b->group;
    info->autotuned = b->tuned;
    info->sieveMs = 0;
    info->searchMs = 0;
    if (cudaEventQuery(b->ev[2]) == cudaSuccess) {
        info->sieveMs = elapsed(b->ev[0], b->ev[1]);
        info->searchMs = elapsed(b->ev[1], b->ev[2]);
    }
    cudaGetLastError();
    return 0;
}
