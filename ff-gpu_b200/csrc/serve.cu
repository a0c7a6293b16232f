// serve.cu -- the serving loop (ffb_serve_*): ff_sieve requests submitted at any time,
// continuously batched into search launches over a resident prime map.
//
// Device memory follows the reference's budget (source/budget.cpp:15-42): of
// min(f x free, cap), the backing bytes hold the prime map and the scratch bytes hold the
// launch slots (records, work queue, counters). The map is sieved in segments as requests
// with larger limits are admitted, up to the bound their probes reach or the backing
// bytes, whichever is smaller; a probe above it goes to Miller-Rabin, which is exact, so
// the output never depends on how far the map reaches.
//
// Two host threads drive the device:
//   * the scheduler waits for a free slot, fills one launch with a slice of every waiting
//     request (oldest first, equal shares of the launch's work, each request's sums in its
//     emission order), grows the map if the launch needs it, merges the slices' sums into
//     disjoint intervals (the search's work queue) and enqueues copy-in, search and
//     copy-out on the slot's stream;
//   * the completer takes launches in the order they were issued, waits for each, formats
//     every slice's solution lines from the slot's records (numbered on from the request's
//     previous slice) and queues them as the request's next chunk.
// Slots run on separate streams, so a launch's tail overlaps the next launch's head and
// new requests join the next launch instead of waiting for the work in front of them.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ffb200.h"
#include "ffb_internal.h"
#include "../host/plan.h"

namespace ffb {
namespace {

constexpr int kMaxSlots = 8;
constexpr uint32_t kMaxPieces = 8192;          // slices (and so intervals) per launch
constexpr uint64_t kGrowStep = 1ull << 32;     // map growth granularity, in values
constexpr double kCostUnit = 2097152.0;        // a sum s costs s / 2^21 units

using Clock = std::chrono::steady_clock;

struct Request;

// A slice of one request's sums: the odd sums lo..hi of one of its schedule ranges.
struct Piece {
    Request* r;
    uint32_t lo, hi;
    uint64_t rec_off;  // record index of lo in the slot's records
    bool last;         // the request's final slice
};

struct Request {
    uint64_t id = 0;
    uint32_t start = 0, limit = 0;
    std::string header;
    std::vector<Range> sched;
    // issue cursor (scheduler thread): next schedule range and next odd sum in it
    size_t cur = 0;
    uint32_t next = 0;
    uint32_t top = 0;         // largest sum of the schedule
    uint64_t sums = 0;        // odd sums of the schedule
    bool issued = false;      // every slice handed to a launch
    // emission state (completer thread)
    uint32_t lines = 0, seq = 0;
    uint64_t hash = 1469598103934665603ull;
    uint64_t text_bytes = 0;
    cudaEvent_t grow_a = nullptr, grow_b = nullptr;  // map growth its admission caused
    uint32_t launches = 0;
    uint64_t last_launch = ~0ull;
    int state = 0;            // 0 queued, 1 running, 2 done, -1 failed
    double submit_us = 0, admit_us = 0, first_us = 0, done_us = 0;
};

struct Growth {
    cudaEvent_t a = nullptr, b = nullptr;
    float ms = -1;
};

struct Slot {
    cudaStream_t stream = nullptr;
    uint64_t* d_rec = nullptr;
    uint64_t* h_rec = nullptr;   // pinned
    uint8_t* d_q = nullptr;      // [0,256) words (work counter, error), then the intervals
    uint8_t* h_q = nullptr;      // pinned staging of d_q
    uint32_t* h_err = nullptr;   // pinned copy of the error word
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
    std::vector<Piece> pieces;
    uint64_t nrec = 0;
    uint64_t launch_id = 0;
    bool launched = false;
};

}  // namespace
}  // namespace ffb

using namespace ffb;

struct FfbServer {
    int dev = 0;
    DeviceState* ds = nullptr;
    FfbServeConfig cfg{};
    FfbBudget budget{};
    Clock::time_point t0;
    // resident map: values [0, sieved) are valid, capacity cap_values
    uint8_t* d_map = nullptr;
    uint64_t cap_values = 0;
    uint64_t sieved = 0;
    cudaStream_t grow_stream = nullptr;
    std::vector<Growth> growths;
    unsigned long long* d_stats = nullptr;
    Slot slots[kMaxSlots];
    uint32_t nslots = 0;
    uint64_t slot_recs = 0;   // record capacity of one launch
    // shared state (mu)
    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_out, cv_drain;
    std::vector<std::unique_ptr<Request>> reqs;
    std::deque<Request*> waiting;
    std::deque<int> free_slots, inflight;
    std::deque<FfbServeChunk> out;
    bool stop = false, sched_exited = false;
    uint64_t completed = 0, failed = 0, launches = 0, sums_req = 0, sums_searched = 0;
    uint64_t chunks = 0, text_bytes = 0;
    uint32_t max_queued = 0;
    double sieve_ms = 0, search_ms = 0;
    std::thread sched_thr, done_thr;

    double now_us() const
    {
        return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    }
};

namespace {

uint64_t fnv1a(uint64_t h, const char* p, size_t n)
{
    for (size_t i = 0; i < n; ++i) {
        h ^= (unsigned char)p[i];
        h *= 1099511628211ull;
    }
    return h;
}

// Values the map must cover for sums up to `top`: every probe (ffb_probe_bound), as a
// count of values rounded up to the growth step, capped at the capacity.
uint64_t map_need(const FfbServer* S, uint32_t top)
{
    const uint64_t want = ffb_probe_bound(std::max(top, 5u)) + 1;
    const uint64_t r = (want + kGrowStep - 1) / kGrowStep * kGrowStep;
    return std::min(r, S->cap_values);
}

// Sieves the map's values [S->sieved, hi) on the growth stream (segment output lands at
// its global position: seg_lo is a multiple of 256, so byte seg_lo/16 is 16-byte aligned).
int grow_map(FfbServer* S, uint64_t hi, Growth* growth)
{
    Growth g;
    FFB_CUDA(cudaEventCreate(&g.a));
    FFB_CUDA(cudaEventCreate(&g.b));
    FFB_CUDA(cudaEventRecord(g.a, S->grow_stream));
    const uint64_t lo = S->sieved;
    const int rc = run_sieve_map(S->dev, lo, hi, S->d_map + (lo >> 4), S->grow_stream, lo == 0);
    if (rc || cudaEventRecord(g.b, S->grow_stream) != cudaSuccess) {
        cudaEventDestroy(g.a);
        cudaEventDestroy(g.b);
        return -1;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->growths.push_back(g);
    *growth = g;
    S->sieved = hi;
    return 0;
}

// Takes slices for one launch from the waiting requests (mu held). Returns the largest sum.
uint32_t fill(FfbServer* S, Slot& sl)
{
    sl.pieces.clear();
    sl.nrec = 0;
    const double work_cap = (double)S->cfg.launchWork;
    double work = 0;
    const size_t nwait = S->waiting.size();
    const double quantum = std::max(work_cap / (double)std::max<size_t>(nwait, 1), 256.0);
    uint32_t top = 0;
    const double t = S->now_us();
    size_t k = 0;
    while (k < S->waiting.size() && work < work_cap && sl.nrec < S->slot_recs &&
           sl.pieces.size() < kMaxPieces) {
        Request* r = S->waiting[k];
        if (r->state < 0) {  // failed in an earlier launch: nothing more to search
            S->waiting.erase(S->waiting.begin() + (long)k);
            continue;
        }
        if (r->state == 0) {
            r->state = 1;
            r->admit_us = t;
        }
        double share = std::min(quantum, work_cap - work);
        while (!r->issued && share > 0 && sl.nrec < S->slot_recs && sl.pieces.size() < kMaxPieces) {
            const Range& rg = r->sched[r->cur];
            const uint32_t last = rg.last - !(rg.last & 1);
            const uint32_t lo = r->next;
            uint64_t n = (uint64_t)(share * kCostUnit / (double)lo) + 1;
            n = std::max<uint64_t>(n, 32);
            n = std::min<uint64_t>(n, (uint64_t)(last - lo) / 2 + 1);
            n = std::min<uint64_t>(n, S->slot_recs - sl.nrec);
            const uint32_t hi = lo + 2 * (uint32_t)(n - 1);
            sl.pieces.push_back({r, lo, hi, 0, false});
            sl.nrec += n;
            const double c = (double)n * (0.5 * ((double)lo + hi)) / kCostUnit;
            share -= c;
            work += c;
            top = std::max(top, hi);
            if (hi == last) {
                // next non-empty schedule range
                size_t j = r->cur + 1;
                while (j < r->sched.size() && (r->sched[j].first | 1u) > r->sched[j].last) ++j;
                if (j == r->sched.size()) {
                    r->issued = true;
                    sl.pieces.back().last = true;
                } else {
                    r->cur = j;
                    r->next = r->sched[j].first | 1u;
                }
            } else {
                r->next = hi + 2;
            }
        }
        if (r->issued) S->waiting.erase(S->waiting.begin() + (long)k);
        else ++k;
    }
    return top;
}

// Merged intervals of the launch's slices into the staging buffer; record offsets of the
// slices. Returns the interval count and sets *nchunks and *nrec.
uint32_t build_queue(Slot& sl, uint32_t* nchunks)
{
    struct Iv { uint32_t lo, hi; };
    std::vector<Iv> all;
    all.reserve(sl.pieces.size());
    for (const Piece& p : sl.pieces) all.push_back({p.lo, p.hi});
    std::sort(all.begin(), all.end(), [](const Iv& a, const Iv& b) { return a.lo < b.lo; });
    std::vector<Iv> iv;
    for (const Iv& x : all) {
        if (!iv.empty() && x.lo <= iv.back().hi + 2) iv.back().hi = std::max(iv.back().hi, x.hi);
        else iv.push_back(x);
    }
    std::vector<uint64_t> base(iv.size());
    uint64_t nrec = 0;
    for (size_t k = 0; k < iv.size(); ++k) {
        base[k] = nrec;
        nrec += (iv[k].hi - iv[k].lo) / 2 + 1;
    }
    for (Piece& p : sl.pieces) {
        size_t a = 0, c = iv.size() - 1;
        while (a < c) {
            const size_t m = (a + c + 1) / 2;
            if (iv[m].lo <= p.lo) a = m; else c = m - 1;
        }
        p.rec_off = base[a] + (p.lo - iv[a].lo) / 2;
    }
    uint4* q = reinterpret_cast<uint4*>(sl.h_q + 256);
    uint32_t chunks = 0, n = 0;
    for (size_t k = iv.size(); k-- > 0;) {  // largest sums first
        const uint32_t cnt = (iv[k].hi - iv[k].lo) / 2 + 1;
        q[n++] = make_uint4(iv[k].lo, cnt, (uint32_t)base[k], chunks);
        chunks += (cnt + 31) / 32;
    }
    std::memset(sl.h_q, 0, 256);
    sl.nrec = nrec;
    *nchunks = chunks;
    return n;
}

int enqueue(FfbServer* S, Slot& sl, uint32_t top)
{
    uint32_t nchunks = 0;
    const uint32_t nseg = build_queue(sl, &nchunks);
    if (!S->growths.empty())
        FFB_CUDA(cudaStreamWaitEvent(sl.stream, S->growths.back().b, 0));
    FFB_CUDA(cudaMemcpyAsync(sl.d_q, sl.h_q, 256 + sizeof(uint4) * nseg, cudaMemcpyHostToDevice,
                             sl.stream));
    FFB_CUDA(cudaMemsetAsync(sl.d_rec, 0, 8 * sl.nrec, sl.stream));
    SearchArgs a;
    a.map = S->d_map;
    a.bound = S->sieved - 1;
    a.lo = 5;
    a.hi = std::max(top, 5u);
    a.nsums = (uint32_t)sl.nrec;
    a.rec = sl.d_rec;
    a.grec = nullptr;
    a.grec_base = 0;
    a.gcount = nullptr;
    a.tdiv = S->ds->tdiv;
    a.ntdiv = S->ds->ntdiv;
    a.spf = S->ds->spf;
    a.spf_limit = S->ds->spf_limit;
    a.sched = reinterpret_cast<uint32_t*>(sl.d_q);
    a.err = reinterpret_cast<uint32_t*>(sl.d_q) + 1;
    a.stats = S->d_stats;
    a.seg = reinterpret_cast<const uint4*>(sl.d_q + 256);
    a.nseg = nseg;
    a.nchunks = nchunks;
    a.warps = S->cfg.searchWarps;
    FFB_CUDA(cudaEventRecord(sl.ev0, sl.stream));
    if (launch_search(a, S->ds->sms, sl.stream)) return -1;
    FFB_CUDA(cudaEventRecord(sl.ev1, sl.stream));
    FFB_CUDA(cudaMemcpyAsync(sl.h_rec, sl.d_rec, 8 * sl.nrec, cudaMemcpyDeviceToHost, sl.stream));
    FFB_CUDA(cudaMemcpyAsync(sl.h_err, sl.d_q + 4, 4, cudaMemcpyDeviceToHost, sl.stream));
    FFB_CUDA(cudaEventRecord(sl.done, sl.stream));
    return 0;
}

void fail_pieces(FfbServer* S, Slot& sl, std::vector<FfbServeChunk>& chunks)
{
    for (const Piece& p : sl.pieces) {
        Request* r = p.r;
        if (r->state < 0 || r->state == 2) continue;
        r->state = -1;
        r->done_us = S->now_us();
        chunks.push_back({r->id, r->seq++, -1, nullptr, 0});
    }
}

void scheduler(FfbServer* S)
{
    cudaSetDevice(S->dev);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_sched.wait(lk, [&] { return S->stop || (!S->waiting.empty() && !S->free_slots.empty()); });
        if (S->stop) break;
        const int si = S->free_slots.front();
        S->free_slots.pop_front();
        Slot& sl = S->slots[si];
        const uint32_t top = fill(S, sl);
        sl.launch_id = S->launches++;
        for (Piece& p : sl.pieces) {
            if (p.r->last_launch != sl.launch_id) {
                p.r->last_launch = sl.launch_id;
                ++p.r->launches;
            }
        }
        const uint64_t need = map_need(S, top);
        const uint64_t had = S->sieved;
        lk.unlock();
        Growth growth;
        int rc = 0;
        if (need > had) {
            rc = grow_map(S, need, &growth);
            // the sieve time is charged to the requests admitted by this launch whose sums
            // needed the new part of the map
            if (!rc)
                for (Piece& p : sl.pieces)
                    if (p.r->launches == 1 && !p.r->grow_a && map_need(S, p.hi) > had) {
                        p.r->grow_a = growth.a;
                        p.r->grow_b = growth.b;
                    }
        }
        if (!rc) rc = enqueue(S, sl, top);
        lk.lock();
        sl.launched = rc == 0;
        if (rc) {
            std::fprintf(stderr, "ffb_serve: launch failed: %s\n", cudaGetErrorString(cudaGetLastError()));
        }
        S->inflight.push_back(si);
        S->cv_done.notify_one();
    }
    S->sched_exited = true;
    S->cv_done.notify_all();
}

// What emitting one launch changes in a request's emission state; applied under mu.
struct Emitted {
    Request* r;
    uint32_t lines, seq;
    uint64_t hash, text_bytes;
    double done_us;
};

// Formats the launch's slices (completer thread, mu not held): chunks in slice order. Only
// the completer thread writes a request's emission state, so it reads that state here
// without the lock; its new values go to `upd`, which the caller stores under mu (readers
// such as ffb_serve_request_info take mu). `failed` holds, per piece, whether its request
// had failed when the launch was taken (read under mu).
void emit_launch(FfbServer* S, Slot& sl, const std::vector<char>& failed,
                 std::vector<FfbServeChunk>& chunks, std::vector<Emitted>& upd)
{
    size_t i = 0;
    char line[kMaxLine];
    while (i < sl.pieces.size()) {
        Request* r = sl.pieces[i].r;
        size_t j = i;
        while (j < sl.pieces.size() && sl.pieces[j].r == r) ++j;
        if (failed[i]) { i = j; continue; }
        Emitted* e = nullptr;
        for (Emitted& u : upd)
            if (u.r == r) e = &u;
        if (!e) {
            upd.push_back({r, r->lines, r->seq, r->hash, r->text_bytes, r->done_us});
            e = &upd.back();
        }
        std::string text;
        if (e->seq == 0) text = r->header;
        bool final = false;
        for (size_t k = i; k < j; ++k) {
            const Piece& p = sl.pieces[k];
            const uint64_t* rec = sl.h_rec + p.rec_off;
            const size_t body0 = text.size();
            for (uint32_t s = p.lo; s <= p.hi; s += 2) {
                const uint64_t v = rec[(s - p.lo) >> 1];
                if (!v) continue;
                char* end = format_line(line, ++e->lines, s, rec_low(v), rec_high(v),
                                        rec_low_prime(v), rec_high_prime(v));
                text.append(line, (size_t)(end - line));
            }
            e->hash = fnv1a(e->hash, text.data() + body0, text.size() - body0);
            final = final || p.last;
        }
        if (final) {
            double prime_us = 0;
            float ms = 0;
            if (r->grow_a && cudaEventElapsedTime(&ms, r->grow_a, r->grow_b) == cudaSuccess)
                prime_us = 1e3 * ms;
            e->done_us = S->now_us();
            char tail[160];
            const int n = std::snprintf(
                tail, sizeof tail, "Prime time: %llu \xce\xbcs\nFreudenthal time: %llu \xce\xbcs\n",
                (unsigned long long)prime_us, (unsigned long long)(e->done_us - r->admit_us));
            text.append(tail, (size_t)n);
        }
        char* buf = (char*)std::malloc(text.size() + 1);
        std::memcpy(buf, text.data(), text.size());
        buf[text.size()] = 0;
        e->text_bytes += text.size();
        chunks.push_back({r->id, e->seq++, final ? 1 : 0, buf, text.size()});
        i = j;
    }
}

void completer(FfbServer* S)
{
    cudaSetDevice(S->dev);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_done.wait(lk, [&] { return !S->inflight.empty() || S->sched_exited; });
        if (S->inflight.empty()) break;
        const int si = S->inflight.front();
        Slot& sl = S->slots[si];
        std::vector<char> failed(sl.pieces.size());
        for (size_t k = 0; k < sl.pieces.size(); ++k) failed[k] = sl.pieces[k].r->state < 0;
        lk.unlock();
        std::vector<Emitted> upd;
        std::vector<FfbServeChunk> chunks;
        bool ok = sl.launched && cudaEventSynchronize(sl.done) == cudaSuccess;
        float ms = 0;
        if (ok && cudaEventElapsedTime(&ms, sl.ev0, sl.ev1) != cudaSuccess) ms = 0;
        if (ok && *sl.h_err) {
            std::fprintf(stderr, "ffb_serve: device error flags 0x%x\n", *sl.h_err);
            ok = false;
        }
        uint64_t nsums = 0;
        for (const Piece& p : sl.pieces) nsums += (p.hi - p.lo) / 2 + 1;
        if (ok) emit_launch(S, sl, failed, chunks, upd);
        lk.lock();
        for (const Emitted& u : upd) {
            u.r->lines = u.lines;
            u.r->seq = u.seq;
            u.r->hash = u.hash;
            u.r->text_bytes = u.text_bytes;
            u.r->done_us = u.done_us;
        }
        if (!ok) fail_pieces(S, sl, chunks);
        S->search_ms += ms;
        S->sums_searched += sl.nrec;
        S->sums_req += nsums;
        for (FfbServeChunk& c : chunks) {
            Request* r = S->reqs[c.request].get();
            if (c.seq == 0) r->first_us = S->now_us();
            if (c.status == 1) {
                r->state = 2;
                ++S->completed;
            } else if (c.status < 0) {
                ++S->failed;
            }
            S->text_bytes += c.len;
            ++S->chunks;
            S->out.push_back(c);
        }
        S->inflight.pop_front();
        sl.pieces.clear();
        S->free_slots.push_back(si);
        S->cv_sched.notify_one();
        S->cv_out.notify_all();
        S->cv_drain.notify_all();
    }
}

void release(FfbServer* S)
{
    cudaSetDevice(S->dev);
    for (uint32_t i = 0; i < S->nslots; ++i) {
        Slot& sl = S->slots[i];
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.d_rec) cudaFree(sl.d_rec);
        if (sl.d_q) cudaFree(sl.d_q);
        if (sl.h_rec) cudaFreeHost(sl.h_rec);
        if (sl.h_q) cudaFreeHost(sl.h_q);
        if (sl.h_err) cudaFreeHost(sl.h_err);
        for (cudaEvent_t e : {sl.ev0, sl.ev1, sl.done})
            if (e) cudaEventDestroy(e);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    if (S->grow_stream) {
        cudaStreamSynchronize(S->grow_stream);
        cudaStreamDestroy(S->grow_stream);
    }
    for (Growth& g : S->growths) {
        if (g.a) cudaEventDestroy(g.a);
        if (g.b) cudaEventDestroy(g.b);
    }
    if (S->d_map) cudaFree(S->d_map);
    if (S->d_stats) cudaFree(S->d_stats);
    for (FfbServeChunk& c : S->out) std::free(c.text);
    delete S;
}

}  // namespace

extern "C" FfbServer* ffb_serve_create(int deviceIndex, const FfbServeConfig* cfg)
{
    DeviceState* ds = device_state(deviceIndex);
    if (!ds) return nullptr;
    FfbServer* S = new FfbServer;
    S->dev = deviceIndex;
    S->ds = ds;
    S->t0 = Clock::now();
    if (cfg) S->cfg = *cfg;
    FfbServeConfig& c = S->cfg;
    if (!(c.vramFraction > 0)) c.vramFraction = 0.90;
    if (c.slots == 0) c.slots = 4;
    c.slots = std::min<uint32_t>(c.slots, kMaxSlots);
    if (c.launchWork == 0) c.launchWork = 131072;  // smaller launches leave SMs idle
    if (c.launchSums == 0) c.launchSums = 1u << 22;
    if (c.searchWarps != 4 && c.searchWarps != 16) c.searchWarps = 8;  // fastest measured
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(deviceIndex) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess ||
        ffb_compute_budget(free_b, c.vramFraction, c.vramBudgetBytes, 0, 0, &S->budget)) {
        std::fprintf(stderr, "ffb_serve: cannot read the device's free memory\n");
        delete S;
        return nullptr;
    }
    // slots from the scratch bytes: records + pinned staging of the work queue per slot
    const uint64_t q_bytes = 256 + sizeof(uint4) * kMaxPieces;
    const uint64_t per_slot = S->budget.scratch / c.slots;
    if (per_slot <= q_bytes + 8 * 4096 || S->budget.backing < (1ull << 20)) {
        std::fprintf(stderr, "ffb_serve: budget %llu bytes leaves no room for the map and %u slots\n",
                     S->budget.budget, c.slots);
        delete S;
        return nullptr;
    }
    S->slot_recs = std::min<uint64_t>((per_slot - q_bytes) / 8, c.launchSums);
    S->cap_values = ((S->budget.backing - 256) & ~255ull) * 16;
    S->nslots = c.slots;
    bool ok = cudaStreamCreateWithFlags(&S->grow_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&S->d_map, S->budget.backing) == cudaSuccess &&
              cudaMalloc(&S->d_stats, 32) == cudaSuccess && cudaMemset(S->d_stats, 0, 32) == cudaSuccess;
    for (uint32_t i = 0; ok && i < S->nslots; ++i) {
        Slot& sl = S->slots[i];
        ok = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) == cudaSuccess &&
             cudaMalloc(&sl.d_rec, 8 * S->slot_recs) == cudaSuccess &&
             cudaMalloc(&sl.d_q, q_bytes) == cudaSuccess &&
             cudaMallocHost(&sl.h_rec, 8 * S->slot_recs) == cudaSuccess &&
             cudaMallocHost(&sl.h_q, q_bytes) == cudaSuccess &&
             cudaMallocHost(&sl.h_err, 16) == cudaSuccess &&
             cudaEventCreate(&sl.ev0) == cudaSuccess && cudaEventCreate(&sl.ev1) == cudaSuccess &&
             cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess;
        S->free_slots.push_back((int)i);
    }
    if (ok && c.warmLimit) {
        Growth g;
        ok = c.warmLimit <= kMaxSum && grow_map(S, map_need(S, c.warmLimit), &g) == 0 &&
             cudaStreamSynchronize(S->grow_stream) == cudaSuccess;
    }
    if (!ok) {
        std::fprintf(stderr, "ffb_serve: device allocation failed: %s\n",
                     cudaGetErrorString(cudaGetLastError()));
        release(S);
        return nullptr;
    }
    S->sched_thr = std::thread(scheduler, S);
    S->done_thr = std::thread(completer, S);
    return S;
}

extern "C" int64_t ffb_serve_submit(FfbServer* S, int nargs, int32_t a1, int32_t a2)
{
    if (!S) return -1;
    auto r = std::make_unique<Request>();
    parse_args(nargs, a1, a2, &r->start, &r->limit);
    char hdr[2048];
    Geometry g;
    const int hn = plan_geometry(r->start, r->limit, &g, hdr, sizeof hdr);
    if (hn < 0 || !plan_schedule(r->start, r->limit, g.mpv, kThreads, r->sched)) {
        std::fprintf(stderr, "ffb_serve: request (%d, %d) cannot be run\n", a1, a2);
        return -1;
    }
    r->header.assign(hdr, (size_t)hn);
    size_t first = r->sched.size();
    for (size_t j = 0; j < r->sched.size(); ++j) {
        const Range& rg = r->sched[j];
        if ((rg.first | 1u) > rg.last) continue;
        if (first == r->sched.size()) first = j;
        const uint32_t last = rg.last - !(rg.last & 1);
        r->top = std::max(r->top, last);
        r->sums += (last - (rg.first | 1u)) / 2 + 1;
    }
    if (r->top > kMaxSum) {
        std::fprintf(stderr, "ffb_serve: sums above 2^25 are outside the exact domain\n");
        return -1;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    r->id = S->reqs.size();
    r->submit_us = S->now_us();
    Request* p = r.get();
    S->reqs.push_back(std::move(r));
    if (first == p->sched.size()) {
        // nothing to search: the header and the timing lines only
        p->admit_us = p->first_us = p->done_us = p->submit_us;
        p->issued = true;
        p->state = 2;
        std::string text = p->header + "Prime time: 0 \xce\xbcs\nFreudenthal time: 0 \xce\xbcs\n";
        char* buf = (char*)std::malloc(text.size() + 1);
        std::memcpy(buf, text.data(), text.size() + 1);
        p->text_bytes = text.size();
        p->seq = 1;
        S->out.push_back({p->id, 0, 1, buf, text.size()});
        ++S->completed;
        ++S->chunks;
        S->text_bytes += text.size();
        S->cv_out.notify_all();
        S->cv_drain.notify_all();
        return (int64_t)p->id;
    }
    p->cur = first;
    p->next = p->sched[first].first | 1u;
    S->waiting.push_back(p);
    S->max_queued = std::max<uint32_t>(S->max_queued, (uint32_t)S->waiting.size());
    S->cv_sched.notify_one();
    return (int64_t)p->id;
}

extern "C" int ffb_serve_next(FfbServer* S, FfbServeChunk* out, int timeoutMs)
{
    if (!S || !out) return -1;
    std::unique_lock<std::mutex> lk(S->mu);
    auto ready = [&] { return !S->out.empty(); };
    if (timeoutMs < 0) S->cv_out.wait(lk, ready);
    else if (!S->cv_out.wait_for(lk, std::chrono::milliseconds(timeoutMs), ready)) return 0;
    *out = S->out.front();
    S->out.pop_front();
    return 1;
}

extern "C" int ffb_serve_request_info(FfbServer* S, uint64_t id, FfbServeRequestInfo* o)
{
    if (!S || !o) return -1;
    std::lock_guard<std::mutex> lk(S->mu);
    if (id >= S->reqs.size()) return -1;
    const Request& r = *S->reqs[id];
    o->sumStart = r.start;
    o->sumLimit = r.limit;
    o->sums = r.sums;
    o->textBytes = r.text_bytes;
    o->bodyHash = r.hash;
    o->submitUs = r.submit_us;
    o->admitUs = r.admit_us;
    o->firstChunkUs = r.first_us;
    o->doneUs = r.done_us;
    o->launches = r.launches;
    o->state = r.state;
    return 0;
}

extern "C" int ffb_serve_info(FfbServer* S, FfbServeInfo* o)
{
    if (!S || !o) return -1;
    std::lock_guard<std::mutex> lk(S->mu);
    o->budget = S->budget;
    o->mapBytes = S->sieved >> 4;
    o->mapMaxValue = S->sieved ? S->sieved - 1 : 0;
    o->requests = S->reqs.size();
    o->completed = S->completed;
    o->failed = S->failed;
    o->launches = S->launches;
    o->sumsRequested = S->sums_req;
    o->sumsSearched = S->sums_searched;
    o->chunks = S->chunks;
    o->textBytes = S->text_bytes;
    o->slots = S->nslots;
    o->maxQueued = S->max_queued;
    double sieve = 0;
    for (Growth& g : S->growths) {
        if (g.ms < 0 && cudaEventQuery(g.b) == cudaSuccess) cudaEventElapsedTime(&g.ms, g.a, g.b);
        if (g.ms >= 0) sieve += g.ms;
    }
    o->sieveMs = sieve;
    o->searchMs = S->search_ms;
    unsigned long long w[4] = {0, 0, 0, 0};
    for (uint32_t i = 0; i < S->nslots; ++i) cudaStreamSynchronize(S->slots[i].stream);
    if (cudaMemcpy(w, S->d_stats, sizeof w, cudaMemcpyDeviceToHost) != cudaSuccess) cudaGetLastError();
    o->stage1Probes = w[0];
    o->stage2Items = w[1];
    o->mrCandidates = w[2];
    o->mrBase2Passed = w[3];
    return 0;
}

extern "C" int ffb_serve_drain(FfbServer* S, int timeoutMs)
{
    if (!S) return -1;
    std::unique_lock<std::mutex> lk(S->mu);
    auto done = [&] { return S->completed + S->failed == S->reqs.size(); };
    if (timeoutMs < 0) {
        S->cv_drain.wait(lk, done);
        return 0;
    }
    return S->cv_drain.wait_for(lk, std::chrono::milliseconds(timeoutMs), done) ? 0 : 1;
}

extern "C" void ffb_serve_destroy(FfbServer* S)
{
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_sched.notify_all();
    if (S->sched_thr.joinable()) S->sched_thr.join();
    S->cv_done.notify_all();
    if (S->done_thr.joinable()) S->done_thr.join();
    release(S);
}
