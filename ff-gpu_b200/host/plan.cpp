// plan.cpp -- what an `ff_sieve <sumStart> <sumLimit>` run computes before and after the
// GPU: the argument handling, the map geometry and header lines, the order in which the
// reference evaluates and prints sums, and the solution line format.
//
// The header arithmetic and the partition use the reference's integer widths and its
// double expressions operation for operation (this file is compiled without FMA
// contraction), because their results are printed or decide which sums are printed.
#include "plan.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace ffb {

uint64_t isqrt_u64(uint64_t n)
{
    if (n < 2) return n;
    uint64_t r = (uint64_t)std::sqrt((double)n);
    while (r > 0xFFFFFFFFull || r * r > n) --r;
    while (r < 0xFFFFFFFFull && (r + 1) * (r + 1) <= n) ++r;
    return r;
}

// reference/segmentedSieve.C:844-855
void parse_args(int nargs, int32_t a1, int32_t a2, uint32_t* start, uint32_t* limit)
{
    uint32_t s = 5, l = nargs == 1 ? (uint32_t)a1 : 2627u;
    if (nargs >= 2) {
        s = (uint32_t)a1 | 1u;
        l = (uint32_t)a2;
    }
    if (s < 5) s = 5;
    if (s > l) l = s;
    *start = s;
    *limit = l;
}

namespace {

constexpr uint64_t kPrimeMem = 85ull << 30;  // PRIMEMEM (reference/segmentedSieve.C:9-11)

struct Out {
    char* buf;
    size_t cap, len;
    bool ok;
    void put(const char* fmt, unsigned long long a, unsigned long long b, unsigned long long c)
    {
        int n = std::snprintf(buf + len, cap > len ? cap - len : 0, fmt, a, b, c);
        if (n < 0 || len + (size_t)n >= cap) { ok = false; return; }
        len += (size_t)n;
    }
    void put(const char* s)
    {
        size_t n = std::strlen(s);
        if (len + n >= cap) { ok = false; return; }
        std::memcpy(buf + len, s, n + 1);
        len += n;
    }
};

double est_max_prime(uint64_t n) { return (double)n * (std::log((double)n) + std::log(std::log((double)n))); }

}  // namespace

// main's sizes (reference/segmentedSieve.C:875-879) and Prime::Prime's header lines,
// including its PRIMEMEM renormalisation (reference/segmentedSieve.C:136-182).
int plan_geometry(uint32_t start, uint32_t limit, Geometry* g, char* hdr, size_t cap)
{
    std::memset(g, 0, sizeof *g);
    g->start = start;
    g->limit = limit;
    const uint32_t mgp = (limit + 1u) >> 1;
    const uint64_t product_limit = (uint64_t)mgp * mgp;
    const uint64_t prime_limit = (product_limit >> 2) + 2;
    const double xlogx = (double)mgp / std::log((double)mgp);
    const uint32_t n_arg = (uint32_t)(xlogx + 1.2762 * xlogx / std::log((double)mgp));
    g->product_limit = product_limit;

    Out o{hdr, cap, 0, true};
    if (cap) hdr[0] = 0;
    uint64_t nreq = n_arg > 1 ? n_arg : 1;
    uint64_t size = ((prime_limit > 1 ? prime_limit : 2) + 15) >> 4;
    uint64_t mpv = (size << 4) - 1;
    uint64_t est = (uint64_t)est_max_prime(nreq);
    if (mpv < est) mpv = est;
    size = (mpv + 15) >> 4;
    uint64_t req_bytes = 4 * nreq;
    uint64_t total = req_bytes + size;
    o.put("maxPrimeMapValue %llu numPrimesRequested %llu totalBytes %llu\n", mpv, nreq, total);
    if (total > kPrimeMem) {
        if (16 * kPrimeMem <= 3 * est) {
            o.put("\nThe input parameters would indicate that more memory is required. Please "
                  "adjust input parameters or Prime::maxPrimeAlloc.\n\n");
            g->too_big = true;
            return -1;
        }
        const uint64_t n2 = 2 * nreq / 5, b2 = 4 * n2;
        est = (uint64_t)est_max_prime(n2);
        if (b2 + (est + 1) / 2 > kPrimeMem) {
            nreq = ((req_bytes * kPrimeMem + total - 1) / total + 3) & ~(uint64_t)3;
            req_bytes = 4 * nreq;
            o.put("You probably should consider how badly this run is going to perform, "
                  "just sayin'.\n");
        } else {
            nreq = n2;
            req_bytes = b2;
        }
        size = kPrimeMem - req_bytes;
        total = req_bytes + size;
        mpv = (size << 4) - 1;
        o.put("numPrimesRequested %llu maxPrimeMapValue %llu totalBytes %llu\n", nreq, mpv, total);
    }
    o.put("maxPrimeMapValue %llu numPrimesRequested %llu sqrtLimit %llu\n", mpv, nreq,
          isqrt_u64(mpv));
    g->mpv = mpv;
    g->map_bytes = (mpv + 1 + 15) >> 4;
    g->nreq = nreq;
    g->pmap_sum_limit = isqrt_u64((mpv - 2) << 2) << 1;
    return o.ok ? (int)o.len : -1;
}

// One FreudenthalThreads::GenerateThreads call (reference/segmentedSieve.C:706-761):
// fronts in launch order into `front`, backs in launch order into `back`.
static bool partition(uint32_t start, uint32_t limit, uint32_t threads, std::vector<Range>& front,
                      std::vector<Range>& back)
{
    const uint32_t num = limit - start + 1u;
    if (num > 0x7FFFFFFFu) return false;  // only reachable through unsigned wrap-around
    const double delta = (double)num / (2 * threads);
    uint32_t prev1 = 0, prev2 = num;
    bool new1 = true, new2 = true;
    for (uint32_t t = 0; t < threads; ++t) {
        const uint32_t s1 = (uint32_t)(t * delta + .5);
        if (s1 > prev1) { prev1 = s1; new1 = true; }
        const uint32_t t2 = 2 * threads - t - 1;
        const uint32_t s2 = (uint32_t)(t2 * delta + .5);
        if (s2 < prev2) { prev2 = s2; new2 = true; }
        if (!(new1 && new2)) continue;
        new1 = new2 = false;
        uint32_t e1 = (uint32_t)((t + 1) * delta - .5);
        if (e1 < s1) e1 = s1;
        front.push_back({s1 + start, e1 + start});
        if (s1 < s2) {
            uint32_t e2 = (uint32_t)((t2 + 1) * delta - .5);
            if (e2 < s2) e2 = s2;
            back.push_back({s2 + start, e2 + start});
        }
    }
    return true;
}

// The emission order of ff_seg (reference/segmentedSieve.C:763-791, 905-912): per
// GenerateThreads call, the front files in launch order, then the back files in reverse.
bool plan_schedule(uint32_t start, uint32_t limit, uint64_t mpv, uint32_t threads,
                   std::vector<Range>& out)
{
    out.clear();
    if (threads == 0 || threads > 65536) return false;
    const uint64_t pmap = isqrt_u64((mpv - 2) << 2) << 1;
    uint32_t calls[2][2] = {{start, limit}, {0, 0}};
    int ncalls = 1;
    if (limit > pmap) {
        calls[0][1] = (uint32_t)pmap;
        calls[1][0] = (uint32_t)((pmap + 1) | 1);
        calls[1][1] = limit;
        ncalls = 2;
    }
    for (int c = 0; c < ncalls; ++c) {
        std::vector<Range> f, b;
        if (!partition(calls[c][0], calls[c][1], threads, f, b)) return false;
        out.insert(out.end(), f.begin(), f.end());
        out.insert(out.end(), b.rbegin(), b.rend());
    }
    return true;
}

namespace {
inline char* put_uint(char* p, uint64_t v, int width)
{
    char tmp[24];
    int n = 0;
    do { tmp[n++] = (char)('0' + v % 10); v /= 10; } while (v);
    for (int i = n; i < width; ++i) *p++ = ' ';
    while (n) *p++ = tmp[--n];
    return p;
}
inline char* put_str(char* p, const char* s)
{
    while (*s) *p++ = *s++;
    return p;
}
// OutputTags (reference/segmentedSieve.C:659-677). For a power of two 2^N the reference
// prints floor(log(t)/log(2)+.5), which is N exactly, and pads with setw(3-floor(log10 N))
// before one blank: 3 columns for N < 10, 2 for N < 100.
inline char* put_tag(char* p, uint64_t term, bool prime, bool blanks)
{
    if (prime) {
        p = put_str(p, " (prime)");
        if (blanks) p = put_str(p, ", ");
    } else if ((term & (term - 1)) == 0 && term) {
        const int n = __builtin_ctzll(term);
        p = put_str(p, " (2^");
        p = put_uint(p, (uint64_t)n, 0);
        *p++ = ')';
        if (blanks) {
            *p++ = ',';
            const int w = n < 10 ? 3 : n < 100 ? 2 : 1;
            for (int i = 1; i < w; ++i) *p++ = ' ';
            *p++ = ' ';
        }
    } else if (blanks) {
        p = put_str(p, ",         ");
    }
    return p;
}
}  // namespace

// RunIt's line (reference/segmentedSieve.C:816-819) with the global count the merge
// writes over its first 7 columns (:771-772).
char* format_line(char* p, uint32_t count, uint32_t sum, uint32_t low, uint32_t high,
                  bool low_prime, bool high_prime)
{
    p = put_uint(p, count, 7);
    p = put_str(p, ") sum =");
    p = put_uint(p, sum, 9);
    p = put_str(p, ", product =");
    p = put_uint(p, (uint64_t)low * high, 16);
    p = put_str(p, ",  low term =");
    p = put_uint(p, low, 9);
    p = put_tag(p, low, low_prime, true);
    p = put_str(p, "high term =");
    p = put_uint(p, high, 9);
    p = put_tag(p, high, high_prime, false);
    *p++ = '\n';
    return p;
}

}  // namespace ffb

extern "C" int ffb_format_line(uint32_t count, uint32_t sum, uint32_t low, uint32_t high,
                               int lowPrime, int highPrime, char* buf, size_t cap)
{
    char tmp[ffb::kMaxLine];
    char* e = ffb::format_line(tmp, count, sum, low, high, lowPrime != 0, highPrime != 0);
    const size_t n = (size_t)(e - tmp);
    if (n + 1 > cap) return -1;
    std::memcpy(buf, tmp, n);
    buf[n] = 0;
    return (int)n;
}

extern "C" int ffb_geometry(int nargs, int32_t a1, int32_t a2, FfbGeometry* out, char* hdr,
                            size_t cap)
{
    uint32_t s, l;
    ffb::parse_args(nargs, a1, a2, &s, &l);
    ffb::Geometry g;
    const int n = ffb::plan_geometry(s, l, &g, hdr, cap);
    if (out) {
        out->sumStart = s;
        out->sumLimit = l;
        out->maxPrimeMapValue = g.mpv;
        out->mapBytes = g.map_bytes;
        out->numPrimesRequested = g.nreq;
        out->pmapSumLimit = g.pmap_sum_limit;
    }
    return n;
}

extern "C" int ffb_schedule(uint32_t sumStart, uint32_t sumLimit, uint64_t mpv, uint32_t threads,
                            uint32_t* firsts, uint32_t* lasts, int cap)
{
    std::vector<ffb::Range> r;
    if (!ffb::plan_schedule(sumStart, sumLimit, mpv, threads, r)) return -1;
    if ((int)r.size() > cap) return -1;
    for (size_t i = 0; i < r.size(); ++i) {
        firsts[i] = r[i].first;
        lasts[i] = r[i].last;
    }
    return (int)r.size();
}
