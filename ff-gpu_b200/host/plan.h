// plan.h -- host-side planning of one ff_sieve run (see plan.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "ffb200.h"

namespace ffb {

constexpr int kThreads = 31;    // THREADS of the reference (reference/segmentedSieve.C:12-14)
constexpr int kMaxLine = 160;   // longest solution line is 109 bytes
constexpr uint32_t kMaxSum = 1u << 25;  // products stay below 2^48 (exact Miller-Rabin domain)

struct Geometry {
    uint32_t start, limit;
    uint64_t product_limit;
    uint64_t mpv;             // maxPrimeMapValue
    uint64_t map_bytes;       // (mpv+1+15)>>4
    uint64_t nreq;            // numPrimesRequested
    uint64_t pmap_sum_limit;  // isqrt64((mpv-2)<<2)<<1
    bool too_big;
};

struct Range {
    uint32_t first, last;  // inclusive; evaluated sums are first|1, first|1 + 2, ... <= last
};

uint64_t isqrt_u64(uint64_t n);
void parse_args(int nargs, int32_t a1, int32_t a2, uint32_t* start, uint32_t* limit);
int plan_geometry(uint32_t start, uint32_t limit, Geometry* g, char* hdr, size_t cap);
bool plan_schedule(uint32_t start, uint32_t limit, uint64_t mpv, uint32_t threads,
                   std::vector<Range>& out);
char* format_line(char* p, uint32_t count, uint32_t sum, uint32_t low, uint32_t high,
                  bool low_prime, bool high_prime);

}  // namespace ffb
