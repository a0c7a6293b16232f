// boundary_check.cpp -- a C++ caller of the library's C++ half of the boundary, as the
// reference's own harnesses call it (test/source/m4_order.cpp drives GpuSearchLaunch and
// GpuSearchEmit; source/cpu_search.cpp calls GpuPrime). Built by `make -C ff-gpu_b200 check`
// into ff-gpu_b200/bin/boundary_check and run by tests/test_boundary_cxx.py, which compares
// its output with the oracle and the reference golden.
//
//   boundary_check isprime <mapfile> <mpv>   reads n values from stdin; prints per value
//                                            "n IsPrime(n) operator[](n) AskMillerRabin(n)"
//                                            (AskMillerRabin only for odd n > 2, else -)
//                                            over a host map read from <mapfile> (CPU only)
//   boundary_check tags <mapfile> <mpv>      PrintOutputTags for the terms read from stdin,
//                                            isLast true then false, one line per term
//   boundary_check emit <sumLimit>           the prime map of `ff_sieve 5 <sumLimit>` sieved
//                                            on device 0 (ffb_sieve_map_async), the search run
//                                            through GpuSearchLaunch into GpuRecord slots, then
//                                            GpuSearchEmit over a host copy of the map (GPU)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ffb200.h"
#include "gpu_prime.h"

static std::vector<uint8_t> read_map(const char* path)
{
    std::vector<uint8_t> m;
    FILE* f = std::fopen(path, "rb");
    if (!f) return m;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    m.resize((size_t)n);
    if (std::fread(m.data(), 1, m.size(), f) != m.size()) m.clear();
    std::fclose(f);
    return m;
}

static int isprime_mode(const char* mapfile, uint64_t mpv, bool tags)
{
    const std::vector<uint8_t> map = read_map(mapfile);
    if (map.size() < ((mpv + 1 + 15) >> 4)) {
        std::fprintf(stderr, "boundary_check: map file too short\n");
        return 1;
    }
    GpuPrime prime(map.data(), mpv);
    if (prime.MaxPrimeMapValue() != mpv) return 1;
    unsigned long long n;
    while (std::scanf("%llu", &n) == 1) {
        if (tags) {
            std::printf("%llu|", n);
            PrintOutputTags(prime, n, true);
            std::printf("|");
            PrintOutputTags(prime, n, false);
            std::printf("|\n");
        } else if ((n & 1) && n > 2) {
            std::printf("%llu %d %d %d\n", n, prime.IsPrime(n), prime[n], prime.AskMillerRabin(n));
        } else {
            std::printf("%llu %d %d -\n", n, prime.IsPrime(n), prime[n]);
        }
    }
    return 0;
}

static int emit_mode(int32_t limit)
{
    FfbGeometry g;
    char hdr[2048];
    if (ffb_geometry(2, 5, limit, &g, hdr, sizeof hdr) < 0) return 1;
    const SievePoolOps* ops = SievePoolGet_sm_100a(0);
    if (!ops) {
        std::fprintf(stderr, "boundary_check: no device 0\n");
        return 1;
    }
    const uint64_t mpv = g.maxPrimeMapValue;
    const uint64_t bytes = (mpv + 1 + 15) >> 4;
    const uint64_t lo = g.sumStart | 1, hi = g.sumLimit - !(g.sumLimit & 1);
    const uint32_t slots = (uint32_t)((hi - lo) / 2 + 1);
    uint8_t* d_map = (uint8_t*)ops->alloc(0, bytes + 256);
    GpuRecord* d_rec = (GpuRecord*)ops->alloc(0, sizeof(GpuRecord) * slots);
    uint32_t* d_cnt = (uint32_t*)ops->alloc(0, 256);
    if (!d_map || !d_rec || !d_cnt) return 1;
    std::vector<uint8_t> map(bytes);
    std::vector<GpuRecord> rec(slots);
    uint32_t count = 0;
    int rc = ffb_sieve_map_async(0, mpv, d_map, nullptr);
    rc = rc || ops->memset(0, d_rec, 0, sizeof(GpuRecord) * slots) || ops->memset(0, d_cnt, 0, 4);
    rc = rc || GpuSearchLaunch(0, "nvidia", d_map, mpv, lo, hi, d_rec, d_cnt);
    // the launch is asynchronous on the legacy default stream; the copies complete it
    rc = rc || ops->copyD2H(0, map.data(), d_map, bytes) ||
         ops->copyD2H(0, rec.data(), d_rec, sizeof(GpuRecord) * slots) ||
         ops->copyD2H(0, &count, d_cnt, 4);
    uint32_t flags = 0;
    rc = rc || ffb_take_errors(0, &flags) || flags;
    ops->free(0, d_map);
    ops->free(0, d_rec);
    ops->free(0, d_cnt);
    if (rc) {
        std::fprintf(stderr, "boundary_check: device step failed\n");
        return 1;
    }
    GpuPrime prime(map.data(), mpv);
    GpuSearchEmit(prime, rec.data(), slots);
    std::fprintf(stderr, "boundary_check: %u solutions counted on the device\n", count);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc == 4 && !std::strcmp(argv[1], "isprime"))
        return isprime_mode(argv[2], std::strtoull(argv[3], nullptr, 10), false);
    if (argc == 4 && !std::strcmp(argv[1], "tags"))
        return isprime_mode(argv[2], std::strtoull(argv[3], nullptr, 10), true);
    if (argc == 3 && !std::strcmp(argv[1], "emit")) return emit_mode(std::atoi(argv[2]));
    std::fprintf(stderr, "usage: boundary_check isprime|tags <mapfile> <mpv> | emit <sumLimit>\n");
    return 2;
}
