// gpu_prime.cpp -- GpuPrime (source/gpu_prime.h:6-25) and the stdout emission functions
// of source/m4/gpu_search_emission.cpp:34-96, over the product's line formatter.
#include "gpu_prime.h"

#include <cstdio>

#include "plan.h"

GpuPrime::GpuPrime(const uint8_t* primeMap, uint64_t maxMapValue)
    : primeMap_(primeMap), maxPrimeMapValue_(maxMapValue) {}

GpuPrime::~GpuPrime() {}

GpuPrime::Boolean GpuPrime::IsPrime(uint64_t n) const
{
    if (n == 2) return True;
    if (!(n & 1)) return False;
    if (n > maxPrimeMapValue_) return AskMillerRabin(n);
    return (primeMap_[n >> 4] >> (7 - ((n >> 1) & 7))) & 1 ? True : False;
}

// Strong probable-prime test with the reference's bases and thresholds
// (reference/segmentedSieve.C:354-387); residues from exact 128-bit products.
GpuPrime::Boolean GpuPrime::AskMillerRabin(uint64_t n) const
{
    static const uint64_t bases[7] = {2, 3, 5, 7, 11, 13, 17};
    const int s = __builtin_ctzll(n - 1);
    const uint64_t d = (n - 1) >> s;
    const int tests = n < 3215031751ull ? 4 : n < 2152302898747ull ? 5 : n < 3474749660383ull ? 6 : 7;
    auto mul = [n](uint64_t a, uint64_t b) { return (uint64_t)((unsigned __int128)a * b % n); };
    for (int i = 0; i < tests; ++i) {
        uint64_t x = 1, b = bases[i] % n;
        for (uint64_t e = d; e; e >>= 1) {
            if (e & 1) x = mul(x, b);
            b = mul(b, b);
        }
        if (x == 1 || x == n - 1) continue;
        bool ok = false;
        for (int r = 1; r < s; ++r) {
            x = mul(x, x);
            if (x == 1) return False;
            if (x == n - 1) { ok = true; break; }
        }
        if (!ok) return False;
    }
    return True;
}

// PrintOutputTags (source/m4/gpu_search_emission.cpp:34-50). A term of 0 (which no search
// produces; the reference prints "(2^-inf)" for it) is treated as composite.
void PrintOutputTags(const GpuPrime& prime, uint64_t term, bool isLast)
{
    if (prime.IsPrime(term)) {
        std::fputs(isLast ? " (prime), " : " (prime)", stdout);
    } else if (term && (term & (term - 1)) == 0) {
        // " (2^N)", then "," padded to width 3 - floor(log10(N + 0.001)) (at least 1): six
        // blanks for N = 0, three for 1..9, two for 10..63
        const int n = __builtin_ctzll(term);
        std::printf(" (2^%d)", n);
        if (isLast) std::fputs(n == 0 ? ",      " : n < 10 ? ",   " : ",  ", stdout);
    } else if (isLast) {
        std::fputs(",         ", stdout);
    }
}

void FormatGpuSearchResult(const GpuPrime& prime, uint32_t count, const GpuRecord& rec)
{
    char line[ffb::kMaxLine];
    char* e = ffb::format_line(line, count, rec.sum, (uint32_t)rec.low, (uint32_t)rec.high,
                               prime.IsPrime(rec.low) != 0, prime.IsPrime(rec.high) != 0);
    std::fwrite(line, 1, (size_t)(e - line), stdout);
}

void GpuSearchEmit(const GpuPrime& prime, const GpuRecord* records, uint32_t slotCount)
{
    uint32_t ordinal = 0;
    for (uint32_t i = 0; i < slotCount; ++i) {
        if (records[i].sum == 0) continue;
        FormatGpuSearchResult(prime, ++ordinal, records[i]);
    }
}
