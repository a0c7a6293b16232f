// gpu_prime.h -- host primality over a borrowed prime map, and the reference's text
// emission functions (C++ linkage, as in the reference).
//
// Replaces source/gpu_prime.h:6-25 (class GpuPrime) and the functions of
// source/m4/gpu_search_emission.cpp:34-96 (PrintOutputTags, FormatGpuSearchResult,
// GpuSearchEmit), which print to stdout.
#ifndef FFB_GPU_PRIME_H
#define FFB_GPU_PRIME_H

#include <cstdint>

#include "ffb200.h"

class GpuPrime {
public:
    typedef int Boolean;
    enum { False, True };

    // Borrows primeMap (reference layout, values 0..maxMapValue); no copy, no free.
    GpuPrime(const uint8_t* primeMap, uint64_t maxMapValue);
    ~GpuPrime();

    // n == 2 -> True; even -> False; n > maxMapValue -> Miller-Rabin with the reference's
    // bases/thresholds; else the map bit (reference/segmentedSieve.C:283-296).
    Boolean IsPrime(uint64_t n) const;
    // As in ff-gpu (source/gpu_prime.h:15) this means IsPrime(n), not "n-th prime".
    inline Boolean operator[](uint64_t n) const { return IsPrime(n); }
    inline uint64_t MaxPrimeMapValue() const { return maxPrimeMapValue_; }
    Boolean AskMillerRabin(uint64_t n) const;

private:
    const uint8_t* primeMap_;
    uint64_t maxPrimeMapValue_;
};

// " (prime)" [", "] | " (2^N)" [",   " padded as setw(3-floor(log10 N))] | [",         "]
// for one term; isLast selects the trailing separator (reference OutputTags::blanks).
void PrintOutputTags(const GpuPrime& prime, uint64_t term, bool isLast);
// One line "%7u) sum =..." for a record, to stdout.
void FormatGpuSearchResult(const GpuPrime& prime, uint32_t count, const GpuRecord& rec);
// Every non-empty slot of records[0..slotCount) in slot order, numbered from 1.
void GpuSearchEmit(const GpuPrime& prime, const GpuRecord* records, uint32_t slotCount);

#endif  // FFB_GPU_PRIME_H
