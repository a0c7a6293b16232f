// ffb_device.cuh -- device-side arithmetic shared by the sieve and the search kernels.
//
// Bitmap layout (the reference's, reference/segmentedSieve.C:183-187, 294): byte v>>4,
// bit 0x80>>((v>>1)&7); the bit of an odd v is 1 iff v is prime; an even v shares the
// bit of v+1 and is never asked for (IsPrime answers parity first).
#pragma once

#include <cstdint>

namespace ffb {

// Error flags raised by kernels into a device word the host reads after the launch.
enum : uint32_t {
    kErrMrDomain   = 1u << 0,  // Miller-Rabin asked for n >= 2^48 (outside the exact domain)
    kErrFactorList = 1u << 1,  // divisor list of one product exceeded its fixed capacity
    kErrBadInput   = 1u << 2,  // launch arguments inconsistent (checked on the device)
};

// floor(sqrt(n)) for n < 2^62 (products here stay below 2^52).
__device__ __forceinline__ uint64_t isqrt64(uint64_t n)
{
    uint64_t r = (uint64_t)sqrt((double)n);
    while (r * r > n) --r;
    while ((r + 1) * (r + 1) <= n) ++r;
    return r;
}

// Inverse of an odd q modulo 2^64 by Newton's iteration x <- x(2 - qx); the seed
// x = q is correct to 3 bits, each step doubles the correct bits.
__device__ __forceinline__ uint64_t inv64(uint64_t q)
{
    uint64_t x = q;
#pragma unroll
    for (int i = 0; i < 5; ++i) x *= 2 - q * x;
    return x;
}

// ---------------------------------------------------------------------------------------
// Montgomery arithmetic modulo an odd n < 2^63 with R = 2^64.
// ---------------------------------------------------------------------------------------
struct Mont {
    uint64_t n;     // modulus
    uint64_t nneg;  // -n^-1 mod 2^64
    uint64_t one;   // R mod n
};

__device__ __forceinline__ Mont mont_setup(uint64_t n)
{
    Mont m;
    m.n = n;
    m.nneg = 0 - inv64(n);
    m.one = (0 - n) % n;  // 2^64 mod n
    return m;
}

// REDC(a*b): a, b < n. With T = a*b, m = (T mod R) * nneg, T + m*n is divisible by R and
// (T + m*n)/R = hi(T) + hi(m*n) + [lo(T) != 0] < 2n.
__device__ __forceinline__ uint64_t mont_mul(uint64_t a, uint64_t b, const Mont& M)
{
    uint64_t lo = a * b;
    uint64_t hi = __umul64hi(a, b);
    uint64_t m = lo * M.nneg;
    uint64_t t = hi + __umul64hi(m, M.n) + (lo != 0);
    return t >= M.n ? t - M.n : t;
}

// Deterministic Miller-Rabin with the reference's bases and thresholds
// (reference/segmentedSieve.C:354-387): bases 2,3,5,7 below 3215031751, then ,11 below
// 2152302898747, ,13 below 3474749660383, ,17 above. For odd n in [17, 2^48) the strong
// probable-prime verdicts equal the reference's (its software mulmod is exact there).
static __device__ __noinline__ bool miller_rabin(uint64_t n, uint32_t* err)
{
    if (n >= (1ull << 48)) atomicOr(err, kErrMrDomain);
    const uint32_t s = __ffsll((long long)(n - 1)) - 1;  // n-1 = d * 2^s, d odd
    const uint64_t d = (n - 1) >> s;
    const uint32_t tests = n < 3215031751ull ? 4 : n < 2152302898747ull ? 5
                         : n < 3474749660383ull ? 6 : 7;
    const Mont M = mont_setup(n);
    const uint64_t minus_one = M.n - M.one;
    const int top = 63 - __clzll((long long)d);
    const uint32_t bases[7] = {2, 3, 5, 7, 11, 13, 17};
    for (uint32_t i = 0; i < tests; ++i) {
        // base * R mod n; base <= 17 and R mod n < 2^48 keep the product below 2^53
        const uint64_t a = (uint64_t)bases[i] * M.one % n;
        uint64_t x = a;                       // left-to-right: leading bit of d consumed
        for (int bit = top - 1; bit >= 0; --bit) {
            x = mont_mul(x, x, M);
            if ((d >> bit) & 1) x = mont_mul(x, a, M);
        }
        if (x == M.one || x == minus_one) continue;
        bool ok = false;
        for (uint32_t r = 1; r < s; ++r) {
            x = mont_mul(x, x, M);
            if (x == M.one) return false;
            if (x == minus_one) { ok = true; break; }
        }
        if (!ok) return false;
    }
    return true;
}

// Prime::IsPrime (reference/segmentedSieve.C:283-296): 2 -> prime, even -> not, above the
// map -> Miller-Rabin, else the map bit.
__device__ __forceinline__ bool is_prime(const uint8_t* __restrict__ map, uint64_t bound,
                                         uint64_t n, uint32_t* err)
{
    if (n == 2) return true;
    if (!(n & 1)) return false;
    if (n > bound) return miller_rabin(n, err);
    return (__ldg(map + (n >> 4)) >> (7 - ((n >> 1) & 7))) & 1;
}

// ProductOfTermPairsHasSingleFactorPair (reference/segmentedSieve.C:419-422): an even pair
// sum always has a prime split (Goldbach); an odd one has only 2 + (i-2).
__device__ __forceinline__ bool single_pair(const uint8_t* __restrict__ map, uint64_t bound,
                                            uint64_t i, uint32_t* err)
{
    if (!(i & 1)) return true;
    return is_prime(map, bound, i - 2, err);
}

}  // namespace ffb
