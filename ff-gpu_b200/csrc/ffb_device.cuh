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

// 2^64 mod n for odd n >= 3. Above 2^33 the quotient 2^64/n is below 2^31, so the double
// division lands within one of floor(2^64/n) and one correction step fixes the remainder.
__device__ __forceinline__ uint64_t r_mod(uint64_t n)
{
    if (n < (1ull << 33)) return (0 - n) % n;
    const uint64_t q = (uint64_t)(18446744073709551616.0 / (double)n);
    uint64_t r = 0 - q * n;             // 2^64 - q*n (mod 2^64)
    if ((int64_t)r < 0) r += n;         // q was one too large
    else if (r >= n) r -= n;            // q was one too small
    return r;
}

__device__ __forceinline__ Mont mont_setup(uint64_t n)
{
    Mont m;
    m.n = n;
    m.nneg = 0 - inv64(n);
    m.one = r_mod(n);
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

// b*R mod n for a base b <= 17: below 2^48 the product is below 2^53, exact in a double,
// and the quotient (at most 17) is exact after one correction.
__device__ __forceinline__ uint64_t mont_small(uint32_t b, const Mont& M)
{
    const uint64_t x = (uint64_t)b * M.one;
    if (M.n >= (1ull << 48)) return x % M.n;
    const uint64_t q = (uint64_t)((double)x / (double)M.n);
    uint64_t r = x - q * M.n;
    if ((int64_t)r < 0) r += M.n;
    else if (r >= M.n) r -= M.n;
    return r;
}

// Bases of the reference's Miller-Rabin (reference/segmentedSieve.C:365-389) and how many of
// them it tries for n: 4 below 3215031751, 5 below 2152302898747, 6 below 3474749660383,
// else 7.
__device__ __forceinline__ uint32_t mr_base(uint32_t i)
{
    // 2, 3, 5, 7, 11, 13, 17 packed in 5-bit fields
    constexpr uint64_t kPacked = 2ull | 3ull << 5 | 5ull << 10 | 7ull << 15 | 11ull << 20 |
                                 13ull << 25 | 17ull << 30;
    return (uint32_t)(kPacked >> (5 * i)) & 31u;
}
__device__ __forceinline__ uint32_t mr_tests(uint64_t n)
{
    return n < 3215031751ull ? 4 : n < 2152302898747ull ? 5 : n < 3474749660383ull ? 6 : 7;
}

// One round of the reference's loop: is n a strong probable prime to base b? (x = b^d,
// d odd with n-1 = d*2^s; passes if x == 1 or some x^(2^r) == n-1, r < s.) A base that is a
// multiple of n gives x = 0 and fails, as in the reference. Base 2 multiplies by doubling.
__device__ __forceinline__ bool sprp(uint64_t n, uint32_t b)
{
    const uint32_t s = __ffsll((long long)(n - 1)) - 1;  // n-1 = d * 2^s, d odd
    const uint64_t d = (n - 1) >> s;
    const Mont M = mont_setup(n);
    const uint64_t minus_one = M.n - M.one;
    const int top = 63 - __clzll((long long)d);
    uint64_t x;
    if (b == 2) {
        x = M.one + M.one;
        if (x >= M.n) x -= M.n;
        for (int bit = top - 1; bit >= 0; --bit) {
            x = mont_mul(x, x, M);
            if ((d >> bit) & 1) {
                x += x;
                if (x >= M.n) x -= M.n;
            }
        }
    } else {
        const uint64_t a = mont_small(b, M);
        x = a;
        for (int bit = top - 1; bit >= 0; --bit) {
            x = mont_mul(x, x, M);
            if ((d >> bit) & 1) x = mont_mul(x, a, M);
        }
    }
    if (x == M.one || x == minus_one) return true;
    for (uint32_t r = 1; r < s; ++r) {
        x = mont_mul(x, x, M);
        if (x == M.one) return false;
        if (x == minus_one) return true;
    }
    return false;
}

// Divisibility of n by the odd primes 3..61, each an exact-division test
// n * p^-1 mod 2^64 <= (2^64-1)/p. For n > 61 a hit proves n composite, so the
// Miller-Rabin verdict (which is exact on the composites it rejects) is false without it.
__device__ __forceinline__ bool small_factor(uint64_t n)
{
    constexpr uint32_t P[17] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61};
    bool hit = false;
#pragma unroll
    for (int i = 0; i < 17; ++i) {
        uint64_t inv = P[i];
#pragma unroll
        for (int k = 0; k < 5; ++k) inv *= 2 - P[i] * inv;
        hit |= n * inv <= ~0ull / P[i];
    }
    return hit;
}

// Miller-Rabin with the reference's bases and thresholds (reference/segmentedSieve.C:
// 365-389) for one lane, written plainly (64-bit remainders in the set-up, base by base).
// For odd n in [17, 2^48) the verdicts equal the reference's (its software mulmod is exact
// there). The search calls it only for values that are almost never above the map; the
// probes that do leave the map are tested in batches (mr_rounds). This form of the callee
// measured fastest: its calls shape the kernels' register allocation even when not taken.
static __device__ __noinline__ bool miller_rabin_plain(uint64_t n, uint32_t* err)
{
    if (n >= (1ull << 48)) atomicOr(err, kErrMrDomain);
    const uint32_t s = __ffsll((long long)(n - 1)) - 1;  // n-1 = d * 2^s, d odd
    const uint64_t d = (n - 1) >> s;
    const uint32_t tests = n < 3215031751ull ? 4 : n < 2152302898747ull ? 5
                         : n < 3474749660383ull ? 6 : 7;
    Mont M;
    M.n = n;
    M.nneg = 0 - inv64(n);
    M.one = (0 - n) % n;  // 2^64 mod n
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

// The same verdict batched over a warp (mr_rounds below, all 32 lanes calling together:
// never behind a branch or a short-circuit that some lanes skip): base 2 on every candidate
// at once, then the other bases of the base-2 survivors (nearly all primes) spread one
// (survivor, base) pair per lane, so a warp pays about two base rounds instead of one per
// base whenever one of its lanes holds a prime.
static __device__ __noinline__ bool sprp_leaf(uint64_t n, uint32_t b) { return sprp(n, b); }

// Miller-Rabin rounds for the lanes with `need` (odd candidates without small factors), all
// 32 lanes calling together; one out-of-line copy keeps the calling kernel's code small. cnt (non-null on one lane only) counts [2] candidates and
// [3] base-2 survivors.
static __device__ __noinline__ bool mr_rounds(uint64_t n, bool need, int lane,
                                          unsigned long long* cnt)
{
    const uint32_t want = __ballot_sync(0xFFFFFFFFu, need);
    if (!want) return false;
    bool pp = need && sprp_leaf(n, 2);
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, pp);
    if (cnt) {
        atomicAdd(&cnt[2], (unsigned long long)__popc(want));
        atomicAdd(&cnt[3], (unsigned long long)__popc(m));
    }
    if (!m) return false;
    const uint32_t t = pp ? mr_tests(n) - 1 : 0;   // bases left for this lane's candidate
    const uint32_t per = __reduce_max_sync(0xFFFFFFFFu, t);
    const uint32_t jobs = (uint32_t)__popc(m) * per;
    uint32_t fail = 0;
    for (uint32_t j0 = 0; j0 < jobs; j0 += 32) {
        const uint32_t j = j0 + (uint32_t)lane;
        const bool live = j < jobs;
        const uint32_t c = live ? j / per : 0;       // survivor ordinal
        const uint32_t bi = live ? j - c * per : 0;  // its base index - 1
        uint32_t mm = m;
        for (uint32_t i = 0; i < c; ++i) mm &= mm - 1;
        const int src = __ffs(mm) - 1;              // lane of the c-th survivor
        const uint64_t nn = __shfl_sync(0xFFFFFFFFu, n, src);
        const uint32_t tt = __shfl_sync(0xFFFFFFFFu, t, src);
        bool bad = false;
        if (live && bi < tt) bad = !sprp_leaf(nn, mr_base(bi + 1));
        fail |= __reduce_or_sync(0xFFFFFFFFu, bad ? (1u << src) : 0u);
    }
    return pp && !((fail >> lane) & 1);
}

}  // namespace ffb
