// sieve.cu -- the odd-only bitmap sieve (Prime::SegmentFill, reference/segmentedSieve.C:
// 255-270; slab contract of source/sieve_slab_kernel.h:40-107).
//
// A slab covers the values [seg_lo, seg_hi). Its bit m stands for the odd value
// (seg_lo|1) + 2m and lives at byte m>>3, mask 0x80>>(m&7) of the output (the reference's
// seg_lo-relative layout; with seg_lo == 0 this is the global map layout). Bits of values
// >= seg_hi stay 1, like the reference's untouched 0xff bytes.
//
// The marking list. For the prime map itself (every caller that sieves the map rather than
// a caller-chosen list) the list is made on the device: list_primes sieves the odd values up
// to isqrt(seg_hi - 1) in shared-memory segments and compacts each segment's primes in order
// with __ballot_sync/__popc (each lane holds one candidate bit; its slot is the warp's base
// plus the popcount of the set lanes below it), writing each prime with its Barrett constant
// and the list's regime boundaries. A caller-given list (the reference's slab/engine/pool
// calls) is uploaded instead; the standard prefix 3, 5, 7, ... of it goes through the tiled
// kernel and every other entry through sieve_generic.
//
// sieve_tiles (persistent grid over shared-memory tiles):
//   1. A tile starts as the AND of four pre-computed patterns (the odd numbers free of
//      3..13, of 17,19,23, of 29,31,37 and of 41*43), read with funnel shifts at 32-bit
//      phases advanced incrementally per word: no prime up to 43 is marked.
//   2. Small primes (p <= tile bits / 2048, at least 64 marks per lane): the "comb". The warp
//      takes one prime; at each step its 32 lanes mark the multiples f + p*(r + 32*lane + 1024*t)
//      for the same r, which lie 32p bits = p words apart: the same bit of 32 words whose
//      banks (word + p*lane) mod 32 are all different because p is odd. Every shared-memory
//      atomic of the comb is free of bank conflicts; a round whose 32 marks per lane all lie
//      in the tile runs with no bound test.
//   3. Larger primes: one thread per prime, stepping over the multiples p*k with k prime to
//      30 only (the mod-30 wheel: steps of 3p, 2p, p, 2p, p, 2p, 3p, p bits). The multiples
//      with k divisible by 3 or 5 are multiples of 3 or 5, already cleared by the patterns,
//      so 7 of every 15 odd multiples are never marked. (Without the patterns, a caller list
//      that lacks 3..43, every odd multiple is stepped.)
//   Warps take comb primes (smallest first) and groups of 32 larger primes from per-tile
//   shared counters, so a warp that finishes early takes more work.
//   4. The tile is converted to the reference bit order (brev + byte swap) and written to
//      HBM with 16-byte stores.
#include "ffb_device.cuh"
#include "ffb_internal.h"
#include "../host/plan.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace ffb {

// Device-side description of the marking list (written by list_primes or uploaded):
// primes [0, n) ascending; [ibeg, icomb) are comb primes, [icomb, n) one thread each
// (ibeg skips the pattern primes 3..43 when the patterns are applied).
struct SieveListHeader {
    uint32_t n, ibeg, icomb, pad;
};

namespace {

constexpr int kSieveThreads = 1024;
constexpr int kListThreads = 1024;
constexpr uint32_t kListSegWords = 8192;   // list_primes segment: 262,144 odd values

// Pre-sieve patterns: bit j (LSB-first) of pattern g is 1 iff the odd number 2j+1 has no
// factor among the primes of group g; each pattern repeats with the product of its primes (in
// odd numbers) and is stored with one extra period word so any 32-bit window can be read
// without wrapping. Groups 0..2 cover 3..37 (list_primes uses those three), group 3 the pair
// 41*43. A pattern costs some six instructions per 32-bit word; the comb marks of a pair of
// primes near 50 cost about as much, and above that less (the 2^21 map: patterns for 3..43
// 98.4 ms, for 3..61 99.3 ms, for 3..79 101.2 ms).
constexpr int kGroups = 4;
constexpr uint32_t kPeriod0 = 3 * 5 * 7 * 11 * 13;   // 15015
constexpr uint32_t kPeriod1 = 17 * 19 * 23;          // 7429
constexpr uint32_t kPeriod2 = 29 * 31 * 37;          // 33263
constexpr uint32_t kPeriod3 = 41 * 43;               // 1763
__host__ __device__ constexpr uint32_t words_of(uint32_t period) { return (period + 63) / 32 + 1; }
constexpr uint32_t kWords0 = words_of(kPeriod0);
constexpr uint32_t kWords1 = words_of(kPeriod1);
constexpr uint32_t kWords2 = words_of(kPeriod2);
constexpr uint32_t kWheelWords = kWords0 + kWords1 + kWords2 + words_of(kPeriod3);
constexpr int kWheelPrimes = 13;                     // 3 .. 43
constexpr uint32_t kLastPatternPrime = 43;
__device__ uint32_t g_wheel[kWheelWords];

__host__ __device__ constexpr uint32_t group_period(int g)
{
    return g == 0 ? kPeriod0 : g == 1 ? kPeriod1 : g == 2 ? kPeriod2 : kPeriod3;
}
__host__ __device__ constexpr uint32_t group_offset(int g)
{
    return g == 0 ? 0 : group_offset(g - 1) + words_of(group_period(g - 1));
}

// Steps of the mod-30 wheel in units of p bits, from the residues 1, 7, 11, 13, 17, 19, 23,
// 29 of k (2 bits each, residue index 0 in the low bits), twice over so a 32-bit rotation
// by 2 walks it.
constexpr uint32_t kWheelSteps = 0x799B799Bu;
constexpr uint32_t kPlainSteps = 0x55555555u;       // every odd multiple: step p

struct TileArgs {
    uint8_t* out;
    uint64_t out_bytes;     // relative bytes written
    uint64_t base_odd;      // value of bit 0
    uint64_t nbits;         // bits of odd values < seg_hi
    uint64_t total_bits;    // 8 * out_bytes
    const uint32_t* primes; // marking list (device)
    const uint64_t* mu;     // floor((2^64-1) / p) per prime
    const SieveListHeader* hdr;
    int wheel;              // the patterns are applied (the list holds 3..43)
    int clear_one;          // clear the bit of the value 1 (seg_lo == 0)
    uint32_t tile_words;
    uint64_t ntiles;
};

__device__ __forceinline__ uint32_t window(const uint32_t* w, uint32_t ph)
{
    return __funnelshift_r(w[ph >> 5], w[(ph >> 5) + 1], ph & 31);
}

// The 32-bit window of pattern g at phase ph, then ph advanced by `step` bits (a thread's
// next word in the tile loop): offset, period and step are compile-time constants.
template <int g, uint32_t step>
__device__ __forceinline__ uint32_t pattern_word(const uint32_t* wheel, uint32_t& ph)
{
    constexpr uint32_t period = group_period(g), off = group_offset(g), adv = step % period;
    const uint32_t x = window(wheel + off, ph);
    ph += adv;
    ph -= ph >= period ? period : 0;
    return x;
}

// ~(1 << (x & 31)) in one funnel-shift rotation
__device__ __forceinline__ uint32_t clear_mask(uint32_t x)
{
    return __funnelshift_l(0xFFFFFFFEu, 0xFFFFFFFEu, x);
}

// k0 = ceil(v / p) for odd p, v < 2^63, with mu = floor((2^64-1)/p).
__device__ __forceinline__ uint64_t ceil_div(uint64_t v, uint64_t p, uint64_t mu)
{
    uint64_t q = __umul64hi(v, mu);
    uint64_t r = v - q * p;
    while (r >= p) { r -= p; ++q; }
    return q + (r != 0);
}

__global__ void __launch_bounds__(kSieveThreads) sieve_tiles(const TileArgs A)
{
    extern __shared__ uint32_t smem[];
    uint32_t* tile = smem;
    uint32_t* wheel = smem + A.tile_words;
    __shared__ uint32_t ctr[2];
    __shared__ uint8_t adv_idx[32];   // k mod 30 -> distance to the next k prime to 30 | its index << 4
    if (A.wheel)
        for (uint32_t i = threadIdx.x; i < kWheelWords; i += blockDim.x) wheel[i] = g_wheel[i];
    if (threadIdx.x < 30) {
        const uint32_t c = threadIdx.x;
        uint32_t d = 0;
        while ((c + d) % 2 == 0 || (c + d) % 3 == 0 || (c + d) % 5 == 0) ++d;
        const uint32_t t = (c + d) % 30;
        const uint32_t idx = t == 1 ? 0 : t == 7 ? 1 : t == 11 ? 2 : t == 13 ? 3 : t == 17 ? 4
                           : t == 19 ? 5 : t == 23 ? 6 : 7;
        adv_idx[c] = (uint8_t)(d | idx << 4);
    }
    const SieveListHeader H = *A.hdr;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t tile_bits = (uint64_t)A.tile_words * 32;
    const uint64_t j0 = (A.base_odd - 1) >> 1;  // pattern index of bit 0
    const uint32_t ncomb = H.icomb - H.ibeg;
    const uint32_t nthr = H.n - H.icomb;

    for (uint64_t t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const uint64_t m0 = t * tile_bits;
        const uint64_t m1 = min(m0 + tile_bits, A.total_bits);
        const uint32_t words = (uint32_t)((m1 - m0 + 31) >> 5);
        __syncthreads();  // previous tile fully stored; patterns and tables loaded
        if (threadIdx.x == 0) { ctr[0] = 0; ctr[1] = 0; }
        // ---- 1. initial pattern ----
        {
            // the block is launched with kSieveThreads threads, so a thread's next word is
            // 32 * kSieveThreads bits on: a compile-time phase step per pattern
            const uint64_t j = j0 + m0 + 32ull * threadIdx.x;
            constexpr uint32_t adv = 32u * kSieveThreads;
            uint32_t ph0 = (uint32_t)(j % kPeriod0), ph1 = (uint32_t)(j % kPeriod1),
                     ph2 = (uint32_t)(j % kPeriod2), ph3 = (uint32_t)(j % kPeriod3);
            for (uint32_t w = threadIdx.x; w < words; w += kSieveThreads) {
                const uint64_t gm = m0 + 32ull * w;
                uint32_t x = 0xFFFFFFFFu;
                if (A.wheel) {
                    x = pattern_word<0, adv>(wheel, ph0) & pattern_word<1, adv>(wheel, ph1) &
                        pattern_word<2, adv>(wheel, ph2) & pattern_word<3, adv>(wheel, ph3);
                }
                if (gm + 32 > A.nbits) {  // bits of values >= seg_hi stay set
                    const uint64_t keep = A.nbits > gm ? A.nbits - gm : 0;
                    x |= keep >= 32 ? 0u : ~((1u << keep) - 1u);
                }
                tile[w] = x;
            }
        }
        __syncthreads();
        const uint64_t mlim = min(m1, A.nbits);
        const uint32_t rl = (uint32_t)(mlim > m0 ? mlim - m0 : 0);  // tile-relative limit
        const uint64_t V = A.base_odd + 2 * m0;                     // odd value of tile bit 0
        const uint64_t Vend = A.base_odd + 2 * mlim;                // first value past the tile
        // ---- 2. comb primes, one warp per prime (smallest first) ----
        for (;;) {
            uint32_t c = 0;
            if (lane == 0) c = atomicAdd(&ctr[0], 1u);
            c = __shfl_sync(0xFFFFFFFFu, c, 0);
            if (c >= ncomb) break;
            const uint64_t p = A.primes[H.ibeg + c];
            uint64_t k = ceil_div(V, p, A.mu[H.ibeg + c]);
            if (k < p) k = p;           // marks start at p*p
            k |= 1;                     // odd multiples only
            if (p * k >= Vend) continue;
            const uint32_t f = (uint32_t)((p * k - V) >> 1);
            const uint32_t p32 = (uint32_t)p, step = 1024u * p32;
            for (uint32_t b = f + 32u * p32 * lane; ; b += step) {
                if (!__any_sync(0xFFFFFFFFu, b < rl)) break;
                uint32_t x = b;
                if (__all_sync(0xFFFFFFFFu, b + 31u * p32 < rl)) {
                    // every lane's 32 marks lie in the tile: no bound test per mark
#pragma unroll 8
                    for (int r = 0; r < 32; ++r) {
                        atomicAnd(&tile[x >> 5], clear_mask(x));
                        x += p32;
                    }
                } else {
#pragma unroll 8
                    for (int r = 0; r < 32; ++r) {
                        if (x < rl) atomicAnd(&tile[x >> 5], clear_mask(x));
                        x += p32;
                    }
                }
            }
        }
        // ---- 3. the other primes, one thread each, 32 per warp at a time ----
        const uint32_t pat0 = A.wheel ? kWheelSteps : kPlainSteps;
        for (;;) {
            uint32_t g = 0;
            if (lane == 0) g = atomicAdd(&ctr[1], 32u);
            g = __shfl_sync(0xFFFFFFFFu, g, 0);
            if (g >= nthr) break;
            const uint32_t i = g + lane;
            if (i < nthr) {
                const uint64_t p = A.primes[H.icomb + i];
                uint64_t k = ceil_div(V, p, A.mu[H.icomb + i]);
                if (k < p) k = p;
                uint32_t pat = pat0;
                if (A.wheel) {
                    const uint32_t ai = adv_idx[(uint32_t)(k % 30)];
                    k += ai & 15;
                    pat = __funnelshift_r(pat, pat, 2 * (ai >> 4));
                } else {
                    k |= 1;
                }
                const uint64_t v = p * k;
                uint32_t x = v < Vend ? (uint32_t)((v - V) >> 1) : rl;
                const uint32_t p32 = (uint32_t)p;
                while (x < rl) {
                    atomicAnd(&tile[x >> 5], clear_mask(x));
                    x += (pat & 3) * p32;
                    pat = __funnelshift_r(pat, pat, 2);
                }
            }
        }
        __syncthreads();
        // ---- the pattern primes themselves and the value 1 ----
        if (threadIdx.x == 0 && A.base_odd <= kLastPatternPrime) {
            const uint32_t wp[kWheelPrimes] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43};
            if (A.wheel)
                for (int q = 0; q < kWheelPrimes; ++q) {
                    if (wp[q] < A.base_odd) continue;
                    const uint64_t m = (wp[q] - A.base_odd) >> 1;
                    if (m >= m0 && m < mlim) tile[(m - m0) >> 5] |= 1u << ((m - m0) & 31);
                }
            if (A.clear_one && A.base_odd == 1 && m0 == 0) tile[0] &= ~1u;  // value 1
        }
        __syncthreads();
        // ---- 4. reference bit order, 16-byte stores ----
        uint8_t* dst = A.out + (m0 >> 3);
        const uint64_t bytes = min((uint64_t)words * 4, A.out_bytes - (m0 >> 3));
        const uint32_t vec = (uint32_t)(bytes >> 4);
        for (uint32_t v = threadIdx.x; v < vec; v += blockDim.x) {
            uint4 q;
            q.x = __byte_perm(__brev(tile[4 * v + 0]), 0, 0x0123);
            q.y = __byte_perm(__brev(tile[4 * v + 1]), 0, 0x0123);
            q.z = __byte_perm(__brev(tile[4 * v + 2]), 0, 0x0123);
            q.w = __byte_perm(__brev(tile[4 * v + 3]), 0, 0x0123);
            reinterpret_cast<uint4*>(dst)[v] = q;
        }
        for (uint64_t b = (uint64_t)vec * 16 + threadIdx.x; b < bytes; b += blockDim.x) {
            const uint32_t x = __byte_perm(__brev(tile[b >> 2]), 0, 0x0123);
            dst[b] = (uint8_t)(x >> (8 * (b & 3)));
        }
    }
}

// Exclusive prefix sum of v over the block (kListThreads threads); *total gets the sum.
__device__ uint32_t block_scan(uint32_t v, uint32_t* sh, uint32_t* total)
{
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += t;
    }
    if (lane == 31) sh[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? sh[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, d);
            if (lane >= d) wi += t;
        }
        sh[lane] = wi - w;
        if (lane == 31) sh[32] = wi;
    }
    __syncthreads();
    const uint32_t r = sh[warp] + incl - v;
    *total = sh[32];
    __syncthreads();
    return r;
}

// The odd primes <= L in ascending order with their Barrett constants, and the list header
// for tiles of tile_bits bits (one block of kListThreads threads). Odd value 2j+3 is bit j.
// Level 0 (odd primes up to sqrt(L)) by trial division; level 1 sieved in shared-memory
// segments (the patterns for 3..37, then the level-0 primes from 41 marked warp-strided) and
// compacted in order with __ballot_sync/__popc. cap bounds the list (the caller's buffer).
__global__ void __launch_bounds__(kListThreads) list_primes(uint64_t L, uint32_t pcomb, uint32_t cap,
                                                            int wheel, uint32_t* primes,
                                                            uint64_t* mu, SieveListHeader* hdr,
                                                            uint32_t* err)
{
    __shared__ uint32_t seg[kListSegWords];
    __shared__ uint32_t lvl0[2048];
    __shared__ uint32_t sh[33];
    __shared__ uint32_t s_ibeg, s_icomb;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t lanes_lt = (1u << lane) - 1;
    // ---- level 0: odd primes q with q*q <= L, in order ----
    uint64_t r0 = (uint64_t)sqrt((double)L);
    while (r0 * r0 > L) --r0;
    while ((r0 + 1) * (r0 + 1) <= L) ++r0;
    const uint32_t ncand = r0 >= 3 ? (uint32_t)((r0 - 3) / 2 + 1) : 0;  // q = 2i+3 <= r0
    uint32_t n0 = 0;
    for (uint32_t base = 0; base < ncand; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool isp = false;
        if (i < ncand) {
            const uint32_t q = 2 * i + 3;
            isp = true;
            for (uint32_t d = 3; d * d <= q; d += 2)
                if (q % d == 0) { isp = false; break; }
        }
        uint32_t tot = 0;
        const uint32_t pos = block_scan(isp ? 1u : 0u, sh, &tot);
        if (isp && n0 + pos < 2048) lvl0[n0 + pos] = 2 * i + 3;
        n0 += tot;
    }
    if (n0 > 2048) {   // sqrt(L) beyond what the host admits: an empty list, flagged
        if (threadIdx.x == 0) {
            atomicOr(err, kErrBadInput);
            *hdr = SieveListHeader{0, 0, 0, 0};
        }
        return;
    }
    if (threadIdx.x == 0) { s_ibeg = 0; s_icomb = 0; }
    __syncthreads();
    // ---- level 1: the odd values 3 .. L in segments ----
    const uint64_t nbits = L >= 3 ? (L - 3) / 2 + 1 : 0;
    const uint64_t segbits = 32ull * kListSegWords;
    uint32_t total = 0;
    for (uint64_t b0 = 0; b0 < nbits; b0 += segbits) {
        const uint64_t b1 = min(b0 + segbits, nbits);
        const uint32_t nw = (uint32_t)((b1 - b0 + 31) / 32);
        // pattern init: bit b is the odd value 2(b0+b)+3, pattern index j = b0 + b + 1
        for (uint32_t w = threadIdx.x; w < kListSegWords; w += blockDim.x) {
            const uint64_t j = b0 + 32ull * w + 1;
            uint32_t x = window(g_wheel, (uint32_t)(j % kPeriod0)) &
                         window(g_wheel + kWords0, (uint32_t)(j % kPeriod1)) &
                         window(g_wheel + kWords0 + kWords1, (uint32_t)(j % kPeriod2));
            const uint64_t gb = b0 + 32ull * w;
            if (gb + 32 > b1) {
                const uint64_t keep = b1 > gb ? b1 - gb : 0;
                x &= keep >= 32 ? 0xFFFFFFFFu : (1u << keep) - 1u;
            }
            if (b0 == 0 && w < 2) {  // the pattern primes 3..37 themselves (bits 0..17)
                const uint32_t wp[11] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
                for (int q = 0; q < 11; ++q) {
                    const uint32_t bb = (wp[q] - 3) / 2;
                    if (bb / 32 == w && bb < b1) x |= 1u << (bb & 31);
                }
            }
            seg[w] = x;
        }
        __syncthreads();
        // level-0 primes from 41 on, one warp per prime, lanes strided by q
        const uint64_t vlo = 2 * b0 + 3, vhi = 2 * (b1 - 1) + 3;
        for (uint32_t k = warp; k < n0; k += nwarps) {
            const uint64_t q = lvl0[k];
            if (q <= 37) continue;
            if (q * q > vhi) break;
            uint64_t f = (vlo + q - 1) / q * q;
            if (f < q * q) f = q * q;
            if (!(f & 1)) f += q;
            for (uint64_t v = f + 2 * q * lane; v <= vhi; v += 64 * q) {
                const uint32_t bb = (uint32_t)((v - 3) / 2 - b0);
                atomicAnd(&seg[bb >> 5], clear_mask(bb));
            }
        }
        __syncthreads();
        // ordered compaction: warp w owns a contiguous run of words
        const uint32_t per = (nw + nwarps - 1) / nwarps;
        const uint32_t wa = min(warp * per, nw), wb = min(wa + per, nw);
        uint32_t cnt = 0;
        for (uint32_t w = wa + lane; w < wb; w += 32) cnt += __popc(seg[w]);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, d);
        uint32_t segtot = 0;
        uint32_t base = block_scan(lane == 0 ? cnt : 0u, sh, &segtot);
        base = __shfl_sync(0xFFFFFFFFu, base, 0) + total;
        for (uint32_t w = wa; w < wb; ++w) {
            const bool bit = (seg[w] >> lane) & 1;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, bit);
            if (bit) {
                const uint32_t pos = base + __popc(m & lanes_lt);
                const uint64_t v = 2 * (b0 + 32ull * w + lane) + 3;
                if (pos < cap) {
                    primes[pos] = (uint32_t)v;
                    mu[pos] = ~0ull / v;
                }
                if (v <= kLastPatternPrime) atomicMax(&s_ibeg, pos + 1);
                if (v <= pcomb) atomicMax(&s_icomb, pos + 1);
            }
            base += __popc(m);
        }
        total += segtot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (total > cap) atomicOr(err, kErrBadInput);
        const uint32_t n = min(total, cap);
        const uint32_t ib = wheel ? min(s_ibeg, n) : 0;
        hdr->n = n;
        hdr->ibeg = ib;
        hdr->icomb = max(min(s_icomb, n), ib);
        hdr->pad = 0;
    }
}

// One list entry handled literally (reference/segmentedSieve.C:262-268 and
// source/sieve_slab_kernel.h:82-105): first = max(p*p, ceil(seg_lo/p)*p), made odd by +p
// when even, then every i = first + 2p*t < seg_hi clears bit (i - seg_lo) >> 1.
__global__ void sieve_generic(uint32_t* out_words, uint64_t seg_lo, uint64_t seg_hi,
                              uint64_t p, uint64_t first, uint64_t nmarks)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nmarks;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = first + 2 * p * t;
        const uint64_t m = (i - seg_lo) >> 1;
        const uint64_t byte = m >> 3;
        const uint32_t mask = (0x80u >> (m & 7)) << (8 * (byte & 3));
        atomicAnd(&out_words[byte >> 2], ~mask);
    }
}

int upload_wheel()
{
    static int done_dev = -1;
    int dev = 0;
    FFB_CUDA(cudaGetDevice(&dev));
    if (done_dev == dev) return 0;
    std::vector<uint32_t> w(kWheelWords, 0);
    const uint32_t group[kGroups][5] = {{3, 5, 7, 11, 13}, {17, 19, 23}, {29, 31, 37}, {41, 43}};
    for (int g = 0; g < kGroups; ++g) {
        const uint32_t off = group_offset(g), period = group_period(g);
        for (uint32_t jj = 0; jj < words_of(period) * 32; ++jj) {
            const uint32_t v = 2 * (jj % period) + 1;
            bool keep = true;
            for (int q = 0; q < 5 && group[g][q]; ++q) keep = keep && v % group[g][q] != 0;
            if (keep) w[off + (jj >> 5)] |= 1u << (jj & 31);
        }
    }
    FFB_CUDA(cudaMemcpyToSymbol(g_wheel, w.data(), w.size() * 4));
    done_dev = dev;
    return 0;
}

}  // namespace

void host_odd_primes(uint64_t limit, uint32_t** out, uint32_t* n)
{
    std::vector<uint32_t> v;
    if (limit >= 3) {
        const uint64_t nodd = (limit - 1) / 2;  // 3, 5, ..., index j -> 2j+3
        std::vector<uint8_t> comp(nodd, 0);
        for (uint64_t j = 0; j < nodd; ++j) {
            if (comp[j]) continue;
            const uint64_t p = 2 * j + 3;
            v.push_back((uint32_t)p);
            for (uint64_t m = p * p; m <= limit; m += 2 * p) comp[(m - 3) / 2] = 1;
        }
    }
    *n = (uint32_t)v.size();
    *out = (uint32_t*)std::malloc(sizeof(uint32_t) * (v.size() + 1));
    std::copy(v.begin(), v.end(), *out);
}

// Host-side analysis of one sieve request: the tiled kernel's arguments (device table
// pointers filled in by the caller), its launch shape, the list (for a caller list) or the
// device list's parameters, and the list entries that go through sieve_generic.
struct SieveHost {
    TileArgs T;
    size_t smem = 0;
    unsigned blocks = 0;
    bool tiles = false;
    bool device_list = false;   // list_primes makes the list on the device
    uint64_t list_limit = 0;    // device list: odd primes <= list_limit
    uint32_t list_cap = 0;      // device list: capacity of the buffers
    uint32_t pcomb = 0;         // largest comb prime
    SieveListHeader hdr{};      // caller list: uploaded header
    std::vector<uint64_t> mu;
    std::vector<uint32_t> list;
    struct Gen {
        uint64_t p, first, nmarks;
        unsigned grid;
    };
    std::vector<Gen> gen;
    // device layout of the table: [header 16 B][mu: 8*cap][primes: 4*cap]
    size_t table_bytes() const
    {
        const size_t cap = device_list ? list_cap : std::max<size_t>(list.size(), 1);
        return 16 + 12 * cap + 16;
    }
};

namespace {

// pi(x) < 1.25506 x / ln x for x > 1 (Rosser and Schoenfeld), plus a margin
uint32_t prime_count_bound(uint64_t x)
{
    if (x < 100) return 32;
    return (uint32_t)(1.25506 * (double)x / std::log((double)x)) + 64;
}

int analyse(const SieveArgs& a, int sms, SieveHost& H)
{
    if (upload_wheel()) return -1;
    const uint64_t out_bytes = (a.seg_hi - a.seg_lo + 15) >> 4;
    if (((uintptr_t)a.out & 15) != 0) {
        std::fprintf(stderr, "ffb: sieve output must be 16-byte aligned\n");
        return -1;
    }
    uint32_t tile_bytes = a.tile_bytes ? a.tile_bytes : 216 * 1024;
    tile_bytes = (tile_bytes + 15) & ~15u;
    TileArgs& T = H.T;
    T.tile_words = tile_bytes / 4;
    const uint64_t tile_bits = (uint64_t)T.tile_words * 32;
    // comb primes: at least 2048 multiples per tile (64 per lane)
    H.pcomb = (uint32_t)std::min<uint64_t>(tile_bits / 2048, 1u << 20);
    int wheel = 1;
    if (a.true_map) {
        // the true map: odd primes p with p*p < seg_hi, made on the device
        H.device_list = true;
        H.list_limit = a.seg_hi > 1 ? isqrt_u64(a.seg_hi - 1) : 0;
        // list_primes finds the primes up to sqrt(list_limit) by trial division into a
        // 2048-entry table: list_limit stays below 17,881^2 (the 2048th odd prime is 17,881)
        if (H.list_limit >= 17881ull * 17881ull) {
            std::fprintf(stderr, "ffb: prime map up to %llu is beyond the supported size\n",
                         (unsigned long long)(a.seg_hi - 1));
            return -1;
        }
        H.list_cap = prime_count_bound(H.list_limit);
    } else {
        const uint32_t* h = a.h_primes;
        // longest prefix (after an optional leading 2) equal to 3,5,7,... (checked up to 2^27)
        const uint32_t off = (a.nprimes && h[0] == 2) ? 1 : 0;
        uint32_t std_n = 0;
        if (off < a.nprimes) {
            uint32_t top = 0;
            for (uint32_t i = off; i < a.nprimes; ++i) top = h[i] > top ? h[i] : top;
            if (top > (1u << 27)) top = 1u << 27;
            uint32_t* pr = nullptr;
            uint32_t npr = 0;
            host_odd_primes(top, &pr, &npr);
            while (off + std_n < a.nprimes && std_n < npr && h[off + std_n] == pr[std_n]) ++std_n;
            std::free(pr);
        }
        // primes of the standard prefix with p*p < seg_hi mark something
        uint32_t iend = 0;
        while (iend < std_n && (uint64_t)h[off + iend] * h[off + iend] < a.seg_hi) ++iend;
        wheel = std_n >= kWheelPrimes;  // the patterns need 3..43 in the list
        H.list.assign(h + off, h + off + iend);
        H.mu.resize(iend);
        for (uint32_t i = 0; i < iend; ++i) H.mu[i] = ~0ull / h[off + i];   // Barrett constants
        uint32_t ibeg = wheel ? kWheelPrimes : 0;
        if (ibeg > iend) ibeg = iend;
        uint32_t icomb = ibeg;
        while (icomb < iend && H.list[icomb] <= H.pcomb) ++icomb;
        H.hdr = {iend, ibeg, icomb, 0};
        // every entry outside the standard prefix, literally
        for (uint32_t i = 0; i < a.nprimes; ++i) {
            if (i >= off && i < off + std_n) continue;
            const uint64_t p = h[i];
            if (p == 0) continue;  // the reference divides by p here; nothing to mark
            const uint64_t pp = p * p;
            if (pp >= a.seg_hi) continue;
            uint64_t first = (a.seg_lo + p - 1) / p * p;
            if (first < pp) first = pp;
            if (!(first & 1)) first += p;
            if (first >= a.seg_hi) continue;
            const uint64_t nmarks = (a.seg_hi - first + 2 * p - 1) / (2 * p);
            uint64_t g = (nmarks + 255) / 256;
            if (g > (uint64_t)sms * 16) g = (uint64_t)sms * 16;
            H.gen.push_back({p, first, nmarks, (unsigned)g});
        }
    }
    T.out = a.out;
    T.out_bytes = out_bytes;
    T.base_odd = a.seg_lo | 1;
    T.nbits = a.seg_hi > T.base_odd ? (a.seg_hi - T.base_odd + 1) / 2 : 0;
    T.total_bits = out_bytes * 8;
    T.primes = nullptr;
    T.mu = nullptr;
    T.hdr = nullptr;
    T.wheel = wheel;
    T.clear_one = a.clear_one && a.seg_lo == 0;
    T.ntiles = (T.total_bits + tile_bits - 1) / tile_bits;
    H.smem = 4ull * (T.tile_words + kWheelWords);
    FFB_CUDA(cudaFuncSetAttribute(sieve_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)H.smem));
    int per_sm = 0;
    FFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sieve_tiles, kSieveThreads, H.smem));
    if (per_sm < 1) {
        std::fprintf(stderr, "ffb: sieve tile of %u bytes does not fit on an SM\n", tile_bytes);
        return -1;
    }
    uint64_t blocks = (uint64_t)sms * per_sm;
    if (blocks > T.ntiles) blocks = T.ntiles;
    H.blocks = (unsigned)blocks;
    H.tiles = T.ntiles > 0;
    return 0;
}

// Points the tile arguments at a table laid out as SieveHost::table_bytes() describes.
void bind_table(SieveHost& H, uint8_t* table)
{
    const size_t cap = H.device_list ? H.list_cap : std::max<size_t>(H.list.size(), 1);
    H.T.hdr = reinterpret_cast<const SieveListHeader*>(table);
    H.T.mu = reinterpret_cast<const uint64_t*>(table + 16);
    H.T.primes = reinterpret_cast<const uint32_t*>(table + 16 + 8 * cap);
}

// Fills a caller list's table (header, constants, primes) with stream-ordered copies.
int upload_table(const SieveHost& H, uint8_t* table, cudaStream_t stream)
{
    const size_t cap = std::max<size_t>(H.list.size(), 1);
    FFB_CUDA(cudaMemcpyAsync(table, &H.hdr, sizeof(SieveListHeader), cudaMemcpyHostToDevice, stream));
    if (!H.list.empty()) {
        FFB_CUDA(cudaMemcpyAsync(table + 16, H.mu.data(), 8 * H.mu.size(), cudaMemcpyHostToDevice, stream));
        FFB_CUDA(cudaMemcpyAsync(table + 16 + 8 * cap, H.list.data(), 4 * H.list.size(),
                                 cudaMemcpyHostToDevice, stream));
    }
    return 0;
}

int enqueue(const SieveHost& H, const SieveArgs& a, uint32_t* err, cudaStream_t stream)
{
    if (H.tiles) {
        if (H.device_list) {
            uint8_t* table = (uint8_t*)H.T.hdr;
            list_primes<<<1, kListThreads, 0, stream>>>(
                H.list_limit, H.pcomb, H.list_cap, H.T.wheel, (uint32_t*)H.T.primes,
                (uint64_t*)H.T.mu, (SieveListHeader*)table, err);
            FFB_CUDA(cudaGetLastError());
        }
        sieve_tiles<<<H.blocks, kSieveThreads, H.smem, stream>>>(H.T);
        FFB_CUDA(cudaGetLastError());
    }
    for (const SieveHost::Gen& g : H.gen) {
        sieve_generic<<<g.grid, 256, 0, stream>>>((uint32_t*)a.out, a.seg_lo, a.seg_hi, g.p,
                                                  g.first, g.nmarks);
        FFB_CUDA(cudaGetLastError());
    }
    return 0;
}

}  // namespace

int launch_sieve(const SieveArgs& a, int sms, uint32_t* err, cudaStream_t stream)
{
    if (a.seg_hi <= a.seg_lo) return 0;
    SieveHost H;
    if (analyse(a, sms, H)) return -1;
    // the marking table in stream-ordered scratch
    uint8_t* table = nullptr;
    FFB_CUDA(cudaMallocAsync((void**)&table, H.table_bytes(), stream));
    bind_table(H, table);
    int rc = 0;
    if (!H.device_list && upload_table(H, table, stream)) rc = -1;
    // (copies from pageable host memory are staged before cudaMemcpyAsync returns, so the
    // host vectors may go out of scope here)
    if (!rc) rc = enqueue(H, a, err, stream);
    cudaFreeAsync(table, stream);
    return rc;
}

// A sieve prepared once and launched many times (the device table stays allocated):
// enqueue_sieve_plan only launches kernels, so it can be captured in a CUDA graph.
struct SievePlan {
    SieveHost H;
    SieveArgs a;
    uint32_t* err = nullptr;
    uint8_t* table = nullptr;
};

SievePlan* create_sieve_plan(const SieveArgs& a, int sms, uint32_t* err)
{
    SievePlan* P = new SievePlan;
    P->a = a;
    P->err = err;
    if (a.seg_hi > a.seg_lo && analyse(a, sms, P->H)) {
        delete P;
        return nullptr;
    }
    if (cudaMalloc(&P->table, P->H.table_bytes()) != cudaSuccess) {
        cudaGetLastError();
        delete P;
        return nullptr;
    }
    bind_table(P->H, P->table);
    if (!P->H.device_list && (upload_table(P->H, P->table, 0) || cudaStreamSynchronize(0) != cudaSuccess)) {
        cudaFree(P->table);
        delete P;
        return nullptr;
    }
    return P;
}

int enqueue_sieve_plan(const SievePlan* P, cudaStream_t stream)
{
    if (P->a.seg_hi <= P->a.seg_lo) return 0;
    return enqueue(P->H, P->a, P->err, stream);
}

void destroy_sieve_plan(SievePlan* P)
{
    if (!P) return;
    if (P->table) cudaFree(P->table);
    delete P;
}

}  // namespace ffb
