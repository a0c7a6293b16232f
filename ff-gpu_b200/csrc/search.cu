// search.cu -- the per-sum Freudenthal search (reference/segmentedSieve.C:419-639, 800-823).
//
// Parallel structure (sm_100a, SIMT integer code):
//   * A persistent grid; each warp (or group of warps) pulls chunks of consecutive odd sums
//     from a device counter, largest sums first (their cost grows with the sum, so big ones
//     start early).
//   * Lane-parallel over up to 32 sums per warp: Sammy's first statement (the RunIt filter)
//     and the Power2Prime phase. A sum still open after that (at most one valid split so
//     far) is a "survivor".
//   * Warp-cooperative per survivor: lanes enumerate the Power2Odd / Power2Even splits
//     (k, o) in parallel. The verdict of the reference depends only on WHETHER exactly one
//     split is valid (and then on that split), not on the order the splits are visited, so
//     the order is free and the warp stops as soon as two valid splits are seen.
//   * Rare, expensive work is deferred through per-warp shared-memory queues so lanes stay
//     converged: stage 0 (every split) runs the divisibility filters and the pair probe
//     o + b*2^k - 2; stage 1 (about one split in seven) probes 2^k + o*b - 2; stage 2 (about
//     one split in sixty) runs AllButOne... on the split's product. Both probes read random
//     sectors of the map for all but the smallest k.
//   * AllButOne... is evaluated from the factorisations of o and b (both below the sum, read
//     from a smallest-prime-factor table) instead of the reference's trial-division walk over
//     all primes: the pairs that walk tests are exactly those of the odd divisors up to the
//     square-root limit and their 2^k multiples, which an odometer over the exponents
//     enumerates with no divisor list.
//   * Launch shapes (the candidates the batch's autotuner times): 4, 8 or 16 warps a block;
//     16, 32 or 64 sums per pull of the work counter (a compile-time parameter, so the
//     one-warp-per-sum kernel carries no extra loop); or 2 or 4 warps sharing one sum
//     (search_kernel_group), each enumerating every 2nd or 4th block of splits.
#include "ffb200.h"
#include "ffb_device.cuh"
#include "ffb_internal.h"

namespace ffb {
namespace {

#ifndef FFB_SEARCH_WARPS_PER_SM
#define FFB_SEARCH_WARPS_PER_SM 32
#endif
// Resident warps per SM the kernels' register budget is set for (64 registers a thread at 32
// warps): the search waits on map reads, and more resident warps beat fewer spills.
constexpr int kWarpsPerSm = FFB_SEARCH_WARPS_PER_SM;
constexpr int kQueue = 64;       // per-warp queue capacity (entries)
#ifndef FFB_DRAIN_A
#define FFB_DRAIN_A 32
#endif
#ifndef FFB_DRAIN_B
#define FFB_DRAIN_B 32
#endif
// Queue sizes at which the map-only kernels run stage 1 and stage 2 (at most 32 each, so a
// queue never passes 63 entries). Full warps win: running stage 2 at 16, 8 or 4 queued items
// (a sum's rejection found sooner, fewer lanes busy) took the 2^21 search from 199 ms to 244,
// 304 and 377 ms, and stage 1 at 16 as well to 262 ms.
constexpr uint32_t kDrainA = FFB_DRAIN_A, kDrainB = FFB_DRAIN_B;
constexpr int kMaxDiv = 64;      // divisor list of one AllButOne... call (Miller-Rabin variant)

// Stage 2 works in a per-lane scratch of shared memory (no local memory): word j of a lane
// lies at [32 j + lane] of its warp's area, so a lane always reads its own bank.
//   words 0 .. kFacSlots-1    the product's prime powers, ascending, q | e << 27 (the terms
//                             are below 2^25, so q < 2^27 and e < 32)
//   words kFacSlots ..        the odometer's partial divisors Sd[0..n] in all_but_one, and
//                             the factors of the second term while the product is factored
// A product below 2^50 has at most 12 distinct odd primes (3*5*...*43 > 2^50); one slot more
// shows an overflow, which is reported as kErrFactorList.
constexpr int kFacSlots = 13;
constexpr int kSdSlots = 13;
constexpr uint32_t kWarpScratchWords = 32 * (kFacSlots + kSdSlots);
constexpr uint32_t kWarpScratchBytes = 4 * kWarpScratchWords;

__device__ __forceinline__ uint32_t* lane_scratch()
{
    extern __shared__ uint32_t search_scratch[];
    return search_scratch + (threadIdx.x >> 5) * kWarpScratchWords + (threadIdx.x & 31);
}

__device__ __forceinline__ uint32_t fac_word(uint32_t q, uint32_t e) { return q | e << 27; }
__device__ __forceinline__ uint32_t fac_q(uint32_t w) { return w & 0x07FFFFFFu; }
__device__ __forceinline__ uint32_t fac_e(uint32_t w) { return w >> 27; }

// A product's factorisation in a lane's scratch: n distinct primes (n > kFacSlots: overflow).
struct Fac {
    uint32_t* w;
    int n;
    __device__ uint32_t q(int i) const { return fac_q(w[32 * i]); }
    __device__ uint32_t e(int i) const { return fac_e(w[32 * i]); }
};

// Prime::IsPrime for the search (reference/segmentedSieve.C:283-296), for the values that
// are (almost) always in the map: terms below the sum, cofactors below 2^32. The map-only
// variant is launched only when the map reaches every value the search can ask about, and
// the probes that can leave the map in the Miller-Rabin variant go through pair_class and
// the batched test instead; so the per-lane Miller-Rabin here is the plain form, which
// keeps the register allocation of both kernels at their best measured.
template <bool kMR>
__device__ __forceinline__ bool isp(const SearchArgs& A, uint64_t n)
{
    if (n == 2) return true;
    if (!(n & 1)) return false;
    if (n > A.bound) {
        return miller_rabin_plain(n, A.err);
    }
    return (__ldg(A.map + (n >> 4)) >> (7 - ((n >> 1) & 7))) & 1;
}

// ProductOfTermPairsHasSingleFactorPair (reference/segmentedSieve.C:419-422).
template <bool kMR>
__device__ __forceinline__ bool pair1(const SearchArgs& A, uint64_t i)
{
    if (!(i & 1)) return true;
    return isp<kMR>(A, i - 2);
}

// A probe above the map: 0 when it has an odd prime factor below 64 (composite), else 2
// (Miller-Rabin decides). Out of line: several call sites, taken only above the map.
__device__ __noinline__ int above_map_class(uint64_t n, uint32_t* err)
{
    if (n >= (1ull << 48)) atomicOr(err, kErrMrDomain);
    return n > 61 && small_factor(n) ? 0 : 2;
}

// single_pair(i) as far as it is decided without Miller-Rabin: 0 false, 1 true, 2 the probe
// i - 2 lies above the map and has no factor below 64 (Miller-Rabin decides).
__device__ __forceinline__ int pair_class(const SearchArgs& A, uint64_t i)
{
    if (!(i & 1)) return 1;
    const uint64_t n = i - 2;
    if (n <= A.bound) return (__ldg(A.map + (n >> 4)) >> (7 - ((n >> 1) & 7))) & 1;
    return above_map_class(n, A.err);
}

// Ascending prime factorisation of an odd x < 2^32: by the smallest-prime-factor table when
// x lies inside it, else by the exact-division table with the cofactor's primality read from
// the bitmap after every factor found. put(q, e) receives the prime powers in ascending order.
template <bool kMR, class Put>
__device__ __forceinline__ void factor_odd(uint32_t x, const SearchArgs& A, Put&& put)
{
    uint32_t n = x;
    if (n <= 1) return;
    if (n < A.spf_limit) {
        // the smallest-prime-factor table: one lookup per distinct prime factor, and the
        // cofactor's primality from the same table
        for (;;) {
            const uint32_t idx = __ldg(A.spf + (n >> 1));
            if (idx == 0xFFFFu) { put(n, 1u); return; }
            const TDiv t = A.tdiv[idx];
            uint32_t ex = 0, y = n * t.inv;
            do { n = y; ++ex; y = n * t.inv; } while (y <= t.lim);
            put(t.p, ex);
            if (n == 1) return;
        }
    }
    if (isp<kMR>(A, n)) { put(n, 1u); return; }
    for (uint32_t i = 0; i < A.ntdiv; ++i) {
        const TDiv t = A.tdiv[i];
        if ((uint64_t)t.p * t.p > n) break;
        uint32_t y = n * t.inv;
        if (y <= t.lim) {
            uint32_t ex = 0;
            do { n = y; ++ex; y = n * t.inv; } while (y <= t.lim);
            put(t.p, ex);
            if (n == 1) return;
            if (isp<kMR>(A, n)) { put(n, 1u); return; }
        }
    }
    if (n > 1) put(n, 1u);
}

// The factorisation of a*b (a, b odd) into the lane's scratch L: b's prime powers first go
// to the odometer words, then a's are merged with them on the fly (both lists ascend).
template <bool kMR>
__device__ __forceinline__ Fac factor_product(uint32_t a, uint32_t b, uint32_t* L, const SearchArgs& A)
{
    uint32_t* fb = L + 32 * kFacSlots;
    int nb = 0;
    if (b > 1)
        factor_odd<kMR>(b, A, [&](uint32_t q, uint32_t e) {
            if (nb < kSdSlots) fb[32 * nb] = fac_word(q, e);
            ++nb;
        });
    if (nb > kSdSlots) nb = kSdSlots;  // (b < 2^25 has at most 7 distinct odd primes)
    int j = 0, n = 0;
    auto put = [&](uint32_t w) {
        if (n < kFacSlots) L[32 * n] = w;
        ++n;
    };
    factor_odd<kMR>(a, A, [&](uint32_t q, uint32_t e) {
        for (; j < nb && fac_q(fb[32 * j]) < q; ++j) put(fb[32 * j]);
        if (j < nb && fac_q(fb[32 * j]) == q) e += fac_e(fb[32 * j++]);
        put(fac_word(q, e));
    });
    for (; j < nb; ++j) put(fb[32 * j]);
    return Fac{L, n};
}

// x / d for an odd d that divides x: x times the inverse of d modulo 2^64 (Newton's
// iteration from the seed (3d) xor 2, which is correct to 5 bits; four steps give 80).
__device__ __forceinline__ uint64_t exact_quotient(uint64_t x, uint32_t d)
{
    uint64_t v = (3ull * d) ^ 2;
#pragma unroll
    for (int i = 0; i < 4; ++i) v *= 2 - (uint64_t)d * v;
    return x * v;
}

// AllButOneProductOfTermPairsOfSumOfFactorPairsHasSingleFactorPair
// (reference/segmentedSieve.C:424-477). The reference walks trial divisors and keeps the
// divisors found in factors[]; the pairs it tests are exactly (d, P/d) for the odd divisors
// 1 < d <= lim of oddProduct and (2^k d, P/(2^k d)) for the odd divisors d with 2^k d <= lim
// (lim = isqrt(P), P = oddProduct * 2^k): its skip over sorted runs (:451) and its early
// breaks only leave out divisors above lim. The verdict is "exactly one of those pairs is not
// single", and the reference returns early only once two are found, so the order of the
// tests does not matter. Here the odd divisors <= lim are enumerated from the factorisation
// with an odometer over the exponents (digit i counts the power of factor i, 5 bits each; a
// digit that cannot grow without passing lim is reset and the next one grows), keeping per
// digit the divisor made of the digits from i up; the cofactor oddProduct/d is an exact
// division by d's inverse modulo 2^64. No divisor list is stored (the partial divisors sit
// in the lane's shared scratch). Inlined: as an out-of-line call its caller saved and restored
// some 500 bytes of registers per thread around it (2^21 job: 207 ms inlined, 222 ms not).
template <bool kMR>
__device__ __forceinline__ bool all_but_one(uint32_t k, uint64_t odd_product, const Fac f,
                                            const SearchArgs& A)
{
    const uint64_t P = odd_product << k;
    const uint64_t lim = isqrt64(P);
    uint32_t nm = 0;
    if ((1ull << k) <= lim) nm += !pair1<kMR>(A, (1ull << k) + odd_product);
    const int n = f.n;
    if (n > 12) {   // 12 digits of 5 bits fill the odometer; products < 2^50 have at most 12
        atomicOr(A.err, kErrFactorList);
        return false;
    }
    uint32_t* Sd = f.w + 32 * kFacSlots;   // Sd[j] at Sd[32 j]: the lane's odometer words
    uint64_t ex = 0;
    for (int j = 0; j <= n; ++j) Sd[32 * j] = 1;
    for (;;) {
        int i = 0;
        uint32_t q = 0;
        for (; i < n; ++i) {
            const uint32_t w = f.w[32 * i];
            q = fac_q(w);
            const uint32_t e = fac_e(w), a = (uint32_t)(ex >> (5 * i)) & 31;
            if (a < e && (uint64_t)Sd[32 * i] * q <= lim) break;
            ex &= ~(31ull << (5 * i));
            Sd[32 * i] = Sd[32 * (i + 1)];
        }
        if (i == n) break;
        ex += 1ull << (5 * i);
        const uint32_t d = Sd[32 * i] * q;
        for (int j = 0; j <= i; ++j) Sd[32 * j] = d;
        const uint64_t c = exact_quotient(odd_product, d);
        if ((nm += !pair1<kMR>(A, d + (c << k))) > 1) return false;
        if (((uint64_t)d << k) <= lim && (nm += !pair1<kMR>(A, ((uint64_t)d << k) + c)) > 1)
            return false;
    }
    return nm == 1;
}

// all_but_one for the Miller-Rabin variant: the same divisor pairs in the same order, but a
// pair sum whose probe lies above the map (and has no small factor) is appended to pend[]
// instead of being tested here, so that the warp can test them 32 at a time. Returns the
// count of pairs already known not to be single (2 once the verdict is "no"); the verdict is
// "yes" iff that count plus the pending probes found composite is exactly 1 (the order of the
// tests does not change it). *np receives the number of pending pair sums.
__device__ __noinline__ uint32_t all_but_one_defer(uint32_t k, uint64_t odd_product, const Fac f,
                                                   const SearchArgs& A, uint64_t* pend,
                                                   uint32_t* np)
{
    const uint64_t P = odd_product << k;
    const uint64_t lim = isqrt64(P);
    uint64_t F[kMaxDiv], C[kMaxDiv];
    uint32_t nf = 0, npend = 0, nm = 0, nd = 0;
    *np = 0;
    if (f.n > kFacSlots - 1) {   // more primes than the scratch holds: never for terms < 2^25
        atomicOr(A.err, kErrFactorList);
        return 2;
    }
    // counts a pair sum: 0 not single, 1 single, 2 pending; returns true once nm > 1
    auto visit = [&](uint64_t v) {
        const int c = pair_class(A, v);
        if (c == 2) pend[nd++] = v;
        else nm += c == 0;
        return nm > 1;
    };
    F[0] = 1ull << k;
    C[0] = odd_product;
    if (F[0] <= lim) {
        visit(F[0] + C[0]);
        nf = 1;
    }
    int idx = 0;
    bool first = true;  // the reference tries 3 before its first IsPrime(testProduct)
    for (;;) {
        uint64_t q;
        uint32_t e;
        if (first) {
            first = false;
            if (f.n > 0 && f.q(0) == 3) { q = 3; e = f.e(0); idx = 1; }
            else continue;
        } else {
            if (idx >= f.n) break;                                   // testProduct == 1
            q = f.q(idx);
            e = f.e(idx);
            if (idx == f.n - 1 && e == 1 && q > lim) break;          // prime cofactor > limit
            ++idx;
        }
        const uint64_t qi = inv64(q);
        uint64_t tf = q, tfi = qi;
        for (uint32_t j = 0; j < e; ++j) {
            if (tf <= lim) {
                const uint64_t ctf = (odd_product * tfi) << k;     // P / tf, exact
                if (visit(tf + ctf)) return 2;
                if (nf + npend >= kMaxDiv) { atomicOr(A.err, kErrFactorList); return 2; }
                F[nf + npend] = tf;
                C[nf + npend] = ctf;
                ++npend;
                for (uint32_t g = 0; g < nf; ++g) {
                    const uint64_t m = F[g] * tf;
                    if (m <= lim) {
                        const uint64_t cm = C[g] * tfi;              // C[g] / tf, exact
                        if (visit(m + cm)) return 2;
                        if (nf + npend >= kMaxDiv) { atomicOr(A.err, kErrFactorList); return 2; }
                        F[nf + npend] = m;
                        C[nf + npend] = cm;
                        ++npend;
                    } else {
                        // skip the rest of this ascending run of F (reference :451)
                        for (const uint64_t v = F[g]; g + 1 < nf && v <= F[g + 1]; ++g) {}
                    }
                }
            }
            tf *= q;
            tfi *= qi;
        }
        nf += npend;
        npend = 0;
    }
    *np = nd;
    return nm;
}

// Split encoding in the queues: bits 0..4 k, bit 5 composite (Power2Composite item: the odd
// term is sum - 2^k), bits 6..31 the odd part o of the even term (o < 2^26).
__device__ __forceinline__ uint32_t enc(uint32_t k, uint32_t o, bool comp)
{
    return k | (comp ? 32u : 0u) | (o << 6);
}

// The terms of a stage-2 item and the factorisation of their odd product (in the lane's
// scratch). Power2Composite items (bit 5) pair 2^k with the odd term s - 2^k.
template <bool kMR>
__device__ __forceinline__ Fac stage2_terms(uint32_t item, uint32_t s, const SearchArgs& A,
                                            uint32_t* ta, uint32_t* tb, uint64_t* odd_product)
{
    const uint32_t k = item & 31;
    uint32_t* L = lane_scratch();
    if (item & 32) {
        const uint32_t odd = s - (1u << k);
        *odd_product = odd;
        *ta = 1u << k;
        *tb = odd;
        return factor_product<kMR>(odd, 1, L, A);
    }
    const uint32_t o = item >> 6;
    const uint32_t even = o << k, b = s - even;
    *odd_product = (uint64_t)o * b;
    *ta = even;
    *tb = b;
    return factor_product<kMR>(o, b, L, A);
}

// Stage 2: the split's AllButOne... verdict (DoesPeterKnow's last step, or Power2Composite).
template <bool kMR>
__device__ bool stage2(uint32_t item, uint32_t s, const SearchArgs& A, uint32_t* ta, uint32_t* tb)
{
    uint64_t odd_product;
    const Fac f = stage2_terms<kMR>(item, s, A, ta, tb, &odd_product);
    return all_but_one<kMR>(item & 31, odd_product, f, A);
}

// Stage 2 of the Miller-Rabin variant: the factorisation and the divisor pairs, with the
// pair probes above the map left in pend[] (see all_but_one_defer).
__device__ uint32_t stage2_defer(uint32_t item, uint32_t s, const SearchArgs& A, uint32_t* ta,
                                 uint32_t* tb, uint64_t* pend, uint32_t* np)
{
    uint64_t odd_product;
    const Fac f = stage2_terms<true>(item, s, A, ta, tb, &odd_product);
    return all_but_one_defer(item & 31, odd_product, f, A, pend, np);
}

// Stage 1: the pair sum 2^k + o*b whose probe 2^k + o*b - 2 is DoesPeterKnow's first test.
__device__ __forceinline__ uint64_t stage1_value(uint32_t item, uint32_t s)
{
    const uint32_t k = item & 31, o = item >> 6;
    const uint32_t b = s - (o << k);
    return (1ull << k) + (uint64_t)o * b;
}

// Per-warp queues of pending split items (shared memory). With the Miller-Rabin variant
// a third queue holds the items whose probe lies above the map and survived the small-prime
// test, so that Miller-Rabin always runs on 32 candidates at once. Each queue holds at most
// 127 items: before any stage pushes, every queue holds fewer than 32 (settle_mr below),
// a stage pushes at most 32 items in all, and a drain never outputs more than it takes,
// so the total stays below 128.
template <bool kMR>
struct WarpQ {
    static constexpr int kCap = kMR ? 128 : kQueue;
    uint32_t a[kCap];
    uint32_t b[kCap];
    uint32_t c[kMR ? kCap : 1];
    uint64_t probe[kMR ? 32 : 1];  // stage-2 probes handed to the warp's Miller-Rabin
};

// Appends the items of the lanes with `pred` to q[n..]; returns the new size (uniform).
__device__ __forceinline__ uint32_t push(uint32_t* q, uint32_t n, bool pred, uint32_t item, int lane)
{
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, pred);
    if (pred) q[n + __popc(m & ((1u << lane) - 1))] = item;
    __syncwarp();
    return n + __popc(m);
}

struct SumState {
    uint32_t s;
    uint32_t count;       // valid splits seen so far (saturating use: >= 2 means rejected)
    uint32_t ta, tb;      // terms of the first valid split
    uint32_t na, nb, nc;  // queue sizes
};

// Several warps on one sum (search_kernel_group): the group's shared count of valid splits,
// the terms of the first one found, and which share of the splits this warp takes.
struct GroupRef {
    uint32_t* count;
    uint32_t* terms;
    uint32_t part;
};

// Runs stage 1 on up to 32 queued items: passes go to queue b; with the Miller-Rabin variant,
// probes above the map go to queue c.
template <bool kMR>
__device__ void drain_a(SumState& st, WarpQ<kMR>& Q, const SearchArgs& A, int lane)
{
    const uint32_t take = st.na < 32 ? st.na : 32;
    const uint32_t base = st.na - take;
    const bool act = (uint32_t)lane < take;
    if (lane == 0 && A.stats) atomicAdd(&A.stats[0], (unsigned long long)take);
    const uint32_t item = act ? Q.a[base + lane] : 0;
    __syncwarp();
    st.na = base;
    const uint64_t v = act ? stage1_value(item, st.s) : 0;
    if (kMR) {
        const int cls = act ? pair_class(A, v) : 0;
        st.nb = push(Q.b, st.nb, cls == 1, item, lane);
        if (__any_sync(0xFFFFFFFFu, cls == 2)) st.nc = push(Q.c, st.nc, cls == 2, item, lane);
    } else {
        const bool pass = act && pair1<kMR>(A, v);
        st.nb = push(Q.b, st.nb, pass, item, lane);
    }
}

// Miller-Rabin on up to 32 queued probes at once (bit 5 of an item marks a stage-0 probe
// o + b*2^k - 2, else it is the stage-1 probe 2^k + o*b - 2): stage-0 passes go on to queue
// a, stage-1 passes to queue b.
template <bool kMR>
__device__ void drain_c(SumState& st, WarpQ<kMR>& Q, const SearchArgs& A, int lane)
{
    const uint32_t take = st.nc < 32 ? st.nc : 32;
    const uint32_t base = st.nc - take;
    const bool act = (uint32_t)lane < take;
    const uint32_t item = act ? Q.c[base + lane] : 0;
    __syncwarp();
    st.nc = base;
    uint64_t n = 0;
    if (act) {
        const uint32_t k = item & 31, o = item >> 6;
        const uint32_t b = st.s - (o << k);
        n = (item & 32) ? o + ((uint64_t)b << k) - 2 : (1ull << k) + (uint64_t)o * b - 2;
    }
    unsigned long long* cnt = lane == 0 ? A.stats : nullptr;
    const bool prime = mr_rounds(n, act, lane, cnt);
    const bool from0 = (item & 32) != 0;
    st.na = push(Q.a, st.na, prime && from0, item & ~32u, lane);
    st.nb = push(Q.b, st.nb, prime && !from0, item, lane);
}

// Runs stage 2 on up to 32 queued items and adds the valid ones to the count (with G > 1
// warps on the sum, to the group's count, reading back what the other warps found).
template <bool kMR, int G = 1>
__device__ void drain_b(SumState& st, WarpQ<kMR>& Q, const SearchArgs& A, int lane,
                        const GroupRef* grp = nullptr)
{
    const uint32_t take = st.nb < 32 ? st.nb : 32;
    const uint32_t base = st.nb - take;
    const bool act = (uint32_t)lane < take;
    if (lane == 0 && A.stats) atomicAdd(&A.stats[1], (unsigned long long)take);
    const uint32_t item = act ? Q.b[base + lane] : 0;
    __syncwarp();
    st.nb = base;
    uint32_t a = 0, b = 0;
    bool valid;
    if constexpr (kMR) {
        uint64_t pend[kMaxDiv];
        uint32_t np = 0;
        uint32_t nm = act ? stage2_defer(item, st.s, A, &a, &b, pend, &np) : 2;
        // the pending pair probes of all lanes, packed 32 to a Miller-Rabin round: each lane
        // fills the slots [excl, excl + take) of the staging area with its next probes, and
        // counts the composites among them
        uint32_t next = 0;
        for (;;) {
            const uint32_t rem = nm <= 1 ? np - next : 0;
            uint32_t incl = rem;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if (lane >= d) incl += t;
            }
            const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
            if (total == 0) break;
            const uint32_t excl = incl - rem;
            const uint32_t take = excl < 32 ? (rem < 32 - excl ? rem : 32 - excl) : 0;
            for (uint32_t i = 0; i < take; ++i) Q.probe[excl + i] = pend[next + i] - 2;
            __syncwarp();
            const bool need = (uint32_t)lane < (total < 32 ? total : 32);
            const uint64_t n = need ? Q.probe[lane] : 0;
            __syncwarp();
            const bool prime = mr_rounds(n, need, lane, lane == 0 ? A.stats : nullptr);
            const uint32_t comp = __ballot_sync(0xFFFFFFFFu, need && !prime);
            if (take) {
                const uint32_t mine = take == 32 ? 0xFFFFFFFFu : ((1u << take) - 1) << excl;
                nm += __popc(comp & mine);
            }
            next += take;
        }
        valid = act && nm == 1;
    } else {
        valid = act && stage2<kMR>(item, st.s, A, &a, &b);
    }
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, valid);
    if constexpr (G > 1) {
        const int src = m ? __ffs(m) - 1 : 0;
        a = __shfl_sync(0xFFFFFFFFu, a, src);
        b = __shfl_sync(0xFFFFFFFFu, b, src);
        uint32_t total = 0;
        if (lane == 0) {
            if (m) {
                const uint32_t old = atomicAdd(grp->count, (uint32_t)__popc(m));
                if (old == 0) { grp->terms[0] = a; grp->terms[1] = b; }
                total = old + __popc(m);
            } else {
                total = *(volatile uint32_t*)grp->count;
            }
        }
        st.count = __shfl_sync(0xFFFFFFFFu, total, 0);
    } else if (m) {
        const int src = __ffs(m) - 1;
        a = __shfl_sync(0xFFFFFFFFu, a, src);
        b = __shfl_sync(0xFFFFFFFFu, b, src);
        if (st.count == 0) { st.ta = a; st.tb = b; }
        st.count += __popc(m);
    }
}

// The Miller-Rabin variant's queue work in one non-inlined routine (all 32 lanes call it
// together), so each drain's code exists once: that kernel is otherwise large enough to
// stall on instruction fetch. Drains every queue that holds 32 or more items (b first: it
// may reject the sum and pushes nothing); with `flush`, also the partly filled ones, until
// all are empty. Returns false once the sum is rejected.
__device__ __noinline__ bool settle_mr(SumState& st, WarpQ<true>& Q, const SearchArgs& A,
                                       int lane, bool flush)
{
    for (;;) {
        if (st.nb >= 32 || (flush && st.nb > 0 && st.na == 0 && st.nc == 0)) {
            drain_b(st, Q, A, lane);
            if (st.count > 1) return false;
        } else if (st.nc >= 32 || (flush && st.nc > 0 && st.na == 0)) {
            drain_c(st, Q, A, lane);
        } else if (st.na >= 32 || (flush && st.na > 0)) {
            drain_a(st, Q, A, lane);
        } else {
            return true;
        }
    }
}

// Stage 0 of a split. Power2Odd (reference/segmentedSieve.C:573-586): o*b not a multiple of
// 3. Power2Even (:614-627): o*b a multiple of 3 or b prime. Then, in both, the cheap probe
// of DoesPeterKnow (:636): o == b or o + b*2^k - 2 prime. Returns 0 rejected, 1 passed,
// 2 the probe waits for Miller-Rabin (only when kMR).
template <bool kOdd, bool kMR>
__device__ __forceinline__ int stage0(uint32_t s, uint32_t k, uint32_t o, bool act,
                                      const SearchArgs& A)
{
    // The divisibility filters come first and the probe's map word is read only for a split
    // that passes them (a random sector of the map: most of the search's DRAM traffic); the
    // reads of the two splits a lane holds per step are still issued before either is used.
    // b = s - o*2^k is odd and below s (its bit lies in the cache-resident prefix of the map);
    // v = o + b*2^k is odd, so the probe of single_pair(v) is v - 2.
    const uint32_t b = act ? s - (o << k) : 1;
    const uint64_t v = o + ((uint64_t)b << k);
    const uint64_t n = v - 2;
    bool pre;
    uint32_t mv = 0;
    if (kOdd) {
        pre = act && o % 3 != 0 && b % 3 != 0;
        if (pre && n <= A.bound) mv = __ldg(A.map + (n >> 4));
    } else {
        const bool m3 = o % 3 == 0 || b % 3 == 0;
        // the b-prime case (no multiple of 3) reads the probe after b's bit: rare
        if (act && m3 && n <= A.bound) mv = __ldg(A.map + (n >> 4));
        pre = act && (m3 || ((__ldg(A.map + (b >> 4)) >> (7 - ((b >> 1) & 7))) & 1));
        if (pre && !m3 && n <= A.bound) mv = __ldg(A.map + (n >> 4));
    }
    if (!pre) return 0;
    if (o == b) return 1;
    if (n > A.bound) {
        if constexpr (kMR) return pair_class(A, v);
        else return miller_rabin_plain(n, A.err) ? 1 : 0;
    }
    return (mv >> (7 - ((n >> 1) & 7))) & 1;
}

// Enumerates the splits of one phase for sum s: k = kfirst, kfirst+2, ... while o0<<k < s-2;
// for each k the odd parts o = o0, o0+2, ... with o<<k < s-2, two per lane per step. Returns
// false once the sum is rejected (two valid splits).
template <bool kOdd, bool kMR, int G = 1>
__device__ bool run_phase(SumState& st, WarpQ<kMR>& Q, const SearchArgs& A, int lane,
                          const GroupRef* grp = nullptr)
{
    const uint32_t s = st.s;
    const uint32_t o0 = kOdd ? 5 : 3;
    for (uint32_t k = kOdd ? 3 : 2; (o0 << k) < s - 2; k += 2) {
        // odd o in [o0, omax] with o<<k <= s-3
        const uint32_t omax = (s - 3) >> k;
        const uint32_t n = omax >= o0 ? ((omax - o0) >> 1) + 1 : 0;
        uint32_t first = 0;
        if constexpr (G > 1) first = 64 * grp->part;
        for (uint32_t base = first; base < n; base += 64 * G) {
            const uint32_t i0 = base + lane, i1 = i0 + 32;
            const uint32_t oa = o0 + 2 * i0, ob = o0 + 2 * i1;
            const int ca = stage0<kOdd, kMR>(s, k, oa, i0 < n, A);
            const int cb = stage0<kOdd, kMR>(s, k, ob, i1 < n, A);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int cls = h ? cb : ca;
                const uint32_t o = h ? ob : oa;
                st.na = push(Q.a, st.na, cls == 1, enc(k, o, false), lane);
                if constexpr (kMR) {
                    if (__any_sync(0xFFFFFFFFu, cls == 2))
                        st.nc = push(Q.c, st.nc, cls == 2, enc(k, o, true), lane);
                    if ((st.na >= 32 || st.nc >= 32) && !settle_mr(st, Q, A, lane, false))
                        return false;
                } else if (st.na >= kDrainA) {
                    drain_a(st, Q, A, lane);
                    if (st.nb >= kDrainB) {
                        drain_b<kMR, G>(st, Q, A, lane, grp);
                        if (st.count > 1) return false;
                    }
                }
            }
        }
    }
    return true;
}

template <bool kMR>
__device__ void write_result(const SearchArgs& A, uint32_t s, uint32_t ri, uint32_t ta, uint32_t tb)
{
    uint32_t lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
    if (A.rec) {
        const bool lp = isp<kMR>(A, lo);
        const bool hp = isp<kMR>(A, hi);
        A.rec[ri] = ((uint64_t)(lo | (lp ? 0x80000000u : 0u)) << 32) |
                                 (uint64_t)(hi | (hp ? 0x80000000u : 0u));
    }
    if (A.grec) {
        // GpuRecord {u32 sum @0, u64 low @8, u64 high @16, u8 tag @24}, 32 bytes
        uint8_t* r = (uint8_t*)A.grec + (size_t)((s - A.grec_base) >> 1) * 32;
        *(uint32_t*)(r + 0) = s;
        *(uint64_t*)(r + 8) = lo;
        *(uint64_t*)(r + 16) = hi;
        r[24] = 0;
        if (A.gcount) atomicAdd(A.gcount, 1u);
    }
}

template <int W, bool kMR, int K>
__device__ __forceinline__ void search_body(const SearchArgs& A)
{
    static_assert(K == 16 || K == 32 || K == 64, "sums per chunk");
    __shared__ WarpQ<kMR> queues[W];
    const int lane = threadIdx.x & 31;
    WarpQ<kMR>& Q = queues[threadIdx.x >> 5];
    const uint32_t nchunks = A.nseg ? A.nchunks : (A.nsums + K - 1) / K;
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(A.sched, 1u);
        c = __shfl_sync(0xFFFFFFFFu, c, 0);
        if (c >= nchunks) break;
        uint4 g = make_uint4(0, 0, 0, 0);
        if (A.nseg) {
            // work queue of disjoint sum intervals, largest first: the interval whose chunks
            // contain chunk c (entries {lo, count, record base, first chunk}, ascending in .w)
            uint32_t a = 0, b = A.nseg - 1;
            while (a < b) {
                const uint32_t m = (a + b + 1) >> 1;
                if (__ldg(&A.seg[m].w) <= c) a = m; else b = m - 1;
            }
            g = __ldg(&A.seg[a]);
        }
#pragma unroll 1
        for (uint32_t h = 0; h < K; h += 32) {
            // ---- lane-parallel: filter + Power2Prime for up to 32 sums (largest first) ----
            bool act = K >= 32 || (uint32_t)lane < K;
            uint32_t s = 5, ri = 0;
            if (A.nseg == 0) {
                const uint32_t idx = c * K + h + lane;
                act = act && idx < A.nsums;
                if (act) {
                    s = A.hi - 2 * idx;
                    ri = (s - A.lo) >> 1;
                }
            } else {
                const uint32_t idx = (c - g.w) * K + h + lane;
                act = act && idx < g.y;
                if (act) {
                    s = g.x + 2 * (g.y - 1 - idx);  // descending within the interval
                    ri = g.z + ((s - g.x) >> 1);
                }
            }
            bool surv = false;
            uint32_t cnt = 0, ta = 0, tb = 0, comp = 0;
            if (act) {
                // Sammy's first statement (reference/segmentedSieve.C:805-806)
                const uint32_t d3 = s / 3;
                bool pass = !pair1<kMR>(A, s) &&
                            (s != 3 * d3 || isp<kMR>(A, d3));
                if (pass) {
                    // Power2Prime (reference/segmentedSieve.C:547-564)
                    for (uint32_t even = 4, k = 2; even < s - 2; even <<= 1, ++k) {
                        const uint32_t odd = s - even;
                        if (isp<kMR>(A, odd)) {
                            if (++cnt > 1) break;
                            if (cnt == 1) { ta = even; tb = odd; }
                        } else {
                            comp |= 1u << k;
                        }
                    }
                    surv = cnt <= 1;
                }
            }

            // ---- warp-cooperative: the remaining phases, one survivor at a time ----
            uint32_t smask = __ballot_sync(0xFFFFFFFFu, surv);
            while (smask) {
                const int src = __ffs(smask) - 1;
                smask &= smask - 1;
                SumState st;
                st.s = __shfl_sync(0xFFFFFFFFu, s, src);
                const uint32_t sri = __shfl_sync(0xFFFFFFFFu, ri, src);
                st.count = __shfl_sync(0xFFFFFFFFu, cnt, src);
                st.ta = __shfl_sync(0xFFFFFFFFu, ta, src);
                st.tb = __shfl_sync(0xFFFFFFFFu, tb, src);
                const uint32_t cmask = __shfl_sync(0xFFFFFFFFu, comp, src);
                st.na = 0;
                st.nb = 0;
                st.nc = 0;
                // Power2Composite items (reference/segmentedSieve.C:591-605) go straight to stage 2
                st.nb = push(Q.b, 0, (cmask >> lane) & 1, enc(lane, 0, true), lane);
                bool open = true;
                if constexpr (kMR) {
                    if (st.nb >= 32) open = settle_mr(st, Q, A, lane, false);
                } else if (st.nb >= kDrainB) {
                    drain_b(st, Q, A, lane);
                    open = st.count <= 1;
                }
                if (open) open = run_phase<true, kMR>(st, Q, A, lane);
                if (open) open = run_phase<false, kMR>(st, Q, A, lane);
                // flush the partly filled queues: stage 1, then Miller-Rabin, then stage 2
                if constexpr (kMR) {
                    if (open) open = settle_mr(st, Q, A, lane, true);
                } else {
                    // stage 1 first while queue b has room, then stage 2 (one copy of each)
                    while (open && (st.na > 0 || st.nb > 0)) {
                        if (st.na > 0 && st.nb < 32) {
                            drain_a(st, Q, A, lane);
                        } else {
                            drain_b(st, Q, A, lane);
                            open = st.count <= 1;
                        }
                    }
                }
                if (open && st.count == 1 && lane == 0) write_result<kMR>(A, st.s, sri, st.ta, st.tb);
                __syncwarp();
            }
        }   // rounds of 32 sums of the chunk
    }
}


// The map-only kernel keeps kWarpsPerSm warps resident (its register budget follows); the
// Miller-Rabin variant, whose deferred divisor lists are larger, keeps the compiler's own.
template <int W, int K>
__global__ void __launch_bounds__(W * 32, kWarpsPerSm / W) search_kernel(const SearchArgs A)
{
    search_body<W, false, K>(A);
}

template <int W>
__global__ void __launch_bounds__(W * 32) search_kernel_mr(const SearchArgs A)
{
    search_body<W, true, 32>(A);
}

// Several warps on one sum (map-only variant): a group of G warps takes chunks of 32*G sums;
// each warp runs the lane-parallel filter on 32 of them and appends its survivors to the
// group's list, then the G warps take the survivors one at a time, each enumerating every
// G-th block of 64 splits (and every G-th Power2Composite item) with its own queues, adding
// the valid splits it finds to the group's shared count. The verdict depends only on whether
// exactly one split is valid, so how the splits are shared out does not change it. Warps of
// a group meet at a named barrier (id 1 + group index) around each survivor.
template <int G>
struct GroupShared {
    uint32_t chunk, n, count;
    uint32_t terms[2];
    uint32_t s[32 * G], ri[32 * G], cnt[32 * G], ta[32 * G], tb[32 * G], comp[32 * G];
};

__device__ __forceinline__ void group_bar(uint32_t id, uint32_t threads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

template <int W, int G>
__global__ void __launch_bounds__(W * 32, kWarpsPerSm / W) search_kernel_group(const SearchArgs A)
{
    static_assert(G > 1 && W % G == 0 && W / G <= 15, "group shape");
    __shared__ WarpQ<false> queues[W];
    __shared__ GroupShared<G> groups[W / G];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t gi = warp / G, part = warp % G, bar = gi + 1, nthr = 32 * G;
    WarpQ<false>& Q = queues[warp];
    GroupShared<G>& gs = groups[gi];
    const GroupRef grp{&gs.count, gs.terms, part};
    const uint32_t K = 32 * G;  // sums per chunk
    const uint32_t nchunks = A.nseg ? A.nchunks : (A.nsums + K - 1) / K;
    if (part == 0 && lane == 0) gs.n = 0;
    for (;;) {
        if (part == 0 && lane == 0) gs.chunk = atomicAdd(A.sched, 1u);
        group_bar(bar, nthr);
        const uint32_t c = gs.chunk;
        if (c >= nchunks) break;
        // ---- lane-parallel: filter + Power2Prime for this warp's 32 sums of the chunk ----
        bool act;
        uint32_t s = 5, ri = 0;
        if (A.nseg == 0) {
            const uint32_t idx = c * K + 32 * part + lane;
            act = idx < A.nsums;
            if (act) {
                s = A.hi - 2 * idx;
                ri = (s - A.lo) >> 1;
            }
        } else {
            uint32_t a = 0, b = A.nseg - 1;
            while (a < b) {
                const uint32_t m = (a + b + 1) >> 1;
                if (__ldg(&A.seg[m].w) <= c) a = m; else b = m - 1;
            }
            const uint4 g = __ldg(&A.seg[a]);
            const uint32_t idx = (c - g.w) * K + 32 * part + lane;
            act = idx < g.y;
            if (act) {
                s = g.x + 2 * (g.y - 1 - idx);  // descending within the interval
                ri = g.z + ((s - g.x) >> 1);
            }
        }
        bool surv = false;
        uint32_t cnt = 0, ta = 0, tb = 0, comp = 0;
        if (act) {
            // Sammy's first statement (reference/segmentedSieve.C:805-806)
            const uint32_t d3 = s / 3;
            const bool pass = !pair1<false>(A, s) && (s != 3 * d3 || isp<false>(A, d3));
            if (pass) {
                // Power2Prime (reference/segmentedSieve.C:547-564)
                for (uint32_t even = 4, k = 2; even < s - 2; even <<= 1, ++k) {
                    const uint32_t odd = s - even;
                    if (isp<false>(A, odd)) {
                        if (++cnt > 1) break;
                        if (cnt == 1) { ta = even; tb = odd; }
                    } else {
                        comp |= 1u << k;
                    }
                }
                surv = cnt <= 1;
            }
        }
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, surv);
        uint32_t base = 0;
        if (lane == 0 && m) base = atomicAdd(&gs.n, (uint32_t)__popc(m));
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (surv) {
            const uint32_t j = base + __popc(m & ((1u << lane) - 1));
            gs.s[j] = s;
            gs.ri[j] = ri;
            gs.cnt[j] = cnt;
            gs.ta[j] = ta;
            gs.tb[j] = tb;
            gs.comp[j] = comp;
        }
        group_bar(bar, nthr);
        // ---- the group on one survivor at a time ----
        const uint32_t nsurv = gs.n;
        for (uint32_t i = 0; i < nsurv; ++i) {
            if (part == 0 && lane == 0) {
                gs.count = gs.cnt[i];
                gs.terms[0] = gs.ta[i];
                gs.terms[1] = gs.tb[i];
            }
            group_bar(bar, nthr);
            SumState st;
            st.s = gs.s[i];
            st.count = gs.cnt[i];
            st.ta = st.tb = 0;
            st.na = 0;
            st.nc = 0;
            const uint32_t cmask = gs.comp[i];
            // Power2Composite items (reference/segmentedSieve.C:591-605), every G-th to this warp
            st.nb = push(Q.b, 0, ((cmask >> lane) & 1) && lane % G == part, enc(lane, 0, true), lane);
            bool open = true;
            if (st.nb >= kDrainB) {
                drain_b<false, G>(st, Q, A, lane, &grp);
                open = st.count <= 1;
            }
            if (open) open = run_phase<true, false, G>(st, Q, A, lane, &grp);
            if (open) open = run_phase<false, false, G>(st, Q, A, lane, &grp);
            while (open && (st.na > 0 || st.nb > 0)) {
                if (st.na > 0 && st.nb < 32) {
                    drain_a(st, Q, A, lane);
                } else {
                    drain_b<false, G>(st, Q, A, lane, &grp);
                    open = st.count <= 1;
                }
            }
            group_bar(bar, nthr);
            if (part == 0 && lane == 0 && gs.count == 1)
                write_result<false>(A, st.s, gs.ri[i], gs.terms[0], gs.terms[1]);
            group_bar(bar, nthr);
        }
        if (part == 0 && lane == 0) gs.n = 0;
    }
}

}  // namespace

// The stage-2 scratch is dynamic shared memory, W * 3.3 KB a block (above the 48 KB a block
// gets without asking for 16 warps); the attribute is set at every launch, which stream
// capture allows.
template <int W, bool kMR, int K>
int launch_w(const SearchArgs& a, int sms, cudaStream_t stream)
{
    void (*kernel)(SearchArgs) = kMR ? search_kernel_mr<W> : search_kernel<W, K>;
    const uint32_t dyn = W * kWarpScratchBytes;
    FFB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    int per_sm = 0;
    FFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, W * 32, dyn));
    if (per_sm < 1) per_sm = 1;
    const uint32_t chunks = a.nseg ? a.nchunks : (a.nsums + K - 1) / K;
    uint32_t blocks = (uint32_t)sms * (uint32_t)per_sm;
    const uint32_t need = (chunks + W - 1) / W;
    if (blocks > need) blocks = need;
    if (blocks == 0) return 0;
    kernel<<<blocks, W * 32, dyn, stream>>>(a);
    FFB_CUDA(cudaGetLastError());
    return 0;
}

template <int W, int G>
int launch_group(const SearchArgs& a, int sms, cudaStream_t stream)
{
    const uint32_t dyn = W * kWarpScratchBytes;
    FFB_CUDA(cudaFuncSetAttribute(search_kernel_group<W, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    int per_sm = 0;
    FFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search_kernel_group<W, G>, W * 32, dyn));
    if (per_sm < 1) per_sm = 1;
    const uint32_t chunks = a.nseg ? a.nchunks : (a.nsums + 32 * G - 1) / (32 * G);
    uint32_t blocks = (uint32_t)sms * (uint32_t)per_sm;
    const uint32_t need = (chunks + W / G - 1) / (W / G);
    if (blocks > need) blocks = need;
    if (blocks == 0) return 0;
    search_kernel_group<W, G><<<blocks, W * 32, dyn, stream>>>(a);
    FFB_CUDA(cudaGetLastError());
    return 0;
}

template <int W>
int launch_map_only(const SearchArgs& a, int sms, cudaStream_t stream)
{
    switch (a.chunk) {
    case 16: return launch_w<W, false, 16>(a, sms, stream);
    case 64: return launch_w<W, false, 64>(a, sms, stream);
    default: return launch_w<W, false, 32>(a, sms, stream);
    }
}

// The map-only kernel when the map reaches every value the sums up to a.hi probe (nothing
// goes to Miller-Rabin in stages 0 and 1), else the variant that batches Miller-Rabin (32
// sums per chunk, one warp per sum). Shapes outside the offered ones are refused.
int launch_search(const SearchArgs& a, int sms, cudaStream_t stream)
{
    if (a.nseg == 0 && a.nsums == 0) return 0;
    const uint64_t pb = ffb_probe_bound(a.hi);
    const bool mr = pb == 0 || a.bound < pb;
    const bool warps_ok = a.warps == 0 || a.warps == 4 || a.warps == 8 || a.warps == 16;
    const bool shape_ok = a.group == 1 ? (a.chunk == 32 || (!mr && (a.chunk == 16 || a.chunk == 64)))
                                       : ((a.group == 2 || a.group == 4) && a.chunk == 32 * a.group && !mr);
    if (!warps_ok || !shape_ok) {
        std::fprintf(stderr, "ffb: search shape (%u warps a block, %u per sum, %u sums a chunk) not "
                     "offered%s\n", a.warps, a.group, a.chunk,
                     mr ? " with a map below the probes (one warp per sum, 32 sums a chunk)" : "");
        return -1;
    }
    if (a.warps == 0 && a.group == 1 && a.chunk == 32 && a.nseg == 0 && !mr) {
        // unset shape on one range over a map covering every probe: 16 warps a block, 2 per
        // sum, 64-sum chunks (2^21 job on one box: 187.5 ms; 4 per sum 219 ms, one warp per
        // sum 216-256 ms)
        SearchArgs b = a;
        b.warps = 16;
        b.group = 2;
        b.chunk = 64;
        return launch_group<16, 2>(b, sms, stream);
    }
    if (a.group == 2 || a.group == 4) {
        switch (a.warps) {
        case 4: return a.group == 2 ? launch_group<4, 2>(a, sms, stream) : launch_group<4, 4>(a, sms, stream);
        case 16: return a.group == 2 ? launch_group<16, 2>(a, sms, stream) : launch_group<16, 4>(a, sms, stream);
        default: return a.group == 2 ? launch_group<8, 2>(a, sms, stream) : launch_group<8, 4>(a, sms, stream);
        }
    }
    if (mr) {
        switch (a.warps) {
        // unset: 4 warps (the served mode's first 1,000 seed-1 requests: 914k sums/s with
        // 4-warp blocks, 874k with 16, 843k with 8; 2^21 sums against the served map: 441,
        // 430 and 494 ms)
        case 8: return launch_w<8, true, 32>(a, sms, stream);
        case 16: return launch_w<16, true, 32>(a, sms, stream);
        default: return launch_w<4, true, 32>(a, sms, stream);
        }
    }
    switch (a.warps) {
    case 4: return launch_map_only<4>(a, sms, stream);
    case 16: return launch_map_only<16>(a, sms, stream);
    // unset (a work queue, or a chunk given): 8 warps (2^21 job on one box with 32-sum chunks:
    // 225-228 ms with 8-warp blocks, 226-229 ms with 4, 228-234 ms with 16)
    default: return launch_map_only<8>(a, sms, stream);
    }
}

}  // namespace ffb
