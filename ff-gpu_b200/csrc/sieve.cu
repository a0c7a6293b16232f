// sieve.cu -- the odd-only bitmap sieve (Prime::SegmentFill, reference/segmentedSieve.C:
// 255-270; slab contract of source/sieve_slab_kernel.h:40-107).
//
// A slab covers the values [seg_lo, seg_hi). Its bit m stands for the odd value
// (seg_lo|1) + 2m and lives at byte m>>3, mask 0x80>>(m&7) of the output (the reference's
// seg_lo-relative layout; with seg_lo == 0 this is the global map layout). Bits of values
// >= seg_hi stay 1, like the reference's untouched 0xff bytes.
//
// Fast path (the list starts with the odd primes 3,5,7,... in order):
//   * The slab is cut into shared-memory tiles; a persistent grid walks the tiles.
//   * Each tile starts from three pre-computed patterns (the odd numbers free of 3..13, of
//     17,19,23 and of 29,31,37; periods 15015, 7429 and 33263 odd numbers) read with funnel
//     shifts and ANDed, so the eleven smallest odd primes are never marked one by one.
//   * Primes with many marks per tile are marked warp-cooperatively (each lane a strided
//     subset of the multiples), the rest one prime per thread; all with shared-memory
//     atomicAnd. The first multiple in a tile comes from a Barrett reduction.
//   * The tile is converted to the reference bit order (brev + byte swap) and written to
//     HBM with 16-byte stores.
// Any other list entry (e.g. the 2 some callers pass, or primes out of order) is marked by
// a generic kernel that follows the reference's first-multiple formula literally.
#include "ffb_device.cuh"
#include "ffb_internal.h"

#include <algorithm>
#include <vector>

namespace ffb {
namespace {

constexpr int kSieveThreads = 512;

// Pre-sieve patterns: bit j (LSB-first) of pattern t is 1 iff the odd number 2j+1 has no
// factor among the primes of group t; each pattern repeats with the product of its
// primes (in odd numbers) and is stored with one extra period word so any 32-bit window
// can be read without wrapping.
constexpr uint32_t kPeriod0 = 3 * 5 * 7 * 11 * 13;   // 15015
constexpr uint32_t kPeriod1 = 17 * 19 * 23;          // 7429
constexpr uint32_t kPeriod2 = 29 * 31 * 37;          // 33263
constexpr uint32_t kWords0 = (kPeriod0 + 63) / 32 + 1;
constexpr uint32_t kWords1 = (kPeriod1 + 63) / 32 + 1;
constexpr uint32_t kWords2 = (kPeriod2 + 63) / 32 + 1;
constexpr uint32_t kWheelWords = kWords0 + kWords1 + kWords2;
constexpr int kWheelPrimes = 11;                     // 3 .. 37
__device__ uint32_t g_wheel[kWheelWords];

struct TileArgs {
    uint8_t* out;
    uint64_t out_bytes;     // relative bytes written
    uint64_t base_odd;      // value of bit 0
    uint64_t nbits;         // bits of odd values < seg_hi
    uint64_t total_bits;    // 8 * out_bytes
    const uint32_t* primes; // device list (standard prefix)
    const uint64_t* mu;     // floor((2^64-1) / p) per prime
    uint32_t ibeg, ismall, iend;  // [ibeg, ismall): warp-cooperative, [ismall, iend): per thread
    int wheel;
    int clear_one;          // clear the bit of the value 1 (seg_lo == 0)
    uint32_t tile_words;
    uint64_t ntiles;
};

__device__ __forceinline__ uint64_t mod_barrett(uint64_t x, uint64_t p, uint64_t mu)
{
    uint64_t r = x - __umul64hi(x, mu) * p;
    while (r >= p) r -= p;
    return r;
}

// First bit >= m_lo (relative) of an odd multiple of p that is >= p*p, for odd p.
__device__ __forceinline__ uint64_t first_bit(uint64_t m_lo, uint64_t base_odd, uint64_t p,
                                              uint64_t mu)
{
    const uint64_t v = base_odd + 2 * m_lo;                 // odd value of bit m_lo
    const uint64_t r = mod_barrett(v, p, mu);
    // smallest multiple of p >= v; with v and p odd it is odd iff r is odd (or r == 0),
    // otherwise the next odd multiple is p further
    uint64_t f = r == 0 ? v : v + (p - r);
    if (!(f & 1)) f += p;
    const uint64_t pp = p * p;
    if (f < pp) f = pp;
    return (f - base_odd) >> 1;
}

__device__ __forceinline__ uint32_t window(const uint32_t* w, uint64_t j, uint32_t period)
{
    const uint32_t ph = (uint32_t)(j % period);
    return __funnelshift_r(w[ph >> 5], w[(ph >> 5) + 1], ph & 31);
}

__global__ void __launch_bounds__(kSieveThreads) sieve_tiles(const TileArgs A)
{
    extern __shared__ uint32_t smem[];
    uint32_t* tile = smem;
    uint32_t* wheel = smem + A.tile_words;
    if (A.wheel)
        for (uint32_t i = threadIdx.x; i < kWheelWords; i += blockDim.x) wheel[i] = g_wheel[i];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint64_t tile_bits = (uint64_t)A.tile_words * 32;
    const uint64_t j0 = (A.base_odd - 1) >> 1;  // pattern index of bit 0

    for (uint64_t t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const uint64_t m0 = t * tile_bits;
        const uint64_t m1 = min(m0 + tile_bits, A.total_bits);
        const uint32_t words = (uint32_t)((m1 - m0 + 31) >> 5);
        __syncthreads();  // previous tile fully stored; patterns loaded
        // ---- 1. initial pattern ----
        for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
            const uint64_t gm = m0 + 32ull * w;
            uint32_t x = 0xFFFFFFFFu;
            if (A.wheel) {
                x = window(wheel, j0 + gm, kPeriod0) & window(wheel + kWords0, j0 + gm, kPeriod1) &
                    window(wheel + kWords0 + kWords1, j0 + gm, kPeriod2);
            }
            if (gm + 32 > A.nbits) {  // bits of values >= seg_hi stay set
                const uint64_t keep = A.nbits > gm ? A.nbits - gm : 0;
                x |= keep >= 32 ? 0u : ~((1u << keep) - 1u);
            }
            tile[w] = x;
        }
        __syncthreads();
        const uint64_t mlim = min(m1, A.nbits);
        const uint32_t rl = (uint32_t)(mlim > m0 ? mlim - m0 : 0);  // tile-relative limit
        // ---- 2a. primes with many multiples per tile: one warp per prime ----
        for (uint32_t i = A.ibeg + warp; i < A.ismall; i += nwarps) {
            const uint64_t p = A.primes[i];
            const uint64_t f = first_bit(m0, A.base_odd, p, A.mu[i]);
            if (f >= mlim) continue;
            const uint32_t p32 = (uint32_t)p, step = 32 * p32;
            uint32_t r = (uint32_t)(f - m0) + lane * p32;
#pragma unroll 4
            for (; r < rl; r += step) atomicAnd(&tile[r >> 5], ~(1u << (r & 31)));
        }
        // ---- 2b. the rest: one thread per prime ----
        for (uint32_t i = A.ismall + threadIdx.x; i < A.iend; i += blockDim.x) {
            const uint64_t p = A.primes[i];
            const uint64_t f = first_bit(m0, A.base_odd, p, A.mu[i]);
            if (f >= mlim) continue;
            const uint32_t p32 = (uint32_t)p;
#pragma unroll 4
            for (uint32_t r = (uint32_t)(f - m0); r < rl; r += p32)
                atomicAnd(&tile[r >> 5], ~(1u << (r & 31)));
        }
        __syncthreads();
        // ---- 3. the pattern primes themselves and the value 1 ----
        if (threadIdx.x == 0 && A.base_odd <= 37) {
            const uint32_t wp[kWheelPrimes] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
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
    const uint32_t periods[3] = {kPeriod0, kPeriod1, kPeriod2};
    const uint32_t words[3] = {kWords0, kWords1, kWords2};
    const uint32_t group[3][5] = {{3, 5, 7, 11, 13}, {17, 19, 23, 0, 0}, {29, 31, 37, 0, 0}};
    uint32_t off = 0;
    for (int g = 0; g < 3; ++g) {
        for (uint32_t j = 0; j < words[g] * 32; ++j) {
            const uint32_t v = 2 * (j % periods[g]) + 1;
            bool keep = true;
            for (int q = 0; q < 5 && group[g][q]; ++q) keep = keep && v % group[g][q] != 0;
            if (keep) w[off + (j >> 5)] |= 1u << (j & 31);
        }
        off += words[g];
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
// pointers filled in by the caller), its launch shape, the table contents, and the list
// entries that go through sieve_generic.
struct SieveHost {
    TileArgs T;
    size_t smem = 0;
    unsigned blocks = 0;
    bool tiles = false;
    std::vector<uint64_t> mu;
    std::vector<uint32_t> list;
    struct Gen {
        uint64_t p, first, nmarks;
        unsigned grid;
    };
    std::vector<Gen> gen;
};

namespace {

// The standard prefix of the list goes through the tiled kernel; every other entry through
// sieve_generic. Marks only ever clear bits, so splitting the list is exact.
int analyse(const SieveArgs& a, int sms, SieveHost& H)
{
    if (upload_wheel()) return -1;
    const uint64_t out_bytes = (a.seg_hi - a.seg_lo + 15) >> 4;
    if (((uintptr_t)a.out & 15) != 0) {
        std::fprintf(stderr, "ffb: sieve output must be 16-byte aligned\n");
        return -1;
    }
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
    const int wheel = std_n >= kWheelPrimes;  // the patterns need 3..37 in the list
    H.list.assign(h + off, h + off + iend);
    H.mu.resize(iend);
    for (uint32_t i = 0; i < iend; ++i) H.mu[i] = ~0ull / h[off + i];   // Barrett constants

    TileArgs& T = H.T;
    T.out = a.out;
    T.out_bytes = out_bytes;
    T.base_odd = a.seg_lo | 1;
    T.nbits = a.seg_hi > T.base_odd ? (a.seg_hi - T.base_odd + 1) / 2 : 0;
    T.total_bits = out_bytes * 8;
    T.primes = nullptr;
    T.mu = nullptr;
    T.wheel = wheel;
    T.clear_one = a.clear_one && a.seg_lo == 0;
    T.ibeg = wheel ? kWheelPrimes : 0;
    if (T.ibeg > iend) T.ibeg = iend;
    uint32_t tile_bytes = a.tile_bytes ? a.tile_bytes : 96 * 1024;
    tile_bytes = (tile_bytes + 15) & ~15u;
    T.tile_words = tile_bytes / 4;
    const uint64_t tile_bits = (uint64_t)T.tile_words * 32;
    T.ismall = T.ibeg;
    while (T.ismall < iend && (uint64_t)h[off + T.ismall] * 32 < tile_bits) ++T.ismall;
    T.iend = iend;
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
    return 0;
}

int enqueue(const SieveHost& H, const SieveArgs& a, cudaStream_t stream)
{
    if (H.tiles) {
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

int launch_sieve(const SieveArgs& a, int sms, cudaStream_t stream)
{
    if (a.seg_hi <= a.seg_lo) return 0;
    SieveHost H;
    if (analyse(a, sms, H)) return -1;
    // device copy of the marked prefix and its Barrett constants (stream-ordered scratch)
    const size_t nl = H.list.empty() ? 1 : H.list.size();
    uint8_t* scratch = nullptr;
    FFB_CUDA(cudaMallocAsync((void**)&scratch, 12 * nl + 16, stream));
    H.T.mu = (const uint64_t*)scratch;
    H.T.primes = (const uint32_t*)(scratch + 8 * nl);
    int rc = 0;
    if (!H.list.empty() &&
        (cudaMemcpyAsync(scratch, H.mu.data(), 8 * H.mu.size(), cudaMemcpyHostToDevice, stream) != cudaSuccess ||
         cudaMemcpyAsync(scratch + 8 * nl, H.list.data(), 4 * H.list.size(), cudaMemcpyHostToDevice,
                         stream) != cudaSuccess))
        rc = -1;
    if (!rc) rc = enqueue(H, a, stream);
    // (copies from pageable host memory are staged before cudaMemcpyAsync returns, so the
    // host vectors may go out of scope here)
    cudaFreeAsync(scratch, stream);
    return rc;
}

// A sieve prepared once and launched many times (the device tables stay allocated):
// enqueue_sieve_plan only launches kernels, so it can be captured in a CUDA graph.
struct SievePlan {
    SieveHost H;
    SieveArgs a;
    uint8_t* table = nullptr;
};

SievePlan* create_sieve_plan(const SieveArgs& a, int sms)
{
    SievePlan* P = new SievePlan;
    P->a = a;
    if (a.seg_hi > a.seg_lo && analyse(a, sms, P->H)) {
        delete P;
        return nullptr;
    }
    const size_t nl = P->H.list.empty() ? 1 : P->H.list.size();
    if (cudaMalloc(&P->table, 12 * nl + 16) != cudaSuccess) {
        cudaGetLastError();
        delete P;
        return nullptr;
    }
    P->H.T.mu = (const uint64_t*)P->table;
    P->H.T.primes = (const uint32_t*)(P->table + 8 * nl);
    if (!P->H.list.empty() &&
        (cudaMemcpy(P->table, P->H.mu.data(), 8 * P->H.mu.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(P->table + 8 * nl, P->H.list.data(), 4 * P->H.list.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess)) {
        cudaFree(P->table);
        delete P;
        return nullptr;
    }
    return P;
}

int enqueue_sieve_plan(const SievePlan* P, cudaStream_t stream)
{
    if (P->a.seg_hi <= P->a.seg_lo) return 0;
    return enqueue(P->H, P->a, stream);
}

void destroy_sieve_plan(SievePlan* P)
{
    if (!P) return;
    if (P->table) cudaFree(P->table);
    delete P;
}

}  // namespace ffb
