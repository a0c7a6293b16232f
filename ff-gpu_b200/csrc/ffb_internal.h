// ffb_internal.h -- internal host-side API of the CUDA layer (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

namespace ffb {

// One odd prime of the trial-division table with its exact-division constants:
// n is divisible by p iff n*inv (mod 2^32) <= lim, and then the quotient is n*inv.
struct TDiv {
    uint32_t p, inv, lim, pad;
};

// Arguments of one search launch over the odd sums lo, lo+2, ..., hi.
struct SearchArgs {
    const uint8_t* map;     // reference bitmap (device)
    uint64_t bound;         // values <= bound are answered by the bitmap, above by Miller-Rabin
    uint32_t lo, hi;        // odd sums, lo <= hi, both odd
    uint32_t nsums;         // (hi-lo)/2 + 1
    uint64_t* rec;          // packed result per sum (or null): rec[(s-lo)/2]
    void* grec;             // reference GpuRecord slots (or null): grec[(s-grec_base)/2]
    uint32_t grec_base;     // sumStart the GpuRecord slots are indexed from
    uint32_t* gcount;       // reference solution counter (or null)
    const TDiv* tdiv;       // odd primes below 65536 with exact-division constants
    uint32_t ntdiv;
    uint32_t* sched;        // [0]: next chunk of sums (must be 0 at launch)
    uint32_t* err;          // error flags (ffb_device.cuh)
    unsigned long long* stats;  // [0] stage-1 probes, [1] stage-2 items (or null)
    const uint4* seg = nullptr;  // work queue of disjoint intervals {lo, count, record base, first
                            // chunk}, largest sums first (or null: the single range lo..hi)
    uint32_t nseg = 0;      // intervals in seg (0: single range)
    uint32_t nchunks = 0;   // chunks of `chunk` sums over all intervals
    uint32_t warps = 0;     // warps per block: 4, 8 or 16 (0: 16 map-only, 4 Miller-Rabin)
    uint32_t chunk = 32;    // sums a warp takes per pull of the work counter: 16, 32 or 64
                            // (one warp per sum), 32 * group with group > 1
    uint32_t group = 1;     // warps per sum: 1, or 2 / 4 (map-only variant)
    // smallest prime factor of each odd n < spf_limit: spf[n >> 1] is its index in tdiv, or
    // 0xFFFF when n is 1 or prime (null: factorisations by trial division alone)
    const uint16_t* spf = nullptr;
    uint32_t spf_limit = 0;
};

// Packed per-sum record written by the search: 0 = no solution line, else
//   bits 63: low term prime, 62..32: low term, 31: high term prime, 30..0: high term.
inline uint32_t rec_low(uint64_t r) { return (uint32_t)(r >> 32) & 0x7FFFFFFFu; }
inline uint32_t rec_high(uint64_t r) { return (uint32_t)r & 0x7FFFFFFFu; }
inline bool rec_low_prime(uint64_t r) { return (r >> 63) & 1; }
inline bool rec_high_prime(uint64_t r) { return (r >> 31) & 1; }

// Per-device state the entry points share: the trial-division table, scratch words and
// the SM count. Created on first use of a device, kept until the process exits.
struct DeviceState {
    int device = -1;
    int sms = 0;
    TDiv* tdiv = nullptr;
    uint32_t ntdiv = 0;
    uint32_t* words = nullptr;  // [0..63] scheduler counters, [64] error flags
    uint16_t* spf = nullptr;    // smallest-prime-factor table (SearchArgs::spf), 32 MB
    uint32_t spf_limit = 0;
};
DeviceState* device_state(int device);  // nullptr (and a stderr line) on failure

// Slab sieve over values [seg_lo, seg_hi) into out (seg_lo-relative layout, see sieve.cu),
// with the host list h_primes as the marking list. out must be 16-byte aligned.
struct SieveArgs {
    uint8_t* out;            // (seg_hi - seg_lo + 15) >> 4 bytes are written
    uint64_t seg_lo, seg_hi;
    const uint32_t* h_primes = nullptr;  // marking list (host, ascending in every reference caller)
    uint32_t nprimes = 0;
    uint32_t tile_bytes = 0;   // shared-memory tile (multiple of 16; 0 = default)
    int clear_one = 0;         // clear the value-1 bit when seg_lo == 0 (the map init does)
    int true_map = 0;          // 1: the prime map itself: the list is every odd prime p with
                               // p*p < seg_hi, made on the device (h_primes is ignored)
};

// err: the device error word (a list beyond its bound raises kErrBadInput).
int launch_sieve(const SieveArgs& a, int sms, uint32_t* err, cudaStream_t stream);

// A sieve analysed once (device tables allocated and uploaded); enqueue_sieve_plan launches
// only kernels, so it can be captured into a CUDA graph and replayed.
struct SievePlan;
SievePlan* create_sieve_plan(const SieveArgs& a, int sms, uint32_t* err);
int enqueue_sieve_plan(const SievePlan* p, cudaStream_t stream);
void destroy_sieve_plan(SievePlan* p);
int launch_search(const SearchArgs& a, int sms, cudaStream_t stream);

// Entry helpers shared by the C ABI and the pipeline (capi.cu).
int run_sieve(int dev, const uint32_t* h_primes, uint32_t n, uint64_t seg_lo, uint64_t seg_hi,
              uint8_t* d_out, cudaStream_t stream, int clear_one, uint32_t tile_bytes = 0);
// The prime map's values [seg_lo, seg_hi) (every odd prime p with p*p < seg_hi marks; the list
// is made on the device) into d_out, seg_lo-relative.
int run_sieve_map(int dev, uint64_t seg_lo, uint64_t seg_hi, uint8_t* d_out, cudaStream_t stream,
                  int clear_one, uint32_t tile_bytes = 0);
// The device's error word (kErr* flags, read and cleared by ffb_take_errors).
uint32_t* device_err_word(DeviceState* s);
int run_search(int dev, const uint8_t* d_map, uint64_t bound, uint32_t lo, uint32_t hi,
               uint64_t* d_rec, void* grec, uint32_t grec_base, uint32_t* gcount,
               cudaStream_t stream, uint32_t warps = 0, uint32_t chunk = 32, uint32_t group = 1);

// Odd primes <= limit into the host vector (ascending).
void host_odd_primes(uint64_t limit, uint32_t** out, uint32_t* n);


#define FFB_CUDA(call)                                                                \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            std::fprintf(stderr, "ffb: CUDA error at %s:%d: %s (%s)\n", __FILE__,     \
                         __LINE__, cudaGetErrorName(e_), cudaGetErrorString(e_));     \
            return -1;                                                                \
        }                                                                             \
    } while (0)

}  // namespace ffb
