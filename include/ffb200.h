/*
 * ffb200.h -- C ABI of the B200 (sm_100a) build of ff-gpu's hot path: the odd-only prime
 * sieve and the per-sum Freudenthal search.
 *
 * Every entry point keeps the name, argument meaning, return codes and memory ownership
 * of the reference interface it replaces (cited per declaration), with the arch tag
 * sm_100a. The reference's own harnesses resolve the NVIDIA kernels through the _sm_120
 * names, so those are exported as aliases of the sm_100a functions; the _gfx1201 getters
 * exist for link compatibility and return NULL (there is no AMD path and no dispatch).
 *
 * Plain pointers and sizes only. "d_" pointers are CUDA device pointers, "h_" pointers
 * host memory. All functions return 0 on success and -1 on error (with one line on
 * stderr), unless stated otherwise.
 *
 * Domain: sums up to 2^25 (products below 2^48, where the reference's Miller-Rabin
 * arithmetic is exact); larger sumLimit values are rejected with -1.
 */
#ifndef FFB200_H
#define FFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One solution slot (source/m4/gpu_search_kernel.h:37-42): sum==0 marks an empty slot.
 * Layout {u32 sum @0, u64 low @8, u64 high @16, u8 tag @24}, sizeof 32. tag is 0. */
typedef struct {
    uint32_t sum;
    uint64_t low;
    uint64_t high;
    uint8_t tag;
} GpuRecord;

/* ---------------------------------------------------------------------------------- */
/* Sieve slab (source/sieve_slab_kernel.cpp:41-48, 66-131)                             */
/* ---------------------------------------------------------------------------------- */

typedef int (*SieveSlabRunFn)(int deviceIndex, const uint32_t* h_primes, uint32_t numPrimes,
                              uint64_t segLo, uint64_t segHi, uint8_t* h_out);

/* Sieves the values [segLo, segHi) with the listed primes (ascending; the reference's
 * callers pass the odd primes up to sqrt(segHi), some with a leading 2, which is honoured
 * literally). h_out receives (segHi+15)>>4 bytes: the marks in segLo-RELATIVE layout
 * (value i -> byte (i-segLo)>>4, bit 0x80>>((i-segLo)>>1&7)), all other bytes 0xff,
 * byte 0 = 0x7f when segLo == 0. Synchronous; allocates and frees its own device memory.
 * Replaces SieveSlabRun_<arch> (source/sieve_slab_kernel.cpp:80-131). */
int SieveSlabRun_sm_100a(int deviceIndex, const uint32_t* h_primes, uint32_t numPrimes,
                         uint64_t segLo, uint64_t segHi, uint8_t* h_out);
/* Returns SieveSlabRun_sm_100a when deviceIndex names a visible CUDA device, else NULL.
 * Replaces SieveSlabGetLaunchFn_<arch> (source/sieve_slab_kernel.cpp:124-131). */
SieveSlabRunFn SieveSlabGetLaunchFn_sm_100a(int deviceIndex);
int SieveSlabRun_sm_120(int deviceIndex, const uint32_t* h_primes, uint32_t numPrimes,
                        uint64_t segLo, uint64_t segHi, uint8_t* h_out);
SieveSlabRunFn SieveSlabGetLaunchFn_sm_120(int deviceIndex);
SieveSlabRunFn SieveSlabGetLaunchFn_gfx1201(int deviceIndex); /* always NULL */

/* ---------------------------------------------------------------------------------- */
/* Full-map engine and pool operations (source/sieve_slab_engine.h:27-101)             */
/* ---------------------------------------------------------------------------------- */

typedef int (*SieveSlabEngineRunFn)(int deviceIndex, const uint32_t* h_primes,
                                    uint32_t numPrimes, uint64_t maxPrimeMapValue,
                                    uint8_t* h_out);

/* The whole map for values [0, maxPrimeMapValue]: h_out receives
 * (maxPrimeMapValue+1+15)>>4 bytes in the reference layout. h_primes must hold the odd
 * primes up to sqrt(maxPrimeMapValue) (2 excluded). Synchronous.
 * Replaces SieveSlabEngineRun_<arch> (source/sieve_slab_engine.cpp:115-202). */
int SieveSlabEngineRun_sm_100a(int deviceIndex, const uint32_t* h_primes, uint32_t numPrimes,
                               uint64_t maxPrimeMapValue, uint8_t* h_out);
/* source/sieve_slab_engine.cpp:209-216 */
SieveSlabEngineRunFn SieveSlabEngineGetLaunchFn_sm_100a(int deviceIndex);
int SieveSlabEngineRun_sm_120(int deviceIndex, const uint32_t* h_primes, uint32_t numPrimes,
                              uint64_t maxPrimeMapValue, uint8_t* h_out);
SieveSlabEngineRunFn SieveSlabEngineGetLaunchFn_sm_120(int deviceIndex);
SieveSlabEngineRunFn SieveSlabEngineGetLaunchFn_gfx1201(int deviceIndex); /* always NULL */

/* The pool operation table (source/sieve_slab_engine.h:49-98), same 19 members in the
 * same order. Every op makes vendorIndex the calling thread's current device first.
 * slabCompute / slabComputeAsync clear bits INTO d_slab (bitwise AND, like the reference
 * kernel), so an unprimed buffer gives the same bytes the reference would. */
typedef struct SievePoolOps {
    void* (*alloc)(int vendorIndex, uint64_t bytes);
    int (*memset)(int vendorIndex, void* d_ptr, int v, uint64_t bytes);
    int (*free)(int vendorIndex, void* d_ptr);
    int (*copyH2D)(int vendorIndex, void* d_dst, const void* h_src, uint64_t bytes);
    int (*copyD2H)(int vendorIndex, void* h_dst, const void* d_src, uint64_t bytes);
    int (*slabCompute)(int vendorIndex, const uint32_t* h_primes, uint32_t numPrimes,
                       uint64_t segLo, uint64_t segHi, void* d_slab, uint64_t slabBytes,
                       int primeSlab);
    void* (*createStream)(int vendorIndex);
    int (*destroyStream)(int vendorIndex, void* stream);
    void* (*createEvent)(int vendorIndex);
    int (*destroyEvent)(int vendorIndex, void* ev);
    int (*recordEvent)(int vendorIndex, void* ev, void* stream);
    int (*waitEvent)(int vendorIndex, void* ev, void* stream);
    int (*syncEvent)(int vendorIndex, void* ev);
    int (*elapsedEvents)(int vendorIndex, void* startEv, void* endEv, double* msOut);
    int (*allocPinned)(int vendorIndex, void** h, uint64_t bytes);
    int (*freePinned)(int vendorIndex, void* h);
    int (*copyH2DAsync)(int vendorIndex, void* d_dst, const void* h_src, uint64_t bytes,
                        void* stream);
    int (*copyD2HAsync)(int vendorIndex, void* h_dst, const void* d_src, uint64_t bytes,
                        void* stream);
    int (*slabComputeAsync)(int vendorIndex, const uint32_t* h_primes, uint32_t numPrimes,
                            uint64_t segLo, uint64_t segHi, void* d_slab, uint64_t slabBytes,
                            void* computeStream, void* waitEvent);
} SievePoolOps;

/* source/sieve_slab_engine.cpp:450-457: the table when vendorIndex is a visible device. */
const SievePoolOps* SievePoolGet_sm_100a(int vendorIndex);
const SievePoolOps* SievePoolGet_sm_120(int vendorIndex);
const SievePoolOps* SievePoolGet_gfx1201(int vendorIndex); /* always NULL */

/* ---------------------------------------------------------------------------------- */
/* M4 search (source/m4/gpu_search_kernel.cpp:31-66, gpu_search_launcher.h:43-50)      */
/* ---------------------------------------------------------------------------------- */

typedef int (*SearchKernelRunFn)(int deviceIndex, const uint8_t* d_primeMap,
                                 uint64_t d_maxPrimeMapValue, uint64_t d_sumStart,
                                 uint64_t d_sumLimit, uint32_t* d_pAtomicCount,
                                 GpuRecord* d_pRecords);

/* Evaluates the odd sums d_sumStart, d_sumStart+2, ... <= d_sumLimit (inclusive) against
 * the map (values <= d_maxPrimeMapValue answered by the map, larger ones by Miller-Rabin)
 * and writes each solution to slot (sum-d_sumStart)>>1 of d_pRecords, incrementing
 * *d_pAtomicCount. The caller zero-fills (d_sumLimit-d_sumStart)/2+1 slots and the
 * counter. Asynchronous on the legacy default stream (returns after the launch; a later
 * synchronising copy completes it). d_sumStart must be odd (every reference caller passes
 * sumStart|1). Replaces SearchKernelRun_<arch> (source/m4/gpu_search_kernel.cpp:31-51). */
int SearchKernelRun_sm_100a(int deviceIndex, const uint8_t* d_primeMap,
                            uint64_t d_maxPrimeMapValue, uint64_t d_sumStart,
                            uint64_t d_sumLimit, uint32_t* d_pAtomicCount,
                            GpuRecord* d_pRecords);
/* source/m4/gpu_search_kernel.cpp:56-66 */
SearchKernelRunFn SearchKernelGetLaunchFn_sm_100a(int deviceIndex);
int SearchKernelRun_sm_120(int deviceIndex, const uint8_t* d_primeMap,
                           uint64_t d_maxPrimeMapValue, uint64_t d_sumStart,
                           uint64_t d_sumLimit, uint32_t* d_pAtomicCount,
                           GpuRecord* d_pRecords);
SearchKernelRunFn SearchKernelGetLaunchFn_sm_120(int deviceIndex);
SearchKernelRunFn SearchKernelGetLaunchFn_gfx1201(int deviceIndex); /* always NULL */

/* vendor "nvidia" launches SearchKernelRun_sm_100a; any other vendor returns -1 (the
 * reference returns -1 when no launch function exists). Note the argument order
 * (records before counter). Replaces GpuSearchLaunch (source/m4/gpu_search_launcher.cpp:36-61). */
int GpuSearchLaunch(int deviceIndex, const char* vendor, const uint8_t* d_primeMap,
                    uint64_t d_maxPrimeMapValue, uint64_t d_sumStart, uint64_t d_sumLimit,
                    GpuRecord* d_pRecords, uint32_t* d_pAtomicCount);

/* ---------------------------------------------------------------------------------- */
/* Text output (source/m4/gpu_search_emission.cpp:34-96; reference/segmentedSieve.C:   */
/* 645-677, 816-819). The C++ PrintOutputTags / FormatGpuSearchResult / GpuSearchEmit  */
/* taking a GpuPrime are declared in gpu_prime.h.                                      */
/* ---------------------------------------------------------------------------------- */

/* One solution line (count field included, '\n'-terminated) into buf; returns its length
 * or -1 when cap is too small. lowPrime/highPrime select the " (prime)" tags. */
int ffb_format_line(uint32_t count, uint32_t sum, uint32_t low, uint32_t high, int lowPrime,
                    int highPrime, char* buf, size_t cap);

/* ---------------------------------------------------------------------------------- */
/* Extensions (no reference counterpart): stream-aware device calls and the whole     */
/* ff_sieve pipeline as one call.                                                      */
/* ---------------------------------------------------------------------------------- */

/* Geometry of `ff_sieve <sumStart> <sumLimit>` after the reference's argument handling
 * (reference/segmentedSieve.C:844-879, Prime::Prime :136-182). nargs = number of
 * positional arguments (0-2), a1/a2 their atoi() values. Writes the header lines into
 * hdr (NUL-terminated) and returns their length; -1 on error or when the reference
 * would stop with its "more memory" message (then hdr holds that message). */
typedef struct {
    uint32_t sumStart, sumLimit;
    uint64_t maxPrimeMapValue;  /* mpv after the estimate and renormalisation branches */
    uint64_t mapBytes;          /* (mpv+1+15)>>4 */
    uint64_t numPrimesRequested;
    uint64_t pmapSumLimit;      /* isqrt64((mpv-2)<<2)<<1 */
} FfbGeometry;
int ffb_geometry(int nargs, int32_t a1, int32_t a2, FfbGeometry* g, char* hdr, size_t cap);

/* The sum sub-ranges ff_seg evaluates for [sumStart, sumLimit] in emission order
 * (GenerateThreads' 62-way front/back partition, reference/segmentedSieve.C:706-792,
 * applied once or twice per main's split at :905-912), threads = THREADS (31).
 * Returns the number of ranges (firsts[i]..lasts[i], inclusive; odd sums from
 * firsts[i]|1) or -1. */
int ffb_schedule(uint32_t sumStart, uint32_t sumLimit, uint64_t maxPrimeMapValue,
                 uint32_t threads, uint32_t* firsts, uint32_t* lasts, int cap);

/* Full reference map for [0, maxPrimeMapValue] into d_map ((mpv+1+15)>>4 bytes rounded up
 * to a multiple of 16, 16-byte aligned), stream-ordered on `stream` (a cudaStream_t; NULL = legacy default). */
int ffb_sieve_map_async(int deviceIndex, uint64_t maxPrimeMapValue, uint8_t* d_map,
                        void* stream);

/* ffb_sieve_map_async with the shared-memory tile of the sieve given (1 KB..216 KB, a
 * multiple of 16; the default is 216 KB): the slab-size knob of the reference's engine
 * (--slab-size), for sweeps and tuning. */
int ffb_sieve_map_tiled_async(int deviceIndex, uint64_t maxPrimeMapValue, uint8_t* d_map,
                              uint32_t tileBytes, void* stream);

/* Packed search results for the odd sums lo..hi (lo, hi odd): d_rec[(s-lo)/2] = 0 or
 * (low | lowPrime<<31) << 32 | (high | highPrime<<31). Values <= mapBound are answered by
 * d_map, larger ones by Miller-Rabin. d_rec is zero-filled by the call. Stream-ordered. */
int ffb_search_async(int deviceIndex, const uint8_t* d_map, uint64_t mapBound, uint32_t lo,
                     uint32_t hi, uint64_t* d_rec, void* stream);

/* ffb_search_async with an explicit launch shape (no reference counterpart): `warps` warps
 * per block (4, 8, 16), `group` warps per sum (1, 2, 4) and `chunk` sums taken from the
 * work counter at a time (16, 32, 64 with one warp per sum; 32 * group otherwise). Groups and
 * chunks other than 32 need a map that covers every probe (mapBound >= ffb_probe_bound(hi)).
 * These are the candidates the batch's autotuner times; every shape gives the same records.
 * Other shapes return -1. */
int ffb_search_shape_async(int deviceIndex, const uint8_t* d_map, uint64_t mapBound, uint32_t lo,
                           uint32_t hi, uint64_t* d_rec, uint32_t warps, uint32_t chunk,
                           uint32_t group, void* stream);

/* Work done by the searches on a device since the last reset: out[0] = probes of
 * 2^k + o*b - 2 (one random map sector each), out[1] = AllButOne... evaluations.
 * Synchronises the device; reset != 0 clears the counters. */
int ffb_search_stats(int deviceIndex, uint64_t* out, int reset);

/* The smallest map bound (of the form 16m-1) at or above every value the search probes for
 * sums up to maxSum: the pair sums it tests are at most maxSum^2/12 + maxSum (the divisor 3
 * of a product below maxSum^2/4, or the even-phase pair with odd part 3), so with a map up
 * to this bound no probe needs Miller-Rabin. Returns 0 above the supported domain. */
uint64_t ffb_probe_bound(uint32_t maxSum);

/* The search of ffb_search_async without any device allocation. No counterpart in the
 * reference. For callers that cannot call cudaMalloc: a host whose device memory is owned by
 * its own pool or framework allocator (memory reserved up front, outside allocations
 * forbidden or accounted as failures), or a latency-critical caller for which an allocation
 * or a free may synchronise the device. Every value here lives in a fixed 104,912-byte array
 * compiled into the library (work counter, error word, the table of odd primes below 2^16),
 * which each GPU that loads the library holds until the process exits.
 *   - Same inputs and output as ffb_search_async: odd sums lo..hi (lo odd, hi <= 2^25; other
 *     ranges are rejected with -1 and a message), d_map/mapBound, d_rec zero-filled by the
 *     call. d_err (required, one device word) is cleared by the call and receives the error
 *     flags that ffb_take_errors would report; a NULL d_err is rejected with -1, since no
 *     other call could read the flags back.
 *   - The first call on a device sets the array up (its device address, the prime table
 *     copied in, synchronously) with that device current; make that first call before any
 *     stream capture.
 *   - Calls share the one array; it keeps the last call's contents, and the call clears the
 *     counter it needs. Calls that overlap on the GPU (different streams, same device) race
 *     on it: serialise them. */
int ffb_search_noalloc(int deviceIndex, const uint8_t* d_map, uint64_t mapBound, uint32_t lo,
                       uint32_t hi, uint64_t* d_rec, uint32_t* d_err, void* stream);

/* Measured on-chip peaks of the device (no reference counterpart): the denominators of the
 * search's integer roofline and of the sieve's marking roofline. Each figure is operations
 * per second over the whole GPU from a microbenchmark timed with CUDA events (about 0.1 s in
 * all): 32-bit multiply-adds, 32-bit ALU operations, full 64x64->128-bit products, integer
 * operations with multiply-adds and ALU operations mixed one to two, shared-memory atomicAnd
 * with the 32 lanes of a warp on distinct banks and on pseudo-random words, and plain
 * shared-memory read-modify-writes. */
typedef struct {
    double imad32PerS, alu32PerS, mul64PerS, intOpsPerS;
    double atomsConflictFreePerS, atomsRandomPerS, smemRmwPerS;
    int sms;
    double clockMhz;
} FfbPeaks;
int ffb_measure_peaks(int deviceIndex, FfbPeaks* out);

/* Reads and clears the device error flags raised by kernels (1: Miller-Rabin outside the
 * exact domain, 2: a divisor list overflowed, 4: bad launch input). Synchronises the
 * device. Returns 0 and the flags in *flags. */
int ffb_take_errors(int deviceIndex, uint32_t* flags);

/* A resident context for repeated runs: device map grown to the largest limit asked for,
 * record buffers and pinned staging. One context per thread at a time. */
typedef struct FfbContext FfbContext;
FfbContext* ffb_context_create(int deviceIndex);
void ffb_context_destroy(FfbContext* ctx);
/* Caps the bytes of the context's prime map (0, the default: 90 % of the device's free
 * memory less the job's records and the budget's scratch and headroom, as the reference's
 * computeBudget, source/budget.cpp:15-42). A job whose probes need a larger map gets the
 * largest map under the cap, and Miller-Rabin answers above it: the same output, more
 * search time. The reference caps its own map the same way (PRIMEMEM,
 * reference/segmentedSieve.C:148-176). */
int ffb_context_set_map_budget(FfbContext* ctx, uint64_t bytes);

/* A batch of ff_sieve runs (no reference counterpart): n ranges, each given as the two
 * atoi()-style arguments of `ff_sieve <sumStart> <sumLimit>`, evaluated together. One prime
 * map is sieved for the whole batch, the sums of all ranges' schedules are merged into
 * disjoint intervals that one persistent search launch takes as its work queue (each shared
 * sum evaluated once), and both launches are captured once into a CUDA graph. autotune != 0
 * times the sieve tile sizes (64..216 KB), then the search's block size (4, 8, 16 warps),
 * warps per sum (1, 2, 4) and sums per chunk (16, 32, 64 sums a warp takes from the work
 * queue at a time with one warp per sum; 32 per warp of a group) on the batch first (kept
 * per map size and sum count for later batches). Each range's text is
 * exactly what ff_seg prints for it; the timing lines carry the batch's sieve and search
 * times. Allocates its device buffers at creation. */
typedef struct FfbBatch FfbBatch;
typedef struct {
    uint32_t ranges, intervals;
    uint64_t sums;              /* distinct odd sums evaluated */
    uint64_t mapMaxValue, mapBytes;
    uint32_t sieveTileBytes, searchWarps;
    int autotuned;              /* 0 fixed defaults, 1 timed at creation, 2 reused */
    float sieveMs, searchMs;    /* device times of the last completed launch */
    uint32_t searchChunk;       /* sums per chunk of the work queue */
    uint32_t searchGroup;       /* warps per sum (1, 2 or 4) */
} FfbBatchInfo;
FfbBatch* ffb_batch_create(int deviceIndex, uint32_t n, const int32_t* starts,
                           const int32_t* limits, int autotune);
/* Replays the graph on `stream` (NULL: the batch's own stream). Asynchronous. */
int ffb_batch_launch(FfbBatch* b, void* stream);
/* Waits for the launch, copies the records back and emits every range's text into one
 * malloc'd buffer (free with ffb_free): range i is text[offsets[i] .. offsets[i+1]). */
int ffb_batch_collect(FfbBatch* b, char** text, size_t* offsets);
int ffb_batch_info(const FfbBatch* b, FfbBatchInfo* info);
void ffb_batch_destroy(FfbBatch* b);

/* ---------------------------------------------------------------------------------- */
/* Device memory budget (source/budget.h:23-46, source/budget.cpp:15-51): the         */
/* reference's DeviceBudget and its computeBudget / shrinkFractionForAlloc, as plain   */
/* functions of the free bytes (the reference reads them from a DeviceInfo).           */
/* ---------------------------------------------------------------------------------- */
typedef struct {
    double fraction;                /* f actually used */
    unsigned long long freeQueried; /* free device bytes given */
    unsigned long long freeUsed;    /* floor(f x free) */
    unsigned long long cap;         /* ~0 when uncapped */
    unsigned long long budget;      /* min(freeUsed, cap) */
    unsigned long long scratch;     /* fixed, else min(floor(0.15 x budget), 1 GiB) */
    unsigned long long headroom;    /* 64 MiB */
    unsigned long long backing;     /* budget - scratch - headroom, floored to 4 KiB */
    unsigned long long slabCount;   /* floor(backing / slab bytes) */
} FfbBudget;
/* computeBudget (source/budget.cpp:15-42). capBytes 0 = no cap (the reference's
 * hasBudgetCap false), scratchBytes 0 = the automatic scratch, slabBytes 0 = no slab count.
 * Returns -1 when fraction is outside (0, 1]. */
int ffb_compute_budget(uint64_t freeBytes, double fraction, uint64_t capBytes,
                       uint64_t scratchBytes, uint64_t slabBytes, FfbBudget* out);
/* shrinkFractionForAlloc (source/budget.cpp:44-51): the budget at the midpoint between
 * fraction and the 0.50 floor (at or below the floor: the floor itself). */
int ffb_shrink_budget(uint64_t freeBytes, double fraction, uint64_t capBytes,
                      uint64_t scratchBytes, uint64_t slabBytes, FfbBudget* out);

/* ---------------------------------------------------------------------------------- */
/* Serving loop (no reference counterpart): ff_sieve requests of any size submitted    */
/* while others run. The device keeps one prime map resident (sieved at creation up to */
/* the bound the first requests need, grown to the largest admitted limit, never past  */
/* the budget's backing bytes; Miller-Rabin answers probes above it, so every answer is */
/* the same as with the reference's own map), the factor tables and, per launch       */
/* slot, record and work-queue buffers carved from the budget's scratch bytes.          */
/* Continuous batching: whenever a launch slot is free, the scheduler fills one search  */
/* launch with a slice of every waiting request (oldest first, each request's sums in   */
/* its emission order, equal shares of the launch's work), so requests that arrive      */
/* while others are on the GPU join the next launch and their work overlaps on the      */
/* device. Each request's text is exactly ff_seg's stdout for its arguments, streamed   */
/* back in that order as chunks; its timing lines carry the sieve time its admission    */
/* caused and its time from admission to completion.                                    */
/* ---------------------------------------------------------------------------------- */
typedef struct FfbServer FfbServer;
typedef struct {
    uint64_t vramBudgetBytes;   /* budget cap (the reference's --vram-budget); 0 = none */
    double vramFraction;        /* f of the free device memory; 0 = 0.90 */
    uint32_t slots;             /* launches in flight; 0 = 4 */
    uint32_t launchWork;        /* work of one launch in odd sums at sum 2^21 (a sum s counts
                                   s/2^21); 0 = 131072 */
    uint32_t launchSums;        /* most odd sums of one launch; 0 = 2^22 */
    uint32_t searchWarps;       /* warps per search block: 4, 8 or 16; 0 = 8 */
    uint32_t warmLimit;         /* sieve the map for sums up to this at creation; 0 = none */
} FfbServeConfig;
typedef struct {
    uint64_t request;           /* id returned by ffb_serve_submit */
    uint32_t seq;               /* 0, 1, ... within the request */
    int32_t status;             /* 1 the request's last chunk, 0 more follow, -1 failed */
    char* text;                 /* malloc'd (ffb_free); the request's next bytes */
    size_t len;
} FfbServeChunk;
typedef struct {
    uint32_t sumStart, sumLimit;    /* after the reference's argument handling */
    uint64_t sums;                  /* odd sums in its schedule */
    uint64_t textBytes;             /* bytes delivered so far */
    uint64_t bodyHash;              /* FNV-1a 64 of its solution lines */
    double submitUs, admitUs, firstChunkUs, doneUs;  /* since the server's creation */
    uint32_t launches;              /* launches its sums were spread over */
    int32_t state;                  /* 0 queued, 1 running, 2 done, -1 failed */
} FfbServeRequestInfo;
typedef struct {
    FfbBudget budget;
    uint64_t mapBytes, mapMaxValue;       /* the resident map's sieved part */
    uint64_t requests, completed, failed;
    uint64_t launches, sumsRequested, sumsSearched;
    uint64_t chunks, textBytes;
    uint32_t slots, maxQueued;            /* most requests waiting at once */
    double sieveMs, searchMs;             /* device time of all sieve / search launches */
    uint64_t stage1Probes;                /* probes of 2^k + o*b - 2 */
    uint64_t stage2Items;                 /* AllButOne... evaluations */
    uint64_t mrCandidates;                /* probes above the map given to the batched
                                             Miller-Rabin (after the small-prime test) */
    uint64_t mrBase2Passed;               /* of those, strong probable primes to base 2 */
} FfbServeInfo;
/* NULL (and a stderr line) when the budget leaves no room for the map and the slots. */
FfbServer* ffb_serve_create(int deviceIndex, const FfbServeConfig* cfg);
/* Queues `ff_sieve <a1> <a2>` (nargs positional arguments); returns its id (>= 0), or -1
 * when the reference would not run the range or its sums exceed 2^25. */
int64_t ffb_serve_submit(FfbServer* s, int nargs, int32_t a1, int32_t a2);
/* The next chunk of output of any request (chunks of one request arrive in order).
 * Returns 1 with *out filled, 0 when none came within timeoutMs (< 0: wait forever). */
int ffb_serve_next(FfbServer* s, FfbServeChunk* out, int timeoutMs);
int ffb_serve_request_info(FfbServer* s, uint64_t id, FfbServeRequestInfo* out);
int ffb_serve_info(FfbServer* s, FfbServeInfo* out);
/* Waits until every submitted request has completed or failed (timeoutMs < 0: forever).
 * Returns 0, or 1 on timeout. */
int ffb_serve_drain(FfbServer* s, int timeoutMs);
/* Finishes the launches in flight, drops undelivered output and frees everything. */
void ffb_serve_destroy(FfbServer* s);

/* One slab of the prime map: the values [segLo, segHi) of ff_seg's map (every odd prime p
 * with p*p < segHi marks; the value 1 is cleared when segLo == 0) written to d_out in the
 * map's own layout, so d_out is the map's byte segLo/16 and (segHi-segLo+15)/16 bytes are
 * written (bits of values >= segHi stay 1). segLo must be a multiple of 256 (d_out 16-byte
 * aligned within the map). A sharded job sieves one slab per rank and all-gathers them; the
 * reference distributes the map's slabs over its devices the same way
 * (source/pull_scheduler.cpp:149-202). Asynchronous on `stream`. */
int ffb_sieve_map_range_async(int deviceIndex, uint64_t segLo, uint64_t segHi, uint8_t* d_out,
                              void* stream);

/* The whole `ff_sieve` / ff_seg stdout for the given arguments (see ffb_geometry), with the
 * timing lines in microseconds ("Prime time: <us> μs", "Freudenthal time: <us> μs").
 * *text receives a malloc'd buffer (free with ffb_free), *len its length. ctx may be NULL
 * (a temporary context is used). */
int ffb_run(FfbContext* ctx, int nargs, int32_t a1, int32_t a2, char** text, size_t* len);

/* `ff_seg --dump-map <file> [<sumStart>] [<sumLimit>]` (reference/segmentedSieve.C:830-839,
 * 883-897): the prime map of `ff_sieve <a1> <a2>` (see ffb_geometry), values up to its
 * maxPrimeMapValue in the reference layout, Prime::PrimeMapSize() = (maxPrimeMapValue+15)>>4
 * bytes, sieved on the device into a malloc'd host buffer (*map, free with ffb_free; *bytes
 * its size). hdr (optional) receives the header lines ff_seg prints before it dumps. */
int ffb_map_dump(int deviceIndex, int nargs, int32_t a1, int32_t a2, uint8_t** map,
                 uint64_t* bytes, char* hdr, size_t hdrCap);

/* The ff_sieve / ff_seg stdout for the given arguments from packed records already computed
 * (host memory, the format of ffb_search_async: h_rec[(s-recLo)/2] for odd sums
 * s = recLo, recLo+2, ..., covering every sum of the schedule), with the given timing
 * values in the last two lines. No device work: the host side of a job whose sums were
 * searched elsewhere, e.g. in shards on several GPUs and gathered. */
int ffb_emit(int nargs, int32_t a1, int32_t a2, const uint64_t* h_rec, uint32_t recLo,
             uint64_t nrec, double primeUs, double freudUs, char** text, size_t* len);
void ffb_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* FFB200_H */
