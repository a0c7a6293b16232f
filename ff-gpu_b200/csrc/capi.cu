// capi.cu -- the C ABI (include/ffb200.h): the reference's sieve / engine / pool / M4 search
// entry points over the sm_100a kernels, plus the stream-aware extensions.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "ffb200.h"
#include "ffb_internal.h"
#include "../host/plan.h"

namespace ffb {

namespace {
constexpr int kMaxDevices = 64;
constexpr int kSchedSlots = 64;
DeviceState g_states[kMaxDevices];
std::mutex g_state_mu;
unsigned g_sched_next[kMaxDevices];

// The terms the search factors are below its largest sum, at most 2^25 + 1.
constexpr uint32_t kSpfLimit = (1u << 25) + 2;

// spf[i] for the odd n = 2i + 1: the index in tdiv of n's smallest prime factor, 0xFFFF for
// 1 and the primes (a composite below kSpfLimit has a factor below 5,793, inside the table).
__global__ void build_spf(const TDiv* tdiv, uint32_t ntdiv, uint16_t* spf, uint32_t nodd)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nodd; i += gridDim.x * blockDim.x) {
        const uint32_t n = 2 * i + 1;
        uint16_t r = 0xFFFF;
        for (uint32_t k = 0; k < ntdiv; ++k) {
            const TDiv t = tdiv[k];
            if ((uint64_t)t.p * t.p > n) break;
            if (n * t.inv <= t.lim) {
                r = (uint16_t)k;
                break;
            }
        }
        spf[i] = r;
    }
}

bool device_visible(int dev)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return dev >= 0 && dev < n;
}
}  // namespace

DeviceState* device_state(int dev)
{
    if (dev < 0 || dev >= kMaxDevices || !device_visible(dev)) {
        std::fprintf(stderr, "ffb: no CUDA device %d\n", dev);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_state_mu);
    DeviceState& s = g_states[dev];
    if (s.device == dev) return &s;
    if (cudaSetDevice(dev) != cudaSuccess) return nullptr;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return nullptr;
    if (prop.major < 10) {
        std::fprintf(stderr, "ffb: device %d is sm_%d%d; this build runs on sm_100a\n", dev,
                     prop.major, prop.minor);
        return nullptr;
    }
    // trial-division table: odd primes below 65536 with exact-division constants
    uint32_t* pr = nullptr;
    uint32_t npr = 0;
    host_odd_primes(65535, &pr, &npr);
    std::vector<TDiv> t(npr);
    for (uint32_t i = 0; i < npr; ++i) {
        const uint32_t p = pr[i];
        uint32_t inv = p;  // Newton: inverse of p modulo 2^32
        for (int k = 0; k < 4; ++k) inv *= 2 - p * inv;
        t[i] = {p, inv, 0xFFFFFFFFu / p, 0};
    }
    std::free(pr);
    TDiv* dt = nullptr;
    uint32_t* words = nullptr;
    if (cudaMalloc(&dt, sizeof(TDiv) * npr) != cudaSuccess ||
        cudaMemcpy(dt, t.data(), sizeof(TDiv) * npr, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&words, 4 * (kSchedSlots + 64)) != cudaSuccess ||
        cudaMemset(words, 0, 4 * (kSchedSlots + 64)) != cudaSuccess) {
        std::fprintf(stderr, "ffb: device %d state allocation failed\n", dev);
        cudaGetLastError();
        return nullptr;
    }
    // the smallest-prime-factor table, made once on the device (a few milliseconds)
    const uint32_t nodd = kSpfLimit / 2;
    uint16_t* spf = nullptr;
    if (cudaMalloc(&spf, sizeof(uint16_t) * nodd) != cudaSuccess) {
        std::fprintf(stderr, "ffb: device %d state allocation failed\n", dev);
        cudaGetLastError();
        return nullptr;
    }
    build_spf<<<prop.multiProcessorCount * 8, 256>>>(dt, npr, spf, nodd);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        std::fprintf(stderr, "ffb: device %d factor table failed\n", dev);
        return nullptr;
    }
    s.spf = spf;
    s.spf_limit = kSpfLimit;
    s.sms = prop.multiProcessorCount;
    s.tdiv = dt;
    s.ntdiv = npr;
    s.words = words;
    s.device = dev;
    return &s;
}

// A scheduler counter for one launch (slots rotate so concurrent streams do not share).
static uint32_t* sched_slot(DeviceState* s)
{
    std::lock_guard<std::mutex> lk(g_state_mu);
    const unsigned i = g_sched_next[s->device]++ % kSchedSlots;
    return s->words + i;
}
static uint32_t* err_word(DeviceState* s) { return s->words + kSchedSlots; }
// two 64-bit work counters of the search, 8-byte aligned after the error word
static unsigned long long* stats_words(DeviceState* s)
{
    return reinterpret_cast<unsigned long long*>(s->words + kSchedSlots + 2);
}

// Search over odd sums lo..hi into packed records and/or GpuRecord slots.
int run_search(int dev, const uint8_t* d_map, uint64_t bound, uint32_t lo, uint32_t hi,
               uint64_t* d_rec, void* grec, uint32_t grec_base, uint32_t* gcount,
               cudaStream_t stream, uint32_t warps, uint32_t chunk, uint32_t group)
{
    if (!(lo & 1) || hi < lo || hi >= (1u << 25) + 1 || !d_map) {
        std::fprintf(stderr, "ffb: search range [%u, %u] not supported (odd sums up to 2^25)\n",
                     lo, hi);
        return -1;
    }
    DeviceState* s = device_state(dev);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(dev));
    hi -= !(hi & 1);
    SearchArgs a;
    a.map = d_map;
    a.bound = bound;
    a.lo = lo;
    a.hi = hi;
    a.nsums = (hi - lo) / 2 + 1;
    a.rec = d_rec;
    a.grec = grec;
    a.grec_base = grec_base;
    a.gcount = gcount;
    a.tdiv = s->tdiv;
    a.ntdiv = s->ntdiv;
    a.spf = s->spf;
    a.spf_limit = s->spf_limit;
    a.sched = sched_slot(s);
    a.err = err_word(s);
    a.stats = stats_words(s);
    a.warps = warps;
    a.chunk = chunk;
    a.group = group;
    if (d_rec) FFB_CUDA(cudaMemsetAsync(d_rec, 0, 8ull * a.nsums, stream));
    FFB_CUDA(cudaMemsetAsync(a.sched, 0, 4, stream));
    return launch_search(a, s->sms, stream);
}

int run_sieve(int dev, const uint32_t* h_primes, uint32_t n, uint64_t seg_lo, uint64_t seg_hi,
              uint8_t* d_out, cudaStream_t stream, int clear_one, uint32_t tile_bytes)
{
    DeviceState* s = device_state(dev);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(dev));
    SieveArgs a;
    a.out = d_out;
    a.seg_lo = seg_lo;
    a.seg_hi = seg_hi;
    a.h_primes = h_primes;
    a.nprimes = n;
    a.tile_bytes = tile_bytes;
    a.clear_one = clear_one;
    return launch_sieve(a, s->sms, err_word(s), stream);
}

int run_sieve_map(int dev, uint64_t seg_lo, uint64_t seg_hi, uint8_t* d_out, cudaStream_t stream,
                  int clear_one, uint32_t tile_bytes)
{
    DeviceState* s = device_state(dev);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(dev));
    SieveArgs a;
    a.out = d_out;
    a.seg_lo = seg_lo;
    a.seg_hi = seg_hi;
    a.tile_bytes = tile_bytes;
    a.clear_one = clear_one;
    a.true_map = 1;
    return launch_sieve(a, s->sms, err_word(s), stream);
}

uint32_t* device_err_word(DeviceState* s) { return err_word(s); }

}  // namespace ffb

using namespace ffb;

// ---------------------------------------------------------------------------------------
// sieve slab
// ---------------------------------------------------------------------------------------
extern "C" int SieveSlabRun_sm_100a(int deviceIndex, const uint32_t* h_primes, uint32_t numPrimes,
                                    uint64_t segLo, uint64_t segHi, uint8_t* h_out)
{
    if (segHi < segLo) return -1;
    DeviceState* s = device_state(deviceIndex);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(deviceIndex));
    const uint64_t bytes = (segHi + 15) >> 4;
    uint8_t* d = nullptr;
    FFB_CUDA(cudaMalloc(&d, (bytes + 15) & ~15ull));  // word-granular marks stay inside
    int rc = 0;
    if (cudaMemset(d, 0xff, bytes) != cudaSuccess) rc = -1;
    if (!rc && segHi > segLo) rc = run_sieve(deviceIndex, h_primes, numPrimes, segLo, segHi, d, 0, 1);
    if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = -1;
    if (!rc && bytes && cudaMemcpy(h_out, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = -1;
    cudaFree(d);
    if (rc) {
        std::fprintf(stderr, "ffb: SieveSlabRun failed: %s\n", cudaGetErrorString(cudaGetLastError()));
    }
    return rc;
}

extern "C" SieveSlabRunFn SieveSlabGetLaunchFn_sm_100a(int deviceIndex)
{
    return device_visible(deviceIndex) ? &SieveSlabRun_sm_100a : nullptr;
}
extern "C" int SieveSlabRun_sm_120(int d, const uint32_t* p, uint32_t n, uint64_t lo, uint64_t hi,
                                   uint8_t* out)
{
    return SieveSlabRun_sm_100a(d, p, n, lo, hi, out);
}
extern "C" SieveSlabRunFn SieveSlabGetLaunchFn_sm_120(int d) { return SieveSlabGetLaunchFn_sm_100a(d); }
extern "C" SieveSlabRunFn SieveSlabGetLaunchFn_gfx1201(int) { return nullptr; }

// ---------------------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------------------
extern "C" int SieveSlabEngineRun_sm_100a(int deviceIndex, const uint32_t* h_primes,
                                          uint32_t numPrimes, uint64_t maxPrimeMapValue,
                                          uint8_t* h_out)
{
    DeviceState* s = device_state(deviceIndex);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(deviceIndex));
    const uint64_t bytes = (maxPrimeMapValue + 1 + 15) >> 4;
    uint8_t* d = nullptr;
    FFB_CUDA(cudaMalloc(&d, (bytes + 15) & ~15ull));
    int rc = run_sieve(deviceIndex, h_primes, numPrimes, 0, maxPrimeMapValue + 1, d, 0, 1);
    if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = -1;
    if (!rc && cudaMemcpy(h_out, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = -1;
    cudaFree(d);
    if (rc) std::fprintf(stderr, "ffb: SieveSlabEngineRun failed\n");
    return rc;
}
extern "C" SieveSlabEngineRunFn SieveSlabEngineGetLaunchFn_sm_100a(int d)
{
    return device_visible(d) ? &SieveSlabEngineRun_sm_100a : nullptr;
}
extern "C" int SieveSlabEngineRun_sm_120(int d, const uint32_t* p, uint32_t n, uint64_t mpv, uint8_t* o)
{
    return SieveSlabEngineRun_sm_100a(d, p, n, mpv, o);
}
extern "C" SieveSlabEngineRunFn SieveSlabEngineGetLaunchFn_sm_120(int d)
{
    return SieveSlabEngineGetLaunchFn_sm_100a(d);
}
extern "C" SieveSlabEngineRunFn SieveSlabEngineGetLaunchFn_gfx1201(int) { return nullptr; }

// ---------------------------------------------------------------------------------------
// pool operations (source/sieve_slab_engine.cpp:240-457)
// ---------------------------------------------------------------------------------------
namespace ffb_pool {

#define POOL_CHECK(call)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            std::fprintf(stderr, "ffb pool: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return -1;                                                                    \
        }                                                                                 \
    } while (0)

void* pool_alloc(int v, uint64_t bytes)
{
    void* p = nullptr;
    if (cudaSetDevice(v) != cudaSuccess || cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}
int pool_memset(int v, void* d, int x, uint64_t bytes)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaMemset(d, x, bytes));
    POOL_CHECK(cudaDeviceSynchronize());
    return 0;
}
int pool_free(int v, void* d)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaFree(d));
    return 0;
}
int pool_h2d(int v, void* d, const void* h, uint64_t bytes)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice));
    return 0;
}
int pool_d2h(int v, void* h, const void* d, uint64_t bytes)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost));
    return 0;
}
// Sieves [segLo, segHi) into d_slab AND-wise: the tile result is computed into a 16-byte
// aligned scratch and ANDed into the slab, so the bytes equal the reference kernel's
// clears on whatever the slab held.
int slab_and_into(int v, const uint32_t* h_primes, uint32_t n, uint64_t lo, uint64_t hi,
                  uint8_t* d_slab, cudaStream_t st);
int pool_slab(int v, const uint32_t* h_primes, uint32_t n, uint64_t lo, uint64_t hi, void* d_slab,
              uint64_t slab_bytes, int prime)
{
    POOL_CHECK(cudaSetDevice(v));
    if (prime) {
        POOL_CHECK(cudaMemset(d_slab, 0xff, slab_bytes));
        if (lo == 0) POOL_CHECK(cudaMemset(d_slab, 0x7f, 1));
    }
    if (slab_and_into(v, h_primes, n, lo, hi, (uint8_t*)d_slab, 0)) return -1;
    POOL_CHECK(cudaDeviceSynchronize());
    return 0;
}
void* pool_stream(int v)
{
    cudaStream_t s = nullptr;
    if (cudaSetDevice(v) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return nullptr;
    return (void*)s;
}
int pool_stream_destroy(int v, void* s)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaStreamDestroy((cudaStream_t)s));
    return 0;
}
void* pool_event(int v)
{
    cudaEvent_t e = nullptr;
    if (cudaSetDevice(v) != cudaSuccess || cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return (void*)e;
}
int pool_event_destroy(int v, void* e)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaEventDestroy((cudaEvent_t)e));
    return 0;
}
int pool_record(int v, void* e, void* s)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaEventRecord((cudaEvent_t)e, (cudaStream_t)s));
    return 0;
}
int pool_wait(int v, void* e, void* s)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaStreamWaitEvent((cudaStream_t)s, (cudaEvent_t)e, 0));
    return 0;
}
int pool_sync_event(int v, void* e)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaEventSynchronize((cudaEvent_t)e));
    return 0;
}
int pool_elapsed(int v, void* a, void* b, double* ms)
{
    float f = 0;
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaEventElapsedTime(&f, (cudaEvent_t)a, (cudaEvent_t)b));
    *ms = f;
    return 0;
}
int pool_alloc_pinned(int v, void** h, uint64_t bytes)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaMallocHost(h, bytes));
    return 0;
}
int pool_free_pinned(int v, void* h)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaFreeHost(h));
    return 0;
}
int pool_h2d_async(int v, void* d, const void* h, uint64_t bytes, void* s)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, (cudaStream_t)s));
    return 0;
}
int pool_d2h_async(int v, void* h, const void* d, uint64_t bytes, void* s)
{
    POOL_CHECK(cudaSetDevice(v));
    POOL_CHECK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)s));
    return 0;
}
int pool_slab_async(int v, const uint32_t* h_primes, uint32_t n, uint64_t lo, uint64_t hi,
                    void* d_slab, uint64_t, void* stream, void* wait)
{
    POOL_CHECK(cudaSetDevice(v));
    if (wait) POOL_CHECK(cudaStreamWaitEvent((cudaStream_t)stream, (cudaEvent_t)wait, 0));
    return slab_and_into(v, h_primes, n, lo, hi, (uint8_t*)d_slab, (cudaStream_t)stream);
}

__global__ void and_bytes(uint8_t* dst, const uint8_t* src, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] &= src[i];
}

int slab_and_into(int v, const uint32_t* h_primes, uint32_t n, uint64_t lo, uint64_t hi,
                  uint8_t* d_slab, cudaStream_t st)
{
    if (hi <= lo) return 0;
    const uint64_t bytes = (hi - lo + 15) >> 4;
    uint8_t* tmp = nullptr;
    POOL_CHECK(cudaMallocAsync((void**)&tmp, (bytes + 15) & ~15ull, st));
    // clear_one = 0: the reference kernel never clears the bit of the value 1 itself
    int rc = run_sieve(v, h_primes, n, lo, hi, tmp, st, 0);
    if (!rc) {
        unsigned g = (unsigned)((bytes + 255) / 256);
        if (g > 65535) g = 65535;
        and_bytes<<<g, 256, 0, st>>>(d_slab, tmp, bytes);
        if (cudaGetLastError() != cudaSuccess) rc = -1;
    }
    cudaFreeAsync(tmp, st);
    return rc;
}

const SievePoolOps kPool = {
    pool_alloc,  pool_memset,        pool_free,      pool_h2d,      pool_d2h,
    pool_slab,   pool_stream,        pool_stream_destroy, pool_event, pool_event_destroy,
    pool_record, pool_wait,          pool_sync_event, pool_elapsed,  pool_alloc_pinned,
    pool_free_pinned, pool_h2d_async, pool_d2h_async, pool_slab_async};

}  // namespace ffb_pool

extern "C" const SievePoolOps* SievePoolGet_sm_100a(int v) { return device_visible(v) ? &ffb_pool::kPool : nullptr; }
extern "C" const SievePoolOps* SievePoolGet_sm_120(int v) { return SievePoolGet_sm_100a(v); }
extern "C" const SievePoolOps* SievePoolGet_gfx1201(int) { return nullptr; }

// ---------------------------------------------------------------------------------------
// M4 search
// ---------------------------------------------------------------------------------------
extern "C" int SearchKernelRun_sm_100a(int deviceIndex, const uint8_t* d_primeMap,
                                       uint64_t d_maxPrimeMapValue, uint64_t d_sumStart,
                                       uint64_t d_sumLimit, uint32_t* d_pAtomicCount,
                                       GpuRecord* d_pRecords)
{
    if (d_sumLimit < d_sumStart || !(d_sumStart & 1) || d_sumLimit > (1u << 25)) {
        std::fprintf(stderr, "ffb: SearchKernelRun: sums [%llu, %llu] not supported (odd "
                     "sumStart, sumLimit <= 2^25)\n", (unsigned long long)d_sumStart,
                     (unsigned long long)d_sumLimit);
        return -1;
    }
    return run_search(deviceIndex, d_primeMap, d_maxPrimeMapValue, (uint32_t)d_sumStart,
                      (uint32_t)d_sumLimit, nullptr, d_pRecords, (uint32_t)d_sumStart,
                      d_pAtomicCount, 0);
}
extern "C" SearchKernelRunFn SearchKernelGetLaunchFn_sm_100a(int d)
{
    return device_visible(d) ? &SearchKernelRun_sm_100a : nullptr;
}
extern "C" int SearchKernelRun_sm_120(int d, const uint8_t* m, uint64_t mpv, uint64_t s, uint64_t l,
                                      uint32_t* c, GpuRecord* r)
{
    return SearchKernelRun_sm_100a(d, m, mpv, s, l, c, r);
}
extern "C" SearchKernelRunFn SearchKernelGetLaunchFn_sm_120(int d) { return SearchKernelGetLaunchFn_sm_100a(d); }
extern "C" SearchKernelRunFn SearchKernelGetLaunchFn_gfx1201(int) { return nullptr; }

extern "C" int GpuSearchLaunch(int deviceIndex, const char* vendor, const uint8_t* d_primeMap,
                               uint64_t d_maxPrimeMapValue, uint64_t d_sumStart,
                               uint64_t d_sumLimit, GpuRecord* d_pRecords, uint32_t* d_pAtomicCount)
{
    if (!vendor || std::strcmp(vendor, "nvidia") != 0) return -1;
    SearchKernelRunFn fn = SearchKernelGetLaunchFn_sm_100a(deviceIndex);
    if (!fn) return -1;
    return fn(deviceIndex, d_primeMap, d_maxPrimeMapValue, d_sumStart, d_sumLimit, d_pAtomicCount,
              d_pRecords);
}

// ---------------------------------------------------------------------------------------
// extensions
// ---------------------------------------------------------------------------------------
extern "C" int ffb_sieve_map_async(int deviceIndex, uint64_t mpv, uint8_t* d_map, void* stream)
{
    return run_sieve_map(deviceIndex, 0, mpv + 1, d_map, (cudaStream_t)stream, 1);
}

extern "C" int ffb_sieve_map_range_async(int deviceIndex, uint64_t segLo, uint64_t segHi,
                                         uint8_t* d_out, void* stream)
{
    if (segLo & 255) {
        std::fprintf(stderr, "ffb_sieve_map_range_async: segLo %llu is not a multiple of 256\n",
                     (unsigned long long)segLo);
        return -1;
    }
    if (segHi <= segLo) return 0;
    return run_sieve_map(deviceIndex, segLo, segHi, d_out, (cudaStream_t)stream, segLo == 0);
}

extern "C" int ffb_sieve_map_tiled_async(int deviceIndex, uint64_t mpv, uint8_t* d_map,
                                         uint32_t tileBytes, void* stream)
{
    if (tileBytes < 1024 || tileBytes > 216 * 1024 || (tileBytes & 15)) {
        std::fprintf(stderr, "ffb_sieve_map_tiled_async: tile of %u bytes outside 1 KB..216 KB "
                     "(multiple of 16)\n", tileBytes);
        return -1;
    }
    return run_sieve_map(deviceIndex, 0, mpv + 1, d_map, (cudaStream_t)stream, 1, tileBytes);
}

extern "C" int ffb_search_async(int deviceIndex, const uint8_t* d_map, uint64_t mapBound,
                                uint32_t lo, uint32_t hi, uint64_t* d_rec, void* stream)
{
    return run_search(deviceIndex, d_map, mapBound, lo, hi, d_rec, nullptr, 0, nullptr,
                      (cudaStream_t)stream);
}

extern "C" int ffb_search_shape_async(int deviceIndex, const uint8_t* d_map, uint64_t mapBound,
                                      uint32_t lo, uint32_t hi, uint64_t* d_rec, uint32_t warps,
                                      uint32_t chunk, uint32_t group, void* stream)
{
    if ((warps != 4 && warps != 8 && warps != 16) || (group != 1 && group != 2 && group != 4)) {
        std::fprintf(stderr, "ffb_search_shape_async: %u warps per block, %u per sum not offered\n",
                     warps, group);
        return -1;
    }
    return run_search(deviceIndex, d_map, mapBound, lo, hi, d_rec, nullptr, 0, nullptr,
                      (cudaStream_t)stream, warps, chunk, group);
}

extern "C" int ffb_search_stats(int deviceIndex, uint64_t* out, int reset)
{
    DeviceState* s = device_state(deviceIndex);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(deviceIndex));
    FFB_CUDA(cudaDeviceSynchronize());
    FFB_CUDA(cudaMemcpy(out, stats_words(s), 16, cudaMemcpyDeviceToHost));
    if (reset) FFB_CUDA(cudaMemset(stats_words(s), 0, 32));
    return 0;
}

extern "C" uint64_t ffb_probe_bound(uint32_t maxSum)
{
    if (maxSum > kMaxSum) return 0;
    const uint64_t s = maxSum;
    const uint64_t v = s * s / 12 + s + 16;
    return ((v >> 4) << 4) | 15;  // 16m-1: whole bytes of the map
}

extern "C" int ffb_take_errors(int deviceIndex, uint32_t* flags)
{
    DeviceState* s = device_state(deviceIndex);
    if (!s) return -1;
    FFB_CUDA(cudaSetDevice(deviceIndex));
    FFB_CUDA(cudaDeviceSynchronize());
    uint32_t f = 0;
    FFB_CUDA(cudaMemcpy(&f, err_word(s), 4, cudaMemcpyDeviceToHost));
    FFB_CUDA(cudaMemset(err_word(s), 0, 4));
    *flags = f;
    return 0;
}
