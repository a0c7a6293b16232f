// search_noalloc.cu -- ffb_search_noalloc: the Freudenthal search without any device
// allocation, for callers that must not call cudaMalloc.
//
// The ordinary entry points keep their work counter, error flags and the trial-division
// table in device memory allocated on first use of a GPU. This variant keeps the counter
// and the table in one file-scope array compiled into the library instead, and writes the
// error flags to a word the caller passes, so a call only memsets, launches and returns.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "ffb200.h"
#include "ffb_internal.h"
#include "../host/plan.h"

namespace ffb {
namespace {

constexpr uint32_t kTablePrimes = 6541;     // the odd primes below 2^16
constexpr size_t kTableOffset = 256;        // after the work counter
constexpr size_t kScratchBytes = kTableOffset + sizeof(TDiv) * kTablePrimes;  // 104,912 bytes
constexpr int kMaxDevices = 64;

// Layout: bytes [0,4) the search's work counter, [4,256) unused (the error flags go to the
// caller's word), [256, ...) the
// exact-division table of the odd primes below 2^16. Present on every GPU that loads the
// library, for the life of the process. Host code must not use this name as a device
// address: the address comes from cudaGetSymbolAddress in setup() below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct Ready {
    bool ok;
    unsigned char* scratch;  // device address of g_noalloc_scratch on this GPU
    int sms;
};
Ready g_ready[kMaxDevices];
std::mutex g_mu;
TDiv g_host_table[kTablePrimes];   // host staging of the table (static: no heap either)
bool g_odd_composite[32768];       // odd n < 65536 at index n/2

// One-time set-up of device `dev`, which the caller has made current: the scratch
// address, the table copied in, the SM count.
int setup(int dev)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        std::fprintf(stderr, "ffb_search_noalloc: cudaGetSymbolAddress failed on device %d: %s\n",
                     dev, cudaGetErrorString(e));
        return -1;
    }
    uint32_t n = 0;
    for (uint32_t q = 3; q < 65536; q += 2) {
        if (g_odd_composite[q >> 1]) continue;
        for (uint32_t m = q * q; m < 65536; m += 2 * q) g_odd_composite[m >> 1] = true;
        uint32_t inv = q;  // Newton: inverse of q modulo 2^32
        for (int k = 0; k < 4; ++k) inv *= 2 - q * inv;
        if (n < kTablePrimes) g_host_table[n] = {q, inv, 0xFFFFFFFFu / q, 0};
        ++n;
    }
    if (n != kTablePrimes) {
        std::fprintf(stderr, "ffb_search_noalloc: prime table has %u entries, expected %u\n", n,
                     kTablePrimes);
        return -1;
    }
    e = cudaMemcpyToSymbol(g_noalloc_scratch, g_host_table, sizeof(g_host_table), kTableOffset,
                           cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ffb_search_noalloc: table upload failed on device %d: %s\n", dev,
                     cudaGetErrorString(e));
        return -1;
    }
    int sms = 0, major = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        major < 10) {
        std::fprintf(stderr, "ffb_search_noalloc: device %d is not an sm_100a device\n", dev);
        cudaGetLastError();
        return -1;
    }
    g_ready[dev] = {true, static_cast<unsigned char*>(p), sms};
    return 0;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" int ffb_search_noalloc(int deviceIndex, const uint8_t* d_map, uint64_t mapBound,
                                  uint32_t lo, uint32_t hi, uint64_t* d_rec, uint32_t* d_err,
                                  void* stream)
{
    if (!(lo & 1) || hi < lo || hi > kMaxSum || !d_map || !d_rec || !d_err) {
        std::fprintf(stderr,
                     "ffb_search_noalloc: sums [%u, %u] rejected: need an odd first sum, last >= "
                     "first, last <= 2^25 (%u), and non-null map, record and error-word "
                     "pointers\n",
                     lo, hi, kMaxSum);
        return -1;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || deviceIndex < 0 ||
        deviceIndex >= count || deviceIndex >= kMaxDevices) {
        cudaGetLastError();
        std::fprintf(stderr, "ffb_search_noalloc: no CUDA device %d\n", deviceIndex);
        return -1;
    }
    FFB_CUDA(cudaSetDevice(deviceIndex));
    Ready r;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_ready[deviceIndex].ok && setup(deviceIndex)) return -1;
        r = g_ready[deviceIndex];
    }
    hi -= !(hi & 1);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SearchArgs a;
    a.map = d_map;
    a.bound = mapBound;
    a.lo = lo;
    a.hi = hi;
    a.nsums = (hi - lo) / 2 + 1;
    a.rec = d_rec;
    a.grec = nullptr;
    a.grec_base = lo;
    a.gcount = nullptr;
    a.tdiv = reinterpret_cast<const TDiv*>(r.scratch + kTableOffset);
    a.ntdiv = kTablePrimes;
    a.sched = reinterpret_cast<uint32_t*>(r.scratch);
    a.err = d_err;
    a.stats = nullptr;
    // the scratch keeps the previous call's counter: start this one from zero
    FFB_CUDA(cudaMemsetAsync(r.scratch, 0, 8, st));
    FFB_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    FFB_CUDA(cudaMemsetAsync(d_rec, 0, 8ull * a.nsums, st));
    return launch_search(a, r.sms, st);
}
