// peaks.cu -- measured on-chip peaks that bound the two kernels (no reference counterpart):
// the integer throughput of the SMs (the search's roofline) and the shared-memory atomic
// throughput (the sieve's marking roofline), each from a microbenchmark timed with CUDA
// events on one stream after a warm-up launch.
//
//   * imad32:  chains of 32-bit multiply-adds (IMAD), 8 independent chains per thread;
//   * alu32:   chains of 32-bit add/xor/shift-add (the integer ALU pipe);
//   * mul64:   chains of full 64x64 -> 128-bit products (__umul64hi + the low product), the
//              core of a Montgomery multiplication;
//   * mixed:   IMAD and ALU chains interleaved one to one (the issue rate of integer code
//              that uses both pipes, the search's mix);
//   * atoms_*: shared-memory atomicAnd into a 16 KB tile per block with (a) the 32 lanes of a warp on
//              32 different banks, (b) pseudo-random words (the sieve's large primes),
//              (c) plain read-modify-write stores to distinct banks (no atomic).
// Each kernel runs a persistent grid of 4 blocks x 512 threads per SM; the figures are
// operations per second over the whole GPU.
#include <cuda_runtime.h>

#include <cstdio>

#include "ffb200.h"
#include "ffb_internal.h"

namespace ffb {
namespace {

constexpr int kThreads = 512;
constexpr int kTileWords = 4096;   // 16 KB per block, 4 blocks per SM

__global__ void __launch_bounds__(kThreads) k_imad32(uint32_t* sink, uint32_t iters, uint32_t a)
{
    uint32_t x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = threadIdx.x + 977u * c + blockIdx.x;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 8; ++c) x[c] = x[c] * a + (uint32_t)c;
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) r ^= x[c];
    if (r == 0x9E3779B9u) sink[0] = r;  // keeps the chains live; never true in practice
}

__global__ void __launch_bounds__(kThreads) k_alu32(uint32_t* sink, uint32_t iters, uint32_t a)
{
    uint32_t x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = threadIdx.x + 977u * c + blockIdx.x;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 8; ++c) x[c] = (x[c] ^ a) + (x[c] >> 3);
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) r ^= x[c];
    if (r == 0x9E3779B9u) sink[0] = r;
}

__global__ void __launch_bounds__(kThreads) k_mul64(uint32_t* sink, uint32_t iters, uint64_t a)
{
    uint64_t x[4], y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        x[c] = threadIdx.x + 0x9E3779B97F4A7C15ull * (c + 1) + blockIdx.x;
        y[c] = 0;
    }
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const uint64_t lo = x[c] * a;
                const uint64_t hi = __umul64hi(x[c], a);
                x[c] = lo ^ hi;
                y[c] += hi;
            }
    }
    uint64_t r = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) r ^= x[c] ^ y[c];
    if (r == 0x9E3779B97F4A7C15ull) sink[0] = (uint32_t)r;
}

__global__ void __launch_bounds__(kThreads) k_mixed(uint32_t* sink, uint32_t iters, uint32_t a)
{
    uint32_t x[4], y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        x[c] = threadIdx.x + 977u * c + blockIdx.x;
        y[c] = x[c] ^ 0x5bd1e995u;
    }
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                x[c] = x[c] * a + (uint32_t)c;
                y[c] = (y[c] ^ a) + (y[c] >> 3);
            }
    }
    uint32_t r = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) r ^= x[c] ^ y[c];
    if (r == 0x9E3779B9u) sink[0] = r;
}

// mode 0: atomicAnd, lane l of every warp on bank l (words l + 32*j, j walking the tile);
// mode 1: atomicAnd on pseudo-random words (a per-lane linear congruential walk);
// mode 2: plain read-modify-write on the words of mode 0 (each word owned by one thread).
__global__ void __launch_bounds__(kThreads) k_atoms(uint32_t* sink, uint32_t iters, int mode)
{
    __shared__ uint32_t tile[kTileWords];
    constexpr uint32_t kMask = kTileWords - 1;
    for (uint32_t w = threadIdx.x; w <= kMask; w += blockDim.x) tile[w] = 0xFFFFFFFFu;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t st = threadIdx.x * 2654435761u + blockIdx.x;
    uint32_t j = warp * 32;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            if (mode == 1) {
                st = st * 1664525u + 1013904223u;
                atomicAnd(&tile[(st >> 10) & kMask], ~(1u << (st & 31)));
            } else {
                const uint32_t w = (lane + 32 * j) & kMask;
                if (mode == 0) atomicAnd(&tile[w], ~(1u << (u & 31)));
                else tile[w] &= ~(1u << (u & 31));
                j += 17;   // odd: every warp's row walk covers the tile
            }
        }
    }
    __syncthreads();
    if (tile[threadIdx.x & kMask] == 0x12345u) sink[0] = 1;
}

template <typename K, typename... Args>
float time_kernel(K kern, int blocks, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, Args... args)
{
    kern<<<blocks, kThreads, 0, st>>>(args...);  // warm-up
    cudaEventRecord(e0, st);
    kern<<<blocks, kThreads, 0, st>>>(args...);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -1;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" int ffb_measure_peaks(int deviceIndex, FfbPeaks* out)
{
    if (!out) return -1;
    FFB_CUDA(cudaSetDevice(deviceIndex));
    int sms = 0, clk_khz = 0;
    FFB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, deviceIndex));
    cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, deviceIndex);
    uint32_t* sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    FFB_CUDA(cudaMalloc(&sink, 64));
    int rc = 0;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = -1;
    } else {
        const int blocks = 4 * sms;
        const double threads = (double)blocks * kThreads;
        const uint32_t it = 2048;
        float ms;
        // operations per thread: iters x 16 x chains (x 1 multiply-add each)
        ms = time_kernel(k_imad32, blocks, st, e0, e1, sink, it, 0x01000193u);
        out->imad32PerS = ms > 0 ? threads * it * 16 * 8 / (ms * 1e-3) : 0;
        ms = time_kernel(k_alu32, blocks, st, e0, e1, sink, it, 0x01000193u);
        // two ALU operations per step (xor, shift-add)
        out->alu32PerS = ms > 0 ? threads * it * 16 * 8 * 2 / (ms * 1e-3) : 0;
        ms = time_kernel(k_mul64, blocks, st, e0, e1, sink, it / 2, 0x9E3779B97F4A7C15ull);
        out->mul64PerS = ms > 0 ? threads * (it / 2) * 8 * 4 / (ms * 1e-3) : 0;
        ms = time_kernel(k_mixed, blocks, st, e0, e1, sink, it, 0x01000193u);
        // per step: one IMAD + two ALU operations
        out->intOpsPerS = ms > 0 ? threads * it * 16 * 4 * 3 / (ms * 1e-3) : 0;
        const uint32_t ia = 256;
        ms = time_kernel(k_atoms, blocks, st, e0, e1, sink, ia, 0);
        out->atomsConflictFreePerS = ms > 0 ? threads * ia * 16 / (ms * 1e-3) : 0;
        ms = time_kernel(k_atoms, blocks, st, e0, e1, sink, ia, 1);
        out->atomsRandomPerS = ms > 0 ? threads * ia * 16 / (ms * 1e-3) : 0;
        ms = time_kernel(k_atoms, blocks, st, e0, e1, sink, ia, 2);
        out->smemRmwPerS = ms > 0 ? threads * ia * 16 / (ms * 1e-3) : 0;
        out->sms = sms;
        out->clockMhz = clk_khz / 1000.0;
        if (cudaGetLastError() != cudaSuccess) rc = -1;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(sink);
    return rc;
}
