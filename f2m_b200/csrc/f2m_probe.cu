// Throughput probe of the FP64 pipe (diagnostics; no counterpart in the
// reference).  The dual descent spends its issue slots on FP64 additions
// (reduced costs, potential updates) and FP64 compares (the top-3 insertion),
// so its roofline is the FP64 pipe's instruction rate, not HBM.  This probe
// measures that rate on the GPU it runs on: every thread runs independent
// dependency chains so that the pipe, not latency, bounds the loop.
//
//   kind 0: DADD only, 8 independent chains per thread;
//   kind 1: DSETP-dominated: per round one DADD moves the threshold and eight
//           compares against it feed integer counters (the integer pipe has
//           twice the FP64 lane rate, so the compares bound the loop).
#include <cuda_runtime.h>
#include <stdint.h>

#include "f2m_device.cuh"
#include "f2m_internal.h"

namespace f2m {

constexpr int kProbeThreads = 256;

template <int KIND>
__global__ void __launch_bounds__(kProbeThreads) k_fp64_rate(double* out, int iters, double seed) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = seed * (double)(threadIdx.x + 1) + (double)i;
    const double d = seed * 1e-3;
    if (KIND == 0) {
#pragma unroll 4
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = a[i] + d;
        }
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += a[i];
        if (s == 1.25) out[blockIdx.x] = s;  // keeps the chains live; never true for these seeds
    } else {
        int cnt[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) cnt[i] = 0;
        double t = seed;
#pragma unroll 4
        for (int it = 0; it < iters; ++it) {
            t = t + d;
#pragma unroll
            for (int i = 0; i < 8; ++i) cnt[i] += (a[i] < t) ? 1 : 0;
        }
        int s = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += cnt[i];
        if (s == -1) out[blockIdx.x] = t;  // never true: counts are >= 0
    }
}

// FP64 lane operations per launch of kind `kind` with `blocks` CTAs.
double fp64_probe_ops(int kind, int blocks, int iters) {
    const double per_iter = (kind == 0) ? 8.0 : 9.0;  // kind 1: 8 DSETP + 1 DADD
    return per_iter * (double)iters * (double)blocks * kProbeThreads;
}

cudaError_t launch_fp64_probe(int kind, int blocks, int iters, double* out, cudaStream_t s) {
    if (kind == 0) k_fp64_rate<0><<<blocks, kProbeThreads, 0, s>>>(out, iters, 0.37);
    else k_fp64_rate<1><<<blocks, kProbeThreads, 0, s>>>(out, iters, 0.37);
    return cudaGetLastError();
}

// Self-check of the warp-cooperative partition (diagnostics): every warp
// draws seeded lists (sizes 0-128, values from a few levels so that ties and
// runs are common, thresholds that force the raise-by-one loop, an
// occasional NaN), partitions one copy with the serial loop (qpart_ef_vals,
// lane 0) and one with warp_qpart_ef_vals, and counts the lists whose final
// order or count differ.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
constexpr int kPcWarps = 8;
constexpr int kPcCap = 128;
__global__ void __launch_bounds__(32 * kPcWarps) k_partition_check(int n_cases, unsigned long long seed,
                                                                    unsigned long long* bad) {
    __shared__ double sv[kPcWarps][3][kPcCap];
    __shared__ uint16_t sp[kPcWarps][3][kPcCap];
    __shared__ uint8_t spos[kPcWarps][kPcCap];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = blockIdx.x * kPcWarps + w;
    if (cs >= n_cases) return;
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)cs));
    const int kind = (int)(h % 5);
    const int size = (kind == 4) ? (int)((h >> 8) % 6) : (int)((h >> 8) % (kPcCap + 1));
    const int levels = 1 + (int)((h >> 20) % 40);
    const bool nan = ((h >> 32) % 50) == 0;
    for (int e = lane; e < kPcCap; e += 32) {
        const unsigned long long r = mix64(h + (unsigned long long)e);
        double x = (kind == 0) ? (double)(r >> 11) * 0x1.0p-53 * 4.0 - 1.0
                               : (double)(r % (unsigned long long)levels) * 0.5 - 2.0;
        if (nan && e == (int)((h >> 40) % (unsigned long long)(size > 0 ? size : 1))) x = NAN;
        sv[w][0][e] = sv[w][1][e] = sv[w][2][e] = x;
        sp[w][0][e] = sp[w][1][e] = sp[w][2][e] = (uint16_t)e;
    }
    __syncwarp();
    const double avg = (kind == 1) ? -3.0 - (double)((h >> 48) % 7) : (double)((int)((h >> 48) % 9) - 4) * 0.25;
    const int ef_min = 1 + (int)((h >> 56) % 6);
    int p0 = 0;
    if (lane == 0) p0 = qpart_ef_vals(sp[w][0], sv[w][0], size, avg, ef_min);
    __syncwarp();
    p0 = __shfl_sync(0xffffffffu, p0, 0);
    const int p1 = warp_qpart_ef_vals<kPcCap / 32>(sp[w][1], sv[w][1], spos[w], size, avg, ef_min, lane);
    __syncwarp();
    // the thread-serial pairing form (lists of at most 64 entries without NaN)
    int p2 = p0;
    bool pair = size <= 64;
    if (lane == 0 && pair) {
        double* val = sv[w][2];
        uint16_t* pl = sp[w][2];
        p2 = qpart_ef_bits(
            size, avg, ef_min, [&](int k) { return val[k]; },
            [&](int i, int j) {
                const uint16_t t = pl[i]; pl[i] = pl[j]; pl[j] = t;
                const double u = val[i]; val[i] = val[j]; val[j] = u;
            });
    }
    __syncwarp();
    p2 = __shfl_sync(0xffffffffu, p2, 0);
    pair = pair && p2 >= 0;  // -1: a NaN, which the pairing form leaves to the serial loop
    bool diff = p0 != p1 || (pair && p2 != p0);
    for (int e = lane; e < size; e += 32) diff |= sp[w][0][e] != sp[w][1][e] || (pair && sp[w][0][e] != sp[w][2][e]);
    if (__any_sync(0xffffffffu, diff) && lane == 0) atomicAdd(bad, 1ull);
}

cudaError_t launch_partition_check(int n_cases, unsigned long long seed, unsigned long long* bad, cudaStream_t s) {
    if (n_cases <= 0) return cudaSuccess;
    const int blocks = (n_cases + kPcWarps - 1) / kPcWarps;
    k_partition_check<<<blocks, 32 * kPcWarps, 0, s>>>(n_cases, seed, bad);
    return cudaGetLastError();
}

}  // namespace f2m
