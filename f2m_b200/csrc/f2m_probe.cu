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

}  // namespace f2m
