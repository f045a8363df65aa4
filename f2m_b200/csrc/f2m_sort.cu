// Stable LSD radix sort of 64-bit keys (optionally with 32-bit values), the
// repository's own: the single-instance edge order (ascending cost, then
// emitter, then partner) and the grid solver's Morton ownership order run on
// it.  8-bit digits; one pass is a per-tile digit histogram, an exclusive
// scan of the (digit, tile) counts in digit-major order, and a stable
// scatter.  Inside a tile each warp owns a contiguous run of items and walks
// it in rounds of 32 consecutive items: lanes holding the same digit find
// each other with __match_any_sync, and the rank of an item is the number of
// equal digits before it in the warp's run plus the counts of the warps
// before it, so equal keys keep their input order.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <utility>

#include "f2m_internal.h"

namespace f2m {

constexpr int kRsThreads = 256;
constexpr int kRsPer = 8;                       // items per thread
constexpr int kRsTile = kRsThreads * kRsPer;    // 2,048 items per tile
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsRun = kRsTile / kRsWarps;      // 256 consecutive items per warp

static int64_t rs_tiles(int64_t n) { return (n + kRsTile - 1) / kRsTile; }

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned long long* key, int64_t n, int shift,
                                                       int64_t tiles, int64_t* count) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t0 = (int64_t)blockIdx.x * kRsTile;
    for (int i = threadIdx.x; i < kRsTile; i += kRsThreads) {
        const int64_t g = t0 + i;
        if (g < n) atomicAdd(&h[(int)((key[g] >> shift) & 255)], 1);
    }
    __syncthreads();
    count[(int64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];  // digit-major
}

template <bool VALS>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned long long* kin, const uint32_t* vin,
                                                          unsigned long long* kout, uint32_t* vout, int64_t n,
                                                          int shift, int64_t tiles, const int64_t* offset) {
    __shared__ int wcnt[kRsWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = lane; d < 256; d += 32) wcnt[w][d] = 0;
    __syncwarp();
    const int64_t base = (int64_t)blockIdx.x * kRsTile + (int64_t)w * kRsRun;
    int dig[kRsPer], rank[kRsPer];
#pragma unroll
    for (int r = 0; r < kRsPer; ++r) {
        const int64_t g = base + r * 32 + lane;
        const bool ok = g < n;
        const int d = ok ? (int)((kin[g] >> shift) & 255) : 256 + lane;  // unmatched padding
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int before = __popc(peers & ((1u << lane) - 1u));
        const int c = ok ? wcnt[w][d] : 0;
        __syncwarp();
        if (ok && before == 0) wcnt[w][d] = c + __popc(peers);
        __syncwarp();
        dig[r] = d;
        rank[r] = c + before;
    }
    __syncthreads();
    // counts of the warps before this one, per digit
    {
        const int d = threadIdx.x;  // kRsThreads == 256 digits
        int run = 0;
#pragma unroll
        for (int k = 0; k < kRsWarps; ++k) {
            const int c = wcnt[k][d];
            wcnt[k][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsPer; ++r) {
        const int64_t g = base + r * 32 + lane;
        if (g >= n) continue;
        const int d = dig[r];
        const int64_t pos = offset[(int64_t)d * tiles + blockIdx.x] + wcnt[w][d] + rank[r];
        kout[pos] = kin[g];
        if (VALS) vout[pos] = vin[g];
    }
}

size_t radix_sort_temp_bytes(int64_t n) {
    const int64_t cells = 256 * std::max<int64_t>(rs_tiles(n), 1);
    return (size_t)(2 * cells + scan_scratch_elems(cells) + 2) * sizeof(int64_t);
}

// Sorts n keys (and values, when vals is not null) by bits [begin_bit,
// end_bit), stably.  keys/vals hold the input; kbuf/vbuf are buffers of the
// same size.  The sorted data ends in one of the two, returned in *kres /
// *vres.
cudaError_t radix_sort(unsigned long long* keys, unsigned long long* kbuf, uint32_t* vals, uint32_t* vbuf,
                       int64_t n, int begin_bit, int end_bit, void* temp, size_t temp_bytes, cudaStream_t s,
                       int64_t* launches, unsigned long long** kres, uint32_t** vres) {
    *kres = keys;
    if (vres) *vres = vals;
    if (n <= 1) return cudaSuccess;
    if (temp_bytes < radix_sort_temp_bytes(n)) return cudaErrorInvalidValue;
    const int64_t tiles = rs_tiles(n);
    const int64_t cells = 256 * tiles;
    int64_t* count = static_cast<int64_t*>(temp);
    int64_t* offset = count + cells + 1;
    int64_t* scratch = offset + cells + 1;
    unsigned long long *ki = keys, *ko = kbuf;
    uint32_t *vi = vals, *vo = vbuf;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        k_rs_hist<<<(unsigned)tiles, kRsThreads, 0, s>>>(ki, n, shift, tiles, count);
        ++*launches;
        cudaError_t e = launch_scan(count, offset, cells, scratch, s, launches);
        if (e != cudaSuccess) return e;
        if (vals) k_rs_scatter<true><<<(unsigned)tiles, kRsThreads, 0, s>>>(ki, vi, ko, vo, n, shift, tiles, offset);
        else k_rs_scatter<false><<<(unsigned)tiles, kRsThreads, 0, s>>>(ki, nullptr, ko, nullptr, n, shift, tiles, offset);
        ++*launches;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    *kres = ki;
    if (vres) *vres = vi;
    return cudaSuccess;
}

}  // namespace f2m
