// Device helpers shared by the per-team solver (f2m_kernels.cu) and the
// grid-wide solver (f2m_grid.cu).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "f2m_internal.h"

namespace f2m {

/* ------------------------------------------------------------------ */
/* block-level helpers                                                  */
/* ------------------------------------------------------------------ */
template <int T>
__device__ __forceinline__ double block_max(double x, double* sred) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) sred[w] = x;
    __syncthreads();
    if (w == 0) {
        x = (lane < T / 32) ? sred[lane] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sred[0] = x;
    }
    __syncthreads();
    double r = sred[0];
    __syncthreads();
    return r;
}
template <int T>
__device__ __forceinline__ double block_min(double x, double* sred) {
    return -block_max<T>(-x, sred);
}
template <int T>
__device__ __forceinline__ double block_sum(double x, double* sred) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sred[w] = x;
    __syncthreads();
    if (w == 0) {
        x = (lane < T / 32) ? sred[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sred[0] = x;
    }
    __syncthreads();
    double r = sred[0];
    __syncthreads();
    return r;
}
template <int T>
__device__ __forceinline__ long long block_sum_ll(long long x, long long* sred) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sred[w] = x;
    __syncthreads();
    if (w == 0) {
        x = (lane < T / 32) ? sred[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sred[0] = x;
    }
    __syncthreads();
    long long r = sred[0];
    __syncthreads();
    return r;
}
template <int T>
__device__ __forceinline__ long long block_max_ll(long long x, long long* sred) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, (long long)__shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) sred[w] = x;
    __syncthreads();
    if (w == 0) {
        x = (lane < T / 32) ? sred[lane] : LLONG_MIN;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = max(x, (long long)__shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sred[0] = x;
    }
    __syncthreads();
    long long r = sred[0];
    __syncthreads();
    return r;
}
// Exclusive scan of one int per thread in thread order; *total = block sum.
// swarp needs T/32 + 1 ints.
template <int T>
__device__ __forceinline__ int block_excl_scan(int x, int* swarp, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) swarp[w] = inc;
    __syncthreads();
    if (w == 0) {
        int s = (lane < T / 32) ? swarp[lane] : 0;
        int incs = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, incs, o);
            if (lane >= o) incs += y;
        }
        if (lane < T / 32) swarp[lane] = incs - s;
        if (lane == T / 32 - 1) swarp[T / 32] = incs;
    }
    __syncthreads();
    int r = swarp[w] + inc - x;
    *total = swarp[T / 32];
    __syncthreads();
    return r;
}

struct Inst {
    int V;
    int64_t base;          // first node index
    const int64_t* row;    // row[v], v in [0, V]
    const Slot* slot;
    uint16_t* perm;        // per-node list order (the reference's permuted pointer list)
    Slot* pslot;           // the slots in that order, so a scan reads one record per position
    double* gD;            // global EF arena of this instance (D)
    uint16_t* gN;          // (neighbour)
};

// The views of instance b inside the batch buffers.
__device__ __forceinline__ Inst make_inst(const Batch& B, int b) {
    Inst I;
    I.V = B.Vn[b];
    I.base = B.offs[b];
    I.row = B.row + I.base;
    I.slot = B.slot;
    I.perm = B.perm;
    I.pslot = B.pslot;
    I.gD = B.efD + I.row[0];
    I.gN = B.efN + I.row[0];
    return I;
}

// Reduced cost of a slot of node v: D + 0.5*F[v1] + 0.5*F[v2] with v1<v2
// (cuda_recompute_Edges, graph_cuda_grad.hpp:257-268), from H = F/2.
template <class HP>
__device__ __forceinline__ double red_d(const Slot& s, int v, HP H, double hv) {
    const double hn = H[s.nbr];
    return (v < s.nbr) ? (s.D + hv) + hn : (s.D + hn) + hv;
}

// Sorted insertion of x into (v0 <= v1 <= v2) keeping the three smallest:
// the reference's compare chain (strict <, so ties and NaN leave the triple
// as it is) written as three independent FP64 compares and integer selects.
// The step is bound by latency, not by the FP64 pipe (measured: about a
// tenth of its rate), and the insertion is the loop-carried chain of a
// lane: three compares issued together keep it at one compare and two
// selects deep (a two-compare form, x < v1 first, then x against v0 or v2,
// is one compare deeper and measured slower).
__device__ __forceinline__ void top3_insert(double x, double& v0, double& v1, double& v2) {
    const bool c0 = x < v0, c1 = x < v1, c2 = x < v2;
    v2 = c1 ? v1 : (c2 ? x : v2);
    v1 = c0 ? v0 : (c1 ? x : v1);
    v0 = c0 ? x : v0;
}
// Reduced cost of position k of node v's list (the slot perm[r0 + k]).
template <class HP>
__device__ __forceinline__ double pdv(const Inst& I, int64_t r0, int k, int v, HP H, double hv) {
    return red_d(I.pslot[r0 + k], v, H, hv);
}
// Sets pslot from slot and perm for nodes [v0, V) in steps of `step` (each
// solver keeps the two in step from there: every swap moves both).
// (restrict pointers: an unrolled group's loads may be issued before its stores)
__device__ __forceinline__ void gather_slots(const Slot* __restrict__ slot, const uint16_t* __restrict__ perm,
                                             Slot* __restrict__ out, int64_t n) {
#pragma unroll 4
    for (int64_t k = 0; k < n; ++k) out[k] = slot[perm[k]];
}
__device__ __forceinline__ void init_pslot(const Inst& I, int v0, int step) {
    for (int v = v0; v < I.V; v += step) {
        const int64_t r0 = I.row[v];
        gather_slots(I.slot + r0, I.perm + r0, I.pslot + r0, I.row[v + 1] - r0);
    }
}

// The threshold loop of qpart_ptr_EF, `while (avg < g && bump < limit) {
// avg += 1; ++bump; }`, with the stretches where every `+= 1` is exact taken
// in one addition: above 1 inside a binade (ulp <= 1 and no carry into the
// next binade), and at or below -1 up to 0 (the sums are multiples of the
// ulp below the starting magnitude).  Binade crossings and the steps across
// zero, where `+= 1` may round, run one at a time, so avg and bump end as in
// the plain loop.  The plain loop costs g - avg dependent FP64 additions,
// thousands where reduced costs are large in units of the shortest edge.
__device__ __forceinline__ void bump_until(double& avg, int& bump, double g, int limit) {
    while (avg < g && bump < limit) {
        long long n = 0;  // steps that stay exact
        if (avg >= 1.0 && avg < 4503599627370496.0) {  // [1, 2^52)
            int e;
            frexp(avg, &e);
            n = (long long)ceil(ldexp(1.0, e) - avg) - 1;  // avg + n < 2^e (the difference is exact)
        } else if (avg <= -1.0 && avg > -4503599627370496.0) {
            n = (long long)floor(-avg);  // avg + n <= 0
        }
        if (n >= 1) {
            long long c = (long long)fmin(ceil(g - avg), (double)n);
            if (c < 1) c = 1;
            while (c > 1 && avg + (double)(c - 1) >= g) --c;  // stop where the plain loop stops
            if (c > (long long)(limit - bump)) c = limit - bump;
            avg += (double)c;
            bump += (int)c;
        } else {
            avg += 1;
            ++bump;
        }
    }
}

// qpart_ptr_B / qpart_ptr_EF (graph_cuda_partition.hpp:3-54) with the
// scans' loads run ahead: every reduced cost is a chain of dependent loads
// (the position's slot record from L2, then the neighbour's potential), so
// the scans evaluate kPf positions at once and then test them in order, and
// the loads of a chunk overlap.  Positions are read from pslot, the slots
// kept in list order, and every swap moves both the list (perm, which the
// host stage and the repair loop read) and pslot.  The tests (the bound first, as the reference's loop
// reads one element past either end), the swaps and the threshold sequence
// are the reference's, so the final order and count are too.  On finite
// values a pass performs at most size/2 swaps; the pass cap only matters for
// NaN values, where the reference loops forever.
//
// qpart_ef_la raises the threshold by 1 until at least ef_min entries
// qualify.  A pass whose threshold t stays below the smallest value g of the
// upper part left by the previous pass finds the list already partitioned
// for t: the i-scan stops at the first upper entry, the j-scan at the last
// lower one, no swap happens and the count repeats.  Such passes are counted
// but not run (bump_until), so the threshold sequence (repeated FP64
// `avg += 1`), the final order and the count are those of the plain loop.
// With a NaN in the list every pass runs.
constexpr int kPf = 8;
template <class HP>
__device__ __forceinline__ int qpart_b_la(const Inst& I, int64_t r0, int v, HP H, int size, double avg) {
    uint16_t* list = I.perm + r0;
    const double hv = H[v];
    int low = 0, high = size - 1, i = low, j = high;
    for (int pass = 0; i < j && pass <= size; ++pass) {
        for (bool go = true; go;) {  // while (i <= high && pdv(i) <= avg) i++
            double d[kPf];
#pragma unroll
            for (int c = 0; c < kPf; ++c) d[c] = (i + c <= high) ? pdv(I, r0, i + c, v, H, hv) : 0.0;
#pragma unroll
            for (int c = 0; c < kPf; ++c)
                if (go) {
                    if (i <= high && d[c] <= avg) ++i;
                    else go = false;
                }
        }
        for (bool go = true; go;) {  // while (j >= low && pdv(j) > avg) j--
            double d[kPf];
#pragma unroll
            for (int c = 0; c < kPf; ++c) d[c] = (j - c >= low) ? pdv(I, r0, j - c, v, H, hv) : 0.0;
#pragma unroll
            for (int c = 0; c < kPf; ++c)
                if (go) {
                    if (j >= low && d[c] > avg) --j;
                    else go = false;
                }
        }
        if (i < j) {
            const uint16_t t = list[i]; list[i] = list[j]; list[j] = t;
            Slot* ps = I.pslot + r0;
            const Slot u = ps[i]; ps[i] = ps[j]; ps[j] = u;
        }
    }
    return j + 1;
}
template <class HP>
__device__ __forceinline__ int qpart_ef_la(const Inst& I, int64_t r0, int v, HP H, int size, double avg,
                                           int ef_min) {
    if (size < ef_min) return size;
    constexpr int kLimit = 1 << 20;
    const double hv = H[v];
    for (int bump = 0; bump < kLimit;) {
        const int p = qpart_b_la(I, r0, v, H, size, avg);
        if (p >= ef_min) return p;
        double g = INFINITY;
        bool nan = false;
        for (int k0 = 0; k0 < size; k0 += kPf) {
            double d[kPf];
#pragma unroll
            for (int c = 0; c < kPf; ++c) d[c] = (k0 + c < size) ? pdv(I, r0, k0 + c, v, H, hv) : 0.0;
#pragma unroll
            for (int c = 0; c < kPf; ++c)
                if (k0 + c < size) {
                    nan |= (d[c] != d[c]);
                    if (k0 + c >= p) g = fmin(g, d[c]);
                }
        }
        avg += 1;
        ++bump;
        if (nan) continue;
        bump_until(avg, bump, g, kLimit);
    }
    return size;
}

// The same partition by one thread in the pairing form, for lists of at
// most 64 entries: one sweep evaluates every position (val(k), kPf at a time,
// so their loads are in flight together) and marks those > avg; then the
// Hoare loop's swaps are applied directly -- the t-th marked position below
// the final count Lc (ascending) with the t-th unmarked one at or above Lc
// (descending), through swp(i, j) -- and Lc is returned, as qpart_b_la
// returns it.  *g receives the smallest value > avg (the upper part's
// minimum the threshold loop needs).  A NaN makes it return -1 before any
// swap (the caller then runs the plain loop, whose every pass runs).
template <class Val, class Swap>
__device__ __forceinline__ int qpart_b_bits(int size, double avg, Val val, Swap swp, double* g) {
    uint64_t gt = 0;
    bool nan = false;
    double gm = INFINITY;
    for (int k0 = 0; k0 < size; k0 += kPf) {
        double d[kPf];
#pragma unroll
        for (int c = 0; c < kPf; ++c) d[c] = (k0 + c < size) ? val(k0 + c) : 0.0;
#pragma unroll
        for (int c = 0; c < kPf; ++c)
            if (k0 + c < size) {
                nan |= (d[c] != d[c]);
                if (d[c] > avg) {
                    gt |= 1ull << (k0 + c);
                    gm = fmin(gm, d[c]);
                }
            }
    }
    if (nan) return -1;
    *g = gm;
    if (size <= 1) return size;  // the loop does not run
    const int Lc = size - __popcll(gt);
    const uint64_t low = Lc >= 64 ? ~0ull : ((1ull << Lc) - 1ull);
    const uint64_t all = size >= 64 ? ~0ull : ((1ull << size) - 1ull);
    uint64_t gL = gt & low, lU = ~gt & all & ~low;
    while (gL) {
        const int i = __ffsll((long long)gL) - 1;
        const int j = 63 - __clzll((long long)lU);
        gL &= gL - 1ull;
        lU &= ~(1ull << j);
        swp(i, j);
    }
    return Lc;
}
// qpart_ef_vals / qpart_ef_la's threshold loop over qpart_b_bits; returns -1
// (list untouched) when the list holds a NaN.
template <class Val, class Swap>
__device__ __forceinline__ int qpart_ef_bits(int size, double avg, int ef_min, Val val, Swap swp) {
    if (size < ef_min) return size;
    constexpr int kLimit = 1 << 20;
    for (int bump = 0; bump < kLimit;) {
        double g = INFINITY;
        const int p = qpart_b_bits(size, avg, val, swp, &g);
        if (p < 0) return -1;
        if (p >= ef_min) return p;
        avg += 1;
        ++bump;
        bump_until(avg, bump, g, kLimit);
    }
    return size;
}
// qpart_b_la (one pass) for a node's list in global memory, by the pairing
// form when the list has at most 64 entries and no NaN
template <class HP>
__device__ __forceinline__ int qpart_b_pair(const Inst& I, int64_t r0, int v, HP H, int size, double avg) {
    if (size <= 64) {
        const double hv = H[v];
        uint16_t* list = I.perm + r0;
        Slot* ps = I.pslot + r0;
        double g;
        const int p = qpart_b_bits(
            size, avg, [&](int k) { return red_d(ps[k], v, H, hv); },
            [&](int i, int j) {
                const uint16_t t = list[i]; list[i] = list[j]; list[j] = t;
                const Slot u = ps[i]; ps[i] = ps[j]; ps[j] = u;
            },
            &g);
        if (p >= 0) return p;
    }
    return qpart_b_la(I, r0, v, H, size, avg);
}
// qpart_ef_la for a node's list in global memory (perm and pslot), by the
// pairing form when the list has at most 64 entries and no NaN
template <class HP>
__device__ __forceinline__ int qpart_ef_pair(const Inst& I, int64_t r0, int v, HP H, int size, double avg,
                                             int ef_min) {
    if (size <= 64) {
        const double hv = H[v];
        uint16_t* list = I.perm + r0;
        Slot* ps = I.pslot + r0;
        const int p = qpart_ef_bits(
            size, avg, ef_min, [&](int k) { return red_d(ps[k], v, H, hv); },
            [&](int i, int j) {
                const uint16_t t = list[i]; list[i] = list[j]; list[j] = t;
                const Slot u = ps[i]; ps[i] = ps[j]; ps[j] = u;
            });
        if (p >= 0) return p;
    }
    return qpart_ef_la(I, r0, v, H, size, avg, ef_min);
}

// qpart_ptr_EF on a node's list copied to shared memory: `pl` holds the list
// order and `val` the reduced cost of each position.  The loop is qpart_ef's
// (the Hoare scans, the swaps, which move both arrays, and the threshold
// sequence), so the final order and count are the same; only the values are
// read from shared memory instead of three dependent global loads each.
__device__ inline int qpart_b_vals(uint16_t* pl, double* val, int size, double avg) {
    int low = 0, high = size - 1, i = low, j = high;
    for (int pass = 0; i < j && pass <= size; ++pass) {
        while (i <= high && val[i] <= avg) i++;
        while (j >= low && val[j] > avg) j--;
        if (i < j) {
            const uint16_t t = pl[i]; pl[i] = pl[j]; pl[j] = t;
            const double u = val[i]; val[i] = val[j]; val[j] = u;
        }
    }
    return j + 1;
}
__device__ inline int qpart_ef_vals(uint16_t* pl, double* val, int size, double avg, int ef_min) {
    if (size < ef_min) return size;
    constexpr int kLimit = 1 << 20;
    for (int bump = 0; bump < kLimit;) {
        const int p = qpart_b_vals(pl, val, size, avg);
        if (p >= ef_min) return p;
        double g = INFINITY;
        bool nan = false;
        for (int k = 0; k < size; ++k) {
            nan |= (val[k] != val[k]);
            if (k >= p) g = fmin(g, val[k]);
        }
        avg += 1;
        ++bump;
        if (nan) continue;
        bump_until(avg, bump, g, kLimit);
    }
    return size;
}

// The same partition run by a whole warp.  On finite values the Hoare loop
// of qpart_b_vals is a fixed pairing: with Lc the number of entries <= avg,
// its t-th swap exchanges the t-th entry > avg of [0, Lc) (ascending) with
// the t-th entry <= avg of [Lc, size) (descending), for every t below the
// number m of entries > avg in [0, Lc), and it returns Lc (a list of one
// entry is returned as it is: the loop does not run).  Each lane ranks its
// entries with ballots, the two sides list their positions by rank in
// `pos` (2 x 16 NC bytes: m <= size / 2), and the entries that swap take
// their partner's, so the final order and the count are the serial loop's.
// Lists of at most 32 * NC entries in shared memory; every lane of the warp
// calls it with the same arguments.
template <int NC>
__device__ __forceinline__ int warp_qpart_b_vals(uint16_t* pl, double* val, uint8_t* pos, int size, double avg,
                                                 int lane) {
    if (size <= 1) return size;
    unsigned gt[NC];
    int G = 0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const int e = c * 32 + lane;
        gt[c] = __ballot_sync(0xffffffffu, e < size && val[e] > avg);
        G += __popc(gt[c]);
    }
    const int Lc = size - G;
    // > avg below Lc (ranked ascending into pos[0..m)), <= avg from Lc on
    // (ranked ascending into pos[16 NC ..)); the t-th of the first swaps with
    // the (m-1-t)-th of the second
    uint8_t* gp = pos;
    uint8_t* up = pos + 16 * NC;
    const unsigned below = (1u << lane) - 1u;
    int rg = 0, ru = 0;
    int rank[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const int b0 = c * 32;
        const unsigned lo = Lc >= b0 + 32 ? 0xffffffffu : (Lc <= b0 ? 0u : (1u << (Lc - b0)) - 1u);
        const unsigned in = size >= b0 + 32 ? 0xffffffffu : (size <= b0 ? 0u : (1u << (size - b0)) - 1u);
        const unsigned gL = gt[c] & lo, lU = ~gt[c] & in & ~lo;
        rank[c] = -1;
        if ((gL >> lane) & 1u) { rank[c] = rg + __popc(gL & below); gp[rank[c]] = (uint8_t)(b0 + lane); }
        if ((lU >> lane) & 1u) { rank[c] = ru + __popc(lU & below); up[rank[c]] = (uint8_t)(b0 + lane); }
        rg += __popc(gL);
        ru += __popc(lU);
    }
    const int m = rg;  // == ru
    if (m == 0) return Lc;
    __syncwarp();
    int src[NC];
    double x[NC];
    uint16_t q[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        src[c] = -1;
        if (rank[c] >= 0) {
            const bool low = c * 32 + lane < Lc;
            src[c] = low ? up[m - 1 - rank[c]] : gp[m - 1 - rank[c]];
            x[c] = val[src[c]];
            q[c] = pl[src[c]];
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < NC; ++c)
        if (src[c] >= 0) { val[c * 32 + lane] = x[c]; pl[c * 32 + lane] = q[c]; }
    __syncwarp();
    return Lc;
}
// qpart_ef_vals by a warp: the threshold loop (avg += 1 until ef_min entries
// qualify, the passes that cannot move an entry counted by bump_until) with
// warp_qpart_b_vals as the pass.  A list holding a NaN keeps the serial loop
// (lane 0), whose every pass runs; the values never change, only their order.
template <int NC>
__device__ __noinline__ int warp_qpart_ef_vals(uint16_t* pl, double* val, uint8_t* pos, int size, double avg,
                                              int ef_min, int lane) {
    if (size < ef_min) return size;
    bool nan = false;
    for (int e = lane; e < size; e += 32) nan |= (val[e] != val[e]);
    if (__any_sync(0xffffffffu, nan)) {
        int p = 0;
        if (lane == 0) p = qpart_ef_vals(pl, val, size, avg, ef_min);
        __syncwarp();
        return __shfl_sync(0xffffffffu, p, 0);
    }
    constexpr int kLimit = 1 << 20;
    for (int bump = 0; bump < kLimit;) {
        const int p = warp_qpart_b_vals<NC>(pl, val, pos, size, avg, lane);
        if (p >= ef_min) return p;
        double g = INFINITY;
        for (int e = p + lane; e < size; e += 32) g = fmin(g, val[e]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g = fmin(g, __shfl_xor_sync(0xffffffffu, g, o));
        avg += 1;
        ++bump;
        bump_until(avg, bump, g, kLimit);
    }
    return size;
}

/* ------------------------------------------------------------------ */
/* Ax=b of an irregular comb                                            */
/* ------------------------------------------------------------------ */
// The linear system of one comb (comb::solve_AxB, comb_thread.cpp:272-304):
// a row per comb node whose entries (coefficient 1) are the node's B edges
// (|d| < porog over its whole list, node.cpp:49-57) and whose right-hand side
// is 2 minus its A edges (d <= -porog); the variables are the B edges,
// numbered on first sight.  CSR: row k's variables are col[rs[k] .. rs[k+1]).
struct AxbRows {
    int m, z, q;  // rows, entries, variables
    const int* rs;
    const int* col;
    const int* rhs;
};

// Doubles of scratch an Ax=b system of m rows and z entries needs: ints rs
// (m+1), col (z), rhs (m), the variables' edge slots (<= z); doubles Aj, d,
// b_grad (m each), x, x_grad (<= z each).
__device__ __forceinline__ long long axb_scratch_doubles(long long m, long long z) {
    return 3 * m + 2 * z + (2 * m + 2 * z + 1 + 1) / 2 + 2;
}

// Ax_b::solve (Ax_b.cpp:87-158) by one thread: steepest descent on the
// row-scaled residual with an exact line search, until the largest scaled
// residual is below 1e-8 (at most 999 steps).  FP64 in the reference's
// operation order within each row and over the rows, without multiply-add
// contraction (the reference's host code has none).  Returns the step count
// at convergence, 0 when it did not converge (Ax_b::go_max).
static __device__ __noinline__ int axb_solve(const AxbRows& S, double* Aj, double* d, double* bg, double* x,
                                      double* xg) {
    for (int j = 0; j < S.m; ++j) Aj[j] = sqrt((double)(S.rs[j + 1] - S.rs[j]));
    for (int i = 0; i < S.q; ++i) x[i] = 0.0;
    for (int go = 1; go < 1000; ++go) {
        for (int i = 0; i < S.q; ++i) xg[i] = 0.0;
        double dmax = 0.0;
        for (int j = 0; j < S.m; ++j) {
            double ax = 0.0;
            for (int k = S.rs[j]; k < S.rs[j + 1]; ++k) ax = __dadd_rn(ax, x[S.col[k]]);
            const double dj = __dsub_rn(ax, (double)S.rhs[j]) / Aj[j];
            d[j] = dj;
            if (fabs(dj) > dmax) dmax = fabs(dj);
            const double gj = dj / Aj[j];
            for (int k = S.rs[j]; k < S.rs[j + 1]; ++k) xg[S.col[k]] = __dadd_rn(xg[S.col[k]], gj);
        }
        if (dmax < 1e-8) return go;
        double gg = 0.0, gd = 0.0;
        for (int j = 0; j < S.m; ++j) {
            double bj = 0.0;
            for (int k = S.rs[j]; k < S.rs[j + 1]; ++k) bj = __dadd_rn(bj, xg[S.col[k]]);
            bg[j] = bj;
        }
        for (int j = 0; j < S.m; ++j) gg = __dadd_rn(gg, __dmul_rn(bg[j], bg[j]));
        for (int j = 0; j < S.m; ++j) gd = __dadd_rn(gd, __dmul_rn(d[j], bg[j]));
        const double alfa = -gd / gg;
        for (int i = 0; i < S.q; ++i) x[i] = __dadd_rn(x[i], __dmul_rn(xg[i], alfa));
    }
    return 0;
}

// Potentials H = F/2 read from the saved F (halving is exact).
struct HalfF {
    const double* F;
    __device__ __forceinline__ double operator[](int64_t i) const { return 0.5 * F[i]; }
};

// Sums of the primal over nodes (graph_cuda.cu:135-147, graph_tour.hpp:142-184).
struct PrimalSums {
    double lp = 0.0, dual_neg = 0.0, fsum = 0.0;
    long long maxr = -1, viol = 0;
};
// The primal of node v's slots: x = 1 on A edges, 1/2 on B edges -- or, with
// axb, the Ax=b value when the edge's larger-root comb is irregular (every
// edge of a comb enters graph::X, whatever its value) -- its code per slot
// for the host, OVAL = sum x*Do and MAX edge rank over the edges whose other
// end is the higher id, the degree check (graph_tour.hpp:142-163) and the
// FP64 dual bound's terms.  lab/irr: comb root per node, irregular flag per
// root (read only with axb).
template <class HP, class LP>
__device__ __forceinline__ void primal_node(const Batch& B, const Inst& I, HP H, LP lab, LP irr, bool axb,
                                            int v, double porog, PrimalSums& ps) {
    const int64_t r0 = I.row[v], r1 = I.row[v + 1];
    const double hv = H[v];
    ps.fsum += 2.0 * hv;
    float degsum = 0.0f;
    bool any = false;
    for (int64_t a = r0; a < r1; ++a) {
        const Slot s = I.slot[a];
        const double d = red_d(s, v, H, hv);
        double x = (d < porog) ? ((d > -porog) ? 0.5 : 1.0) : 0.0;
        uint8_t code = (uint8_t)(x == 1.0 ? 2 : (x == 0.5 ? 1 : 0));
        if (axb && code == 1) {
            const int l1 = lab[v], l2 = lab[s.nbr];
            const int c = (l2 == INT_MAX) ? l1 : (l1 == INT_MAX ? l2 : ::max(l1, l2));
            if (c != INT_MAX && irr[c]) { x = (double)B.xval[a]; code = 3; }
        }
        B.xcode[a] = code;
        const bool in_x = (x != 0.0) || code == 3;
        degsum += (float)x;
        any |= in_x;
        if (s.nbr > v) {
            ps.lp += x * B.s_cost[a];
            ps.dual_neg += fmin(0.0, d);
            if (in_x) ps.maxr = ::max(ps.maxr, (long long)::min((int)(a - r0), B.mirror[a]));
        }
    }
    if (any && !(degsum > 2.0f - 1e-2f && degsum < 2.0f + 1e-2f)) ps.viol++;
}

// Doubles of scratch one comb needs: its member list (m ints) and its system.
__device__ __forceinline__ long long axb_comb_doubles(long long m, long long z) {
    return (m + 1) / 2 + 1 + axb_scratch_doubles(m, z);
}

// B edges (|d| < porog) of node u over its whole list.
template <class HP>
__device__ __forceinline__ int count_b(const Slot* slot, const int64_t* row, HP H, int u, double porog) {
    const double hu = H[u];
    int z = 0;
    for (int64_t a = row[u]; a < row[u + 1]; ++a) {
        const double d = red_d(slot[a], u, H, hu);
        if (d < porog && d > -porog) z++;
    }
    return z;
}

// One irregular comb's Ax=b, built and solved by one thread (out of line to
// keep the solvers' registers free).  mem[0..m) are the comb's nodes in
// ascending id (the rows); z their B edges (count_b summed); the system goes
// to w (axb_scratch_doubles(m, z) doubles).  HP reads the potentials H = F/2,
// LP the comb labels (the root of each node's comb, INT_MAX outside combs).
// Writes x (FP32) of the comb's B edges whose larger-root comb is this one
// (r) to both slots of the edge.  Returns 1 when the system did not converge
// within 900 steps or a slot has no twin.
template <class HP, class LP>
__device__ __noinline__ int axb_comb(const Slot* slot, const int64_t* row, int64_t row0, const int32_t* mirror,
                                     HP H, LP lab, const int* mem, int m, int z, int r, double porog, double* w,
                                     float* xval) {
    int* rs = reinterpret_cast<int*>(w);
    int* col = rs + m + 1;
    int* rhs = col + z;
    int* vs = rhs + m;  // canonical slot (offset in the instance) of each variable
    double* Aj = w + (2 * m + 2 * z + 2) / 2;
    double* dd = Aj + m;
    double* bg = dd + m;
    double* x = bg + m;
    double* xg = x + z;
    int k = 0, q = 0;
    for (int j = 0; j < m; ++j) {
        const int u = mem[j];
        const double hu = H[u];
        int na = 0;
        rs[j] = k;
        for (int64_t a = row[u]; a < row[u + 1]; ++a) {
            const Slot s = slot[a];
            const double d = red_d(s, u, H, hu);
            if (!(d < porog)) continue;
            if (!(d > -porog)) { na++; continue; }
            const int mi = mirror[a];
            if (mi < 0 || k >= z) return 1;
            const int cs = (int)((s.nbr > u ? a : row[s.nbr] + mi) - row0);
            int t = 0;
            while (t < q && vs[t] != cs) ++t;
            if (t == q) vs[q++] = cs;
            col[k++] = t;
        }
        rhs[j] = 2 - na;
    }
    rs[m] = k;
    const AxbRows S{m, k, q, rs, col, rhs};
    const int go = axb_solve(S, Aj, dd, bg, x, xg);
    if (go == 0 || go > 900) return 1;
    k = 0;
    for (int j = 0; j < m; ++j) {
        const int u = mem[j];
        const double hu = H[u];
        for (int64_t a = row[u]; a < row[u + 1]; ++a) {
            const Slot s = slot[a];
            const double d = red_d(s, u, H, hu);
            if (!(d < porog) || !(d > -porog)) continue;
            const int t = col[k++];
            const int ln = lab[s.nbr];
            if (ln != INT_MAX && ln > r) continue;  // the neighbour's comb decides
            const float xv = (float)x[t];
            xval[a] = xv;
            xval[row[s.nbr] + mirror[a]] = xv;
        }
    }
    return 0;
}

}  // namespace f2m
