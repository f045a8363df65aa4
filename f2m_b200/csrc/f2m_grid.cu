// Grid-wide solver: one large instance over every SM of the GPU.
//
// The same schedule as the per-team solver (graph_cuda.cu:163-430 and the
// comb stage, graph_cuda_comb.hpp:415-475), for instances whose potentials no
// longer fit one SM's shared memory (10^5+ nodes).  Each CTA owns a spatially
// compact run of nodes (Morton order of the points); H = F/2 (double-buffered)
// and the comb labels live in global memory and are read through L2
// (ld.global.cg) because other SMs write them; a CTA's EF lists are cached in
// its shared memory.  The launch is cooperative, so all CTAs are resident,
// and a bounded software grid barrier orders the steps; a barrier that waits
// too long sets an error flag and every CTA returns.
//
// Halo blocks.  Between two rebuilds of the active sets the Jacobi steps read
// only the EF lists, so a CTA that holds the potentials of every node within
// k EF hops of its own nodes (its halo, in shared memory) can run k steps
// alone: step t recomputes the nodes within k-t hops, and after k steps its
// own nodes hold exactly the values k global steps would give (every node's
// update is the same function of the same inputs).  A block then waits only
// for the CTAs it shares halo nodes with (their published block counts),
// instead of a grid barrier per step.  k is the largest depth whose halo and EF
// entries fit every CTA's shared memory (at most the block depth, 4 by
// default); k = 0 falls back to one barrier per step.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>


#include <algorithm>

#include "f2m_device.cuh"
#include "f2m_internal.h"

namespace f2m {

constexpr int kGT = 1024;              // threads per CTA (one CTA per SM: fewer barrier arrivals)
constexpr int kMaxBlk = 16;            // most Jacobi steps between two grid barriers
constexpr int kMaxNl = 2048;           // most nodes in a CTA's halo
constexpr int kHaloPf = 4;             // EF entries loaded ahead in the halo build
constexpr unsigned long long kHEmpty = ~0ull;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_i32(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned* p, unsigned x) {
    unsigned v;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "r"(x) : "memory");
    return v;
}
__device__ __forceinline__ void red_add_release_u32(unsigned* p, unsigned x) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(x) : "memory");
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned x) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(x) : "memory");
}

// Potentials written by other SMs are read through L2 (ld.global.cg): the
// grid barrier orders the writes, and bypassing L1 keeps a stale line of an
// earlier iteration out (the two buffers alternate every step).
struct L2Ptr {
    const double* p;
    __device__ __forceinline__ double operator[](int64_t i) const { return __ldcg(p + i); }
};

// grad/2 of one node from its EF list (cuda_get_Nodes_grad_R,
// graph_cuda_grad.hpp): from the three smallest of the reduced costs and two
// 1e6 sentinels.  Each word holds the neighbour's index into H and, in bit
// 31, whether the neighbour is the lower node id (the order of the two
// additions).  Entry k of a list is at Dp[k * ST], Wp[k * ST] (ST = 1:
// contiguous lists; ST = 32: SELL-32 slices, entry k of 32 nodes side by
// side).  The global and the halo steps both run this code, so their results
// are identical.
//
// While the first reduced cost is below 1e6 (always, in practice) the
// reference's compare chain is a sorted insertion (top3_insert); otherwise
// the chain itself runs (it can then leave the triple unsorted).
template <class HA>
__device__ __forceinline__ double red_x(uint32_t w, double d, const HA& H, double hv) {
    const double hw = H[w & 0x7fffffffu];
    const bool first = (w >> 31) != 0;
    return (d + (first ? hw : hv)) + (first ? hv : hw);
}
template <int ST, class HA>
__device__ __forceinline__ double grad_chain(int n, const double* Dp, const uint32_t* Wp, const HA& H, double hv) {
    double x0 = red_x(Wp[0], Dp[0], H, hv), x1 = 1e6, x2 = 1e6;
    for (int k = 1; k < n; ++k) {
        const double x = red_x(Wp[k * ST], Dp[k * ST], H, hv);
        if (x < x0) { x2 = x1; x1 = x0; x0 = x; continue; }
        if (x < x1) { x2 = x1; x1 = x; continue; }
        if (x < x2) { x2 = x; }
    }
    return (-(x1 + x2) / 2) * 0.5;
}
template <int ST, class HA>
__device__ __forceinline__ double grad_half(int n, const double* Dp, const uint32_t* Wp, const HA& H, double hv) {
    if (n <= 0) return (-(1e6 + 1e6) / 2) * 0.5;
    const double xf = red_x(Wp[0], Dp[0], H, hv);
    if (!(xf < 1e6)) return grad_chain<ST>(n, Dp, Wp, H, hv);
    double a0 = xf, a1 = 1e6, a2 = 1e6;
    // unrolled by eight (measured against four, and against loading four
    // entries ahead of their insertions: 39.3 / 39.4 / 41.0 ms on 100k points)
#pragma unroll 8
    for (int k = 1; k < n; ++k) top3_insert(red_x(Wp[k * ST], Dp[k * ST], H, hv), a0, a1, a2);
    return (-(a1 + a2) / 2) * 0.5;
}

constexpr int kPartCap = 128;  // longest list partitioned in shared memory by a warp
// halo entries (12 B each) whose room holds the partition scratch of 32 warps
constexpr int kPartScratchEntries = (32 * kPartCap * 11 + 11) / 12;

// update_EF's copy of node v's list prefix (n slots in list order) to the
// slot-indexed arena and, when eD is not null, to the shared-memory cache;
// restrict pointers let the compiler issue an unrolled group's loads before
// its stores.
__device__ __forceinline__ void copy_ef_words(const Slot* __restrict__ ps, double* __restrict__ gD,
                                              uint32_t* __restrict__ gW, double* __restrict__ eD,
                                              uint32_t* __restrict__ eW, int n, int v) {
#pragma unroll 4
    for (int k = 0; k < n; ++k) {
        const Slot sl = ps[k];
        const uint32_t w = (uint32_t)sl.nbr | (sl.nbr < v ? 0x80000000u : 0u);
        gD[k] = sl.D;
        gW[k] = w;
        if (eD) { eD[k] = sl.D; eW[k] = w; }
    }
}

// Open-addressing table node -> local index in shared memory (the halo
// build).  An entry is (node << 32 | local index); node ids are below 2^31,
// so the all-ones word marks a free entry.
__device__ __forceinline__ unsigned hslot(int key, unsigned mask) { return ((unsigned)key * 2654435761u) & mask; }

// Inserts `key` if absent, numbering it with the next local index; returns
// false when the table is full (the caller gives up the deeper levels).
__device__ __forceinline__ bool h_insert(unsigned long long* ht, unsigned mask, int key, int* count, int* map,
                                         int nl) {
    volatile unsigned long long* vt = ht;
    const unsigned long long tag = (unsigned long long)(unsigned)key << 32;
    unsigned h = hslot(key, mask);
    for (unsigned p = 0; p <= mask; ++p, h = (h + 1) & mask) {
        unsigned long long cur = vt[h];
        if (cur == kHEmpty) {
            cur = atomicCAS(ht + h, kHEmpty, tag | 0xffffffffull);
            if (cur == kHEmpty) {
                const int idx = atomicAdd(count, 1);
                if (idx < nl) map[idx] = key;
                atomicExch(ht + h, tag | (unsigned)idx);
                return true;
            }
        }
        if ((cur >> 32) == (unsigned)key) return true;
    }
    return false;
}
// h_insert for a whole warp (every lane calls it; key -1: nothing to
// insert): each lane claims its key's slot, then one counter update per
// warp numbers the keys claimed.  Returns false in a lane whose table probe
// found no room.
__device__ __forceinline__ bool h_insert_warp(unsigned long long* ht, unsigned mask, int key, int* count,
                                              int* map, int nl, int lane) {
    int slot = -1;
    bool ok = true;
    if (key >= 0) {
        volatile unsigned long long* vt = ht;
        const unsigned long long tag = (unsigned long long)(unsigned)key << 32;
        unsigned h = hslot(key, mask);
        ok = false;
        for (unsigned p = 0; p <= mask; ++p, h = (h + 1) & mask) {
            unsigned long long cur = vt[h];
            if (cur == kHEmpty) {
                cur = atomicCAS(ht + h, kHEmpty, tag | 0xffffffffull);
                if (cur == kHEmpty) { slot = (int)h; ok = true; break; }
            }
            if ((cur >> 32) == (unsigned)key) { ok = true; break; }
        }
    }
    const unsigned fm = __ballot_sync(0xffffffffu, slot >= 0);
    if (fm) {
        int base = 0;
        if (lane == 0) base = atomicAdd(count, __popc(fm));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (slot >= 0) {
            const int idx = base + __popc(fm & ((1u << lane) - 1u));
            if (idx < nl) map[idx] = key;
            atomicExch(ht + slot, ((unsigned long long)(unsigned)key << 32) | (unsigned)idx);
        }
    }
    return ok;
}
// largest j in [0, n) with a[j] <= x (a ascending, a[0] <= x)
__device__ __forceinline__ int upper_idx(const int* a, int n, int x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int h_find(const unsigned long long* ht, unsigned mask, int key) {
    unsigned h = hslot(key, mask);
    for (unsigned p = 0; p <= mask; ++p, h = (h + 1) & mask) {
        const unsigned long long cur = ht[h];
        if (cur == kHEmpty) return -1;
        if ((cur >> 32) == (unsigned)key) return (int)(unsigned)cur;
    }
    return -1;
}
// sets the local index of a key that is in the table
__device__ __forceinline__ void h_set(unsigned long long* ht, unsigned mask, int key, int idx) {
    unsigned h = hslot(key, mask);
    for (unsigned p = 0; p <= mask; ++p, h = (h + 1) & mask)
        if ((ht[h] >> 32) == (unsigned)key) {
            ht[h] = ((unsigned long long)(unsigned)key << 32) | (unsigned)idx;
            return;
        }
}

// Shared-memory halo of one CTA.  Local nodes are numbered by EF-hop level:
// [0, lend[0]) are the CTA's own nodes, [lend[d-1], lend[d]) those first
// reached after d hops; inside a level, by decreasing list length.
struct Halo {
    double* h;             // [2*nl] potentials of the local nodes (two buffers); hash table while building
    int* map;              // [nl] local index -> node
    int* nn;               // [nl+1] EF list length of each computed node
    double* D;             // [ne] EF entries in SELL-32 slices: reduced-cost base D
    uint32_t* W;           // [ne] local neighbour index | lower-id flag
    int* lend;             // shared [kMaxBlk+1]
    int* cnt;              // shared [2]: inserted nodes, table-full flag
    int* sb;               // shared [kMaxNl/32+1]: first entry of each 32-node slice
    int* hist;             // shared [kGT]: counting-sort buckets (level, list length)
    int nl = 0, ne = 0;
    int nb = 0;            // own nodes [0, nb) are read by other CTAs' halos
    int kmax = 0;
    int K = 0;             // steps per block of the current active sets (same on every CTA)
    bool built = false;
    long long own_slots = 0;  // EF entries of this thread's own nodes
};

struct GridSolver {
    const Batch& B;
    const DevParams& P;
    const GridState& G;
    const Inst& I;
    int b;
    int o0, o1;            // this CTA's nodes: G.own[o0 .. o1)
    int64_t row0;          // first slot of the instance
    double* Hc;
    double* Hn;
    double* eD;            // shared-memory EF cache of this CTA's own nodes
    uint32_t* eW;
    int cap;
    int* sefo;             // shared: offset of each own node's EF list in the cache
    double* sred;
    long long* sredl;
    int* swarp;
    unsigned long long* sbcv;  // shared broadcast slot of the grid reductions
    int* sflag;                // shared: barrier error flag of this CTA
    int* snb;                  // shared: neighbour CTAs of the halo blocks
    int* snbn;                 // shared: their count
    unsigned* swm;             // shared: mask of the CTAs whose nodes the halo reads
    unsigned pcount = 0;       // halo blocks this CTA has completed
    Halo L;
    int phase = 0;
    long long iters = 0, wslots = 0;
    int checks = 0;
    bool capped = false;
    bool dead = false;     // a barrier timed out

    __device__ int nown() const { return o1 - o0; }
    __device__ int node(int i) const { return G.own[o0 + i]; }  // i-th own node
    __device__ int deg(int v) const { return (int)(I.row[v + 1] - I.row[v]); }

    // Bounded grid barrier (arrival count + generation).  Thread 0 of each CTA
    // arrives with an acquire-release atomic (after the CTA barrier, so it
    // releases the whole CTA's writes), the last arrival resets the count and
    // releases the next generation, the others spin on it with acquire loads;
    // the error flag is polled every 64 spins and broadcast through shared
    // memory, so one thread per CTA touches the barrier words.
    __device__ bool sync() {
        __syncthreads();
        if (threadIdx.x == 0) {
            int bad = ld_acquire_i32(G.err);
            if (!bad) {
                unsigned* gen = G.bar + 1;
                const unsigned g = ld_acquire_u32(gen);
                const unsigned arrived = atom_add_acq_rel_u32(G.bar, 1u);
                if (arrived == gridDim.x - 1) {
                    G.bar[0] = 0;
                    red_add_release_u32(gen, 1u);
                } else {
                    for (long long spins = 1; ld_acquire_u32(gen) == g; ++spins) {
                        if ((spins & 63) == 0 && (bad = ld_acquire_i32(G.err)) != 0) break;
                        if (spins > P.spin_limit) { atomicExch(G.err, 1); bad = 1; break; }
                    }
                }
            }
            *sflag = bad;
        }
        __syncthreads();
        dead = *sflag != 0;
        return !dead;
    }
    // Neighbour waits of the halo blocks.  A block of CTA c reads the
    // potentials of the nodes within K hops of its own (other CTAs' nodes)
    // from one buffer and writes its own nodes to the other, so before block
    // j it needs (a) block j-1 of every CTA whose nodes it reads (their
    // values) and (b) block j-1 of every CTA that reads its nodes (those
    // finished reading the buffer that block j overwrites).  Each CTA
    // publishes its completed block count (a release store after a CTA
    // barrier, as the grid barrier's arrival); warp 0 waits, one
    // neighbour per lane, with acquire loads bounded like the grid barrier.  CTAs that share no halo node do not
    // wait on each other.
    __device__ bool wait_neighbours() {
        if (threadIdx.x < 32) {
            int bad = 0;
            if (threadIdx.x == 0) bad = ld_acquire_i32(G.err);
            bad = __shfl_sync(0xffffffffu, bad, 0);
            const int n = *snbn;
            for (int j = threadIdx.x; j < n && !bad; j += 32) {
                const unsigned* f = G.prog + snb[j];
                for (long long spins = 1; (int)(ld_acquire_u32(f) - pcount) < 0; ++spins) {
                    if ((spins & 63) == 0 && ld_acquire_i32(G.err) != 0) { bad = 1; break; }
                    if (spins > P.spin_limit) { atomicExch(G.err, 1); bad = 1; break; }
                }
            }
            bad = __any_sync(0xffffffffu, bad);
            if (threadIdx.x == 0) *sflag = bad;
        }
        __syncthreads();
        dead = *sflag != 0;
        return !dead;
    }
    __device__ void publish_block() {
        __syncthreads();  // every own potential of the block is written
        // the last warp releases the CTA's writes (its store waits for them),
        // so warp 0 can already poll the neighbours of the next block
        if (threadIdx.x == kGT - 32) st_release_u32(G.prog + blockIdx.x, pcount + 1);
        ++pcount;
    }
    // Deterministic grid reductions through per-CTA partials (double-buffered).
    // After the barrier one warp per CTA reads the partials (lane-strided, then
    // a fixed shuffle tree) and broadcasts through shared memory, so every CTA
    // computes the same value in the same order.
    template <class T, class Op>
    __device__ T greduce(T x, T* part, T ident, Op op) {
        if (threadIdx.x == 0) part[phase * gridDim.x + blockIdx.x] = x;
        sync();
        if (threadIdx.x < 32) {
            const volatile T* pp = part + phase * gridDim.x;
            T r = ident;
            for (unsigned k = threadIdx.x; k < gridDim.x; k += 32) r = op(r, pp[k]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r = op(r, __shfl_xor_sync(0xffffffffu, r, o));
            if (threadIdx.x == 0) *reinterpret_cast<T*>(sbcv) = r;
        }
        __syncthreads();
        const T r = *reinterpret_cast<const T*>(sbcv);
        __syncthreads();
        phase ^= 1;
        return r;
    }
    __device__ double gmax(double x) {
        x = block_max<kGT>(x, sred);
        return greduce<double>(x, G.part, -INFINITY, [](double a, double b) { return fmax(a, b); });
    }
    __device__ double gsum(double x) {
        x = block_sum<kGT>(x, sred);
        return greduce<double>(x, G.part, 0.0, [](double a, double b) { return a + b; });
    }
    __device__ long long gsum_ll(long long x) {
        x = block_sum_ll<kGT>(x, sredl);
        return greduce<long long>(x, G.partl, 0LL, [](long long a, long long b) { return a + b; });
    }
    __device__ long long gmax_ll(long long x) {
        x = block_max_ll<kGT>(x, sredl);
        return greduce<long long>(x, G.partl, LLONG_MIN,
                                  [](long long a, long long b) { return a > b ? a : b; });
    }

    __device__ __forceinline__ L2Ptr hc() const { return L2Ptr{Hc}; }

    // grad/2 of the i-th own node over its EF list (the first efcnt slots of
    // its list, held in shared memory or in the slot-indexed arena)
    __device__ double hgrad(int i, int v) const {
        const int n = G.efc[v];
        const int lo = sefo[i];
        const bool sm = lo + n <= cap;
        const int64_t go = I.row[v] - row0;
        const double* Dp = sm ? eD + lo : G.gD + go;
        const uint32_t* Wp = sm ? eW + lo : G.gW + go;
        const L2Ptr H = hc();
        return grad_half<1>(n, Dp, Wp, H, H[v]);
    }
    __device__ void swap_h() { double* t = Hc; Hc = Hn; Hn = t; }
    // one global Jacobi step (one grid barrier)
    template <bool MASKED>
    __device__ void step() {
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            const double g = hgrad(i, v);
            const double h = hc()[v];
            Hn[v] = (MASKED && B.shift[I.base + v] != 0.0) ? h : h + g;
            wslots += G.efc[v];  // this thread's active slots
        }
        sync();
        swap_h();
        iters++;
    }
    __device__ double grad_max() {
        double m = 0.0;
        for (int i = threadIdx.x; i < nown(); i += kGT) m = fmax(m, fabs(hgrad(i, node(i))));
        return 2.0 * gmax(m);
    }
    // EF-list offsets of the own nodes in the shared cache
    __device__ void own_offsets() {
        __syncthreads();
        int carry = 0;
        for (int r = 0; r < nown(); r += kGT) {
            const int i = r + threadIdx.x;
            const int c = (i < nown()) ? G.efc[node(i)] : 0;
            int tot;
            const int ex = block_excl_scan<kGT>(c, swarp, &tot);
            if (i < nown()) sefo[i] = carry + ex;
            carry += tot;
        }
        if (threadIdx.x == 0) sefo[nown()] = carry;
        __syncthreads();
    }
    // update_EF for this CTA's nodes: local offsets, shared cache, arena copy
    __device__ void rebuild_ef() {
        own_offsets();
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            const int64_t r0 = I.row[v];
            const int n = G.efc[v], lo = sefo[i];
            const int64_t go = r0 - row0;
            const bool sm = lo + n <= cap;
            copy_ef_words(I.pslot + r0, G.gD + go, G.gW + go, sm ? eD + lo : nullptr, sm ? eW + lo : nullptr, n, v);
        }
        __syncthreads();
        L.built = false;
    }

    // Halo of the current EF lists: levels by EF hops from the own nodes,
    // then the deepest k (<= kmax) whose nodes and entries fit, agreed over
    // the grid (the minimum), then the entries of the nodes the steps
    // recompute with their neighbours renumbered to local indices.  Other
    // CTAs' lists and counts are read through L2 (ld.global.cg).
    __device__ void build_halo() {
        L.built = true;
        L.K = 0;
        if (L.nl == 0) return;
        for (int w = threadIdx.x; w < kGridNbWords; w += kGT) G.nbm[(size_t)blockIdx.x * kGridNbWords + w] = 0;
        for (int i = threadIdx.x; i < nown(); i += kGT) G.rd[node(i)] = 0;
        sync();  // every CTA's efc and arena lists are complete (the reader rows and marks clear)
        if (dead) return;
        unsigned long long* ht = reinterpret_cast<unsigned long long*>(L.h);
        const unsigned mask = 2u * (unsigned)L.nl - 1u;
        for (unsigned h = threadIdx.x; h <= mask; h += kGT) ht[h] = kHEmpty;
        if (threadIdx.x == 0) { L.cnt[0] = 0; L.cnt[1] = 0; }
        __syncthreads();
        int depth = -1;
        if (nown() <= L.nl) {
            for (int i = threadIdx.x; i < nown(); i += kGT)
                if (!h_insert(ht, mask, node(i), L.cnt, L.map, L.nl)) L.cnt[1] = 1;
            __syncthreads();
            if (!L.cnt[1]) {
                L.lend[0] = nown();
                depth = 0;
            }
            __syncthreads();
            for (int d = 1; d <= L.kmax && depth == d - 1; ++d) {
                const int f0 = d == 1 ? 0 : L.lend[d - 2], f1 = L.lend[d - 1];
                // the frontier's EF entries, flattened (a thread per entry, so
                // a long list does not hold up its level): prefix of the list
                // lengths in pre, first slot of each list in gof (the entry
                // arrays are free while the levels are built)
                const int F = f1 - f0;
                int* pre = reinterpret_cast<int*>(L.W);
                long long* gof = reinterpret_cast<long long*>(L.D);
                int carry = 0;
                for (int r = 0; r < F; r += kGT) {
                    const int j = r + threadIdx.x;
                    int n = 0;
                    if (j < F) {
                        const int u = L.map[f0 + j];
                        n = __ldcg(G.efc + u);
                        gof[j] = I.row[u] - row0;
                    }
                    int tot;
                    const int ex = block_excl_scan<kGT>(n, swarp, &tot);
                    if (j < F) pre[j] = carry + ex;
                    carry += tot;
                }
                __syncthreads();
                const int lane = threadIdx.x & 31;
                for (int e0 = 0; e0 < carry; e0 += kHaloPf * kGT) {  // same trip count in a warp
                    int key[kHaloPf];
#pragma unroll
                    for (int c = 0; c < kHaloPf; ++c) {  // the chunk's loads in flight together
                        const int e = e0 + c * kGT + threadIdx.x;
                        key[c] = -1;
                        if (e < carry) {
                            const int j = upper_idx(pre, F, e);
                            key[c] = (int)(__ldcg(G.gW + gof[j] + (e - pre[j])) & 0x7fffffffu);
                        }
                    }
#pragma unroll
                    for (int c = 0; c < kHaloPf; ++c)
                        if (!h_insert_warp(ht, mask, key[c], L.cnt, L.map, L.nl, lane)) L.cnt[1] = 1;
                }
                __syncthreads();
                const int c = L.cnt[0], full = L.cnt[1];
                if (!full && c <= L.nl) {
                    if (threadIdx.x == 0) L.lend[d] = c;
                    depth = d;
                }
                __syncthreads();
            }
        }
        // Mark the nodes of levels 1..depth (other CTAs' nodes this CTA's
        // blocks read); after a grid barrier every CTA knows which of its own
        // nodes other CTAs read, and a block computes and publishes those
        // first.
        if (depth >= 1)
            for (int i = L.lend[0] + threadIdx.x; i < L.lend[depth]; i += kGT) G.rd[L.map[i]] = 1;
        sync();
        if (dead) return;
        // The nodes of levels < depth (the ones a block may recompute) are
        // renumbered level by level in decreasing list length, so the
        // 32-node slices of the SELL layout carry little padding; a counting
        // sort over (group, 31 - min(length, 31)) keeps the groups in order:
        // own nodes other CTAs read, the other own nodes, then level 1, 2, ...
        int kc = 0;
        L.nb = 0;
        if (depth >= 1) {
            const int nc = L.lend[depth - 1];  // <= nl
            L.hist[threadIdx.x] = 0;
            __syncthreads();
            long long* order = reinterpret_cast<long long*>(L.D);  // (length, node) in the new order, staged
            int* len = reinterpret_cast<int*>(L.W);                  // list lengths, staged
            for (int i = threadIdx.x; i < nc; i += kGT) {  // bucket and rank, staged in nn
                const int n = __ldcg(G.efc + L.map[i]);
                int lvl = 0;
                while (i >= L.lend[lvl]) ++lvl;
                const int grp = lvl == 0 ? (__ldcg(G.rd + L.map[i]) ? 0 : 1) : lvl + 1;
                const int key = grp * 32 + 31 - min(n, 31);
                L.nn[i] = (key << 16) | atomicAdd(L.hist + key, 1);
                len[i] = n;
            }
            __syncthreads();
            {
                int tot;
                const int ex = block_excl_scan<kGT>(L.hist[threadIdx.x], swarp, &tot);
                __syncthreads();
                L.hist[threadIdx.x] = ex;
            }
            __syncthreads();
            L.nb = L.hist[32];  // own nodes other CTAs read
            for (int i = threadIdx.x; i < nc; i += kGT) {
                const int kr = L.nn[i];
                order[L.hist[kr >> 16] + (kr & 0xffff)] = ((long long)len[i] << 32) | (unsigned)L.map[i];
            }
            __syncthreads();
            for (int i = threadIdx.x; i < nc; i += kGT) {
                const long long o = order[i];
                const int u = (int)(unsigned)o;
                L.map[i] = u;
                L.nn[i] = (int)(o >> 32);
                h_set(ht, mask, u, i);
            }
            __syncthreads();
            // slice widths (warp-wide max) and their prefix
            const int ns = (nc + 31) / 32;
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            for (int sl = wid; sl < ns; sl += kGT / 32) {
                const int i = sl * 32 + lane;
                const int wdt = __reduce_max_sync(0xffffffffu, i < nc ? L.nn[i] : 0);
                if (lane == 0) L.sb[sl + 1] = wdt * 32;
            }
            __syncthreads();
            if (threadIdx.x < 32) {  // prefix of the slice sizes (ns <= 64), one warp
                const int lane = threadIdx.x;
                int carry = 0;
                for (int c0 = 1; c0 <= ns; c0 += 32) {
                    const int sl = c0 + lane;
                    int x = sl <= ns ? L.sb[sl] : 0;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (sl <= ns) L.sb[sl] = carry + x;
                    carry += __shfl_sync(0xffffffffu, x, 31);
                }
                if (lane == 0) L.sb[0] = 0;
            }
            __syncthreads();
            for (int k = depth; k >= 1; --k)
                if (L.sb[(L.lend[k - 1] + 31) / 32] <= L.ne) { kc = k; break; }
        }
        // the entries of levels < kc, neighbours renumbered to local indices:
        // entry k of node i at sb[i/32] + 32 k + i%32
        if (threadIdx.x == 0) L.cnt[1] = 0;
        __syncthreads();
        if (kc >= 1) {
            // a thread per SELL position (padding positions skip): slice s
            // holds positions [sb[s], sb[s+1]), entry k of its node i at
            // sb[s] + 32 k + i % 32
            const int nc = L.lend[kc - 1];
            const int ns = (nc + 31) / 32;
            const int np = L.sb[ns];
            for (int p0 = 0; p0 < np; p0 += kHaloPf * kGT) {
                uint32_t w[kHaloPf];
                double dd[kHaloPf];
                int pos[kHaloPf];
#pragma unroll
                for (int c = 0; c < kHaloPf; ++c) {  // the chunk's loads in flight together
                    const int p = p0 + c * kGT + threadIdx.x;
                    pos[c] = -1;
                    if (p < np) {
                        const int sl = upper_idx(L.sb, ns, p);
                        const int r = p - L.sb[sl];
                        const int i = sl * 32 + (r & 31), k = r >> 5;
                        if (i < nc && k < L.nn[i]) {
                            const int64_t go = I.row[L.map[i]] - row0 + k;
                            w[c] = __ldcg(G.gW + go);
                            dd[c] = __ldcg(G.gD + go);
                            pos[c] = p;
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < kHaloPf; ++c) {
                    if (pos[c] < 0) continue;
                    const int li = h_find(ht, mask, (int)(w[c] & 0x7fffffffu));
                    if (li < 0 || li >= L.lend[kc]) L.cnt[1] = 1;  // cannot happen: all within kc hops
                    L.D[pos[c]] = dd[c];
                    L.W[pos[c]] = (uint32_t)(li < 0 ? 0 : li) | (w[c] & 0x80000000u);
                }
            }
        }
        __syncthreads();
        if (L.cnt[1]) kc = 0;
        L.own_slots = 0;
        for (int i = threadIdx.x; i < nown(); i += kGT) L.own_slots += G.efc[node(i)];
        L.K = (int)(-gmax_ll(-(long long)kc));
        __syncthreads();
        // neighbour CTAs of the blocks: the owners of the nodes the blocks
        // read (levels 1..K) and the CTAs whose blocks read this CTA's nodes
        if (L.K > 0) {
            for (int w = threadIdx.x; w < kGridNbWords; w += kGT) swm[w] = 0;
            __syncthreads();
            for (int i = L.lend[0] + threadIdx.x; i < L.lend[L.K]; i += kGT) {
                const int c = __ldcg(G.owner + L.map[i]);
                if (c != (int)blockIdx.x) atomicOr(swm + (c >> 5), 1u << (c & 31));
            }
            __syncthreads();
            for (int w = threadIdx.x; w < kGridNbWords; w += kGT)
                for (unsigned m = swm[w]; m; m &= m - 1) {
                    const int c = w * 32 + __ffs(m) - 1;
                    atomicOr(G.nbm + (size_t)c * kGridNbWords + (blockIdx.x >> 5), 1u << (blockIdx.x & 31));
                }
            sync();
            if (threadIdx.x == 0) {
                int cnt = 0;
                for (int w = 0; w < kGridNbWords; ++w) {
                    unsigned m = swm[w] | __ldcg(G.nbm + (size_t)blockIdx.x * kGridNbWords + w);
                    if (w == (int)(blockIdx.x >> 5)) m &= ~(1u << (blockIdx.x & 31));
                    for (; m; m &= m - 1) snb[cnt++] = w * 32 + __ffs(m) - 1;
                }
                *snbn = cnt;
            }
            __syncthreads();
        }
    }

    // n unmasked Jacobi steps: blocks of K halo steps, each after a wait on
    // the neighbour CTAs only, and one grid barrier at the end; or single
    // global steps (a grid barrier each) when no halo fits
    __device__ void steps(int n) {
        if (!L.built) build_halo();
        if (L.K == 0) {
            for (int it = 0; it < n && !dead; ++it) step<false>();
            return;
        }
        double* A = L.h;
        double* Bn = L.h + L.nl;
        for (int done = 0; done < n && !dead;) {
            const int k = min(L.K, n - done);
            if (!wait_neighbours()) break;
            const L2Ptr H = hc();
            // after the first block the own nodes ([0, lend[0])) already hold
            // this CTA's last values in A
            for (int i = (done == 0 ? 0 : L.lend[0]) + threadIdx.x; i < L.lend[k]; i += kGT) A[i] = H[L.map[i]];
            __syncthreads();
            for (int t = 1; t <= k; ++t) {
                const int m = L.lend[k - t];  // nodes within k-t hops
                // the last step updates the own nodes (m = lend[0]): those
                // other CTAs read are written to H and published first; the
                // rest stay in shared memory (written to H once, after the
                // last block)
                const bool last = t == k;
                for (int part = 0; part < (last ? 2 : 1); ++part) {
                    const int i0 = (last && part == 1) ? L.nb : 0;
                    const int i1 = (last && part == 0) ? L.nb : m;
                    for (int i = i0 + threadIdx.x; i < i1; i += kGT) {
                        const int lo = L.sb[i >> 5] + (i & 31);
                        const double h = A[i];
                        const double hn = h + grad_half<32>(L.nn[i], L.D + lo, L.W + lo, A, h);
                        Bn[i] = hn;
                        if (last && part == 0) Hn[L.map[i]] = hn;
                    }
                    if (last && part == 0) publish_block();
                }
                __syncthreads();
                double* t2 = A;
                A = Bn;
                Bn = t2;
            }
            wslots += (long long)k * L.own_slots;
            iters += k;
            done += k;
            swap_h();
        }
        // the own nodes no other CTA reads, into the current buffer
        if (n > 0)
            for (int i = L.nb + threadIdx.x; i < L.lend[0] && !dead; i += kGT) Hc[L.map[i]] = A[i];
        sync();  // every CTA's last block is written before grid-wide reads of H
    }

    // update_EF's partitions of the own nodes' lists (cuda_partition_v2 with
    // threshold thr, or v4 with the largest of the first glob_K reduced costs
    // when glob): warps take the own nodes from a shared counter; a list of up to
    // kPartCap entries is copied with its reduced costs into the warp's
    // shared scratch in one parallel round of loads and partitioned there by
    // the whole warp (warp_qpart_ef_vals; the halo region is free here: it is
    // rebuilt after every update_EF); one lane runs the global-memory partition for a longer
    // list.  Without the scratch (no halo), a thread per node partitions in
    // global memory.
    __device__ void partition_own(bool glob, double thr) {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        // per warp: kPartCap values (8 B), list entries (2 B) and rank positions (1 B)
        const bool scratch = L.nl > 0 && L.ne >= kPartScratchEntries;
        double* val = L.D + wid * kPartCap;
        uint16_t* pl = reinterpret_cast<uint16_t*>(L.D + 32 * kPartCap) + wid * kPartCap;
        uint8_t* pos = reinterpret_cast<uint8_t*>(reinterpret_cast<uint16_t*>(L.D + 32 * kPartCap) + 32 * kPartCap) +
                       wid * kPartCap;
        const L2Ptr H = hc();
        if (!scratch) {  // no shared scratch: a thread per node, in global memory
            for (int i = threadIdx.x; i < nown(); i += kGT) {
                const int v = node(i);
                const int d = deg(v);
                if (glob ? d < P.glob_K : d < P.ef_small_deg) { G.efc[v] = d; continue; }
                const int64_t r0 = I.row[v];
                double avg = thr;
                if (glob) {
                    const double hv = H[v];
                    avg = pdv(I, r0, 0, v, H, hv);
                    for (int k = 1; k < P.glob_K; ++k) avg = fmax(avg, pdv(I, r0, k, v, H, hv));
                }
                G.efc[v] = qpart_ef_pair(I, r0, v, H, d, avg, P.ef_min);
            }
            __syncthreads();
            return;
        }
        // warps take the own nodes from a shared counter (the halo build's,
        // free until the next build), so a warp that drew long lists does
        // not hold up the CTA
        if (threadIdx.x == 0) L.cnt[0] = 0;
        __syncthreads();
        for (;;) {
            int i = 0;
            if (lane == 0) i = atomicAdd(L.cnt, 1);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= nown()) break;
            const int v = node(i);
            const int d = deg(v);
            if (glob ? d < P.glob_K : d < P.ef_small_deg) {
                if (lane == 0) G.efc[v] = d;
                continue;
            }
            const int64_t r0 = I.row[v];
            uint16_t* list = I.perm + r0;
            int p = 0;
            if (d <= kPartCap) {
                // pslot holds the slots in list order, so a reduced cost is two
                // dependent loads (the slot, then the neighbour's potential)
                const double hv = H[v];
                uint16_t q0[kPartCap / 32];
#pragma unroll
                for (int c = 0; c < kPartCap / 32; ++c) {
                    const int k = c * 32 + lane;
                    if (k < d) {
                        q0[c] = list[k];
                        pl[k] = q0[c];
                        val[k] = red_d(I.pslot[r0 + k], v, H, hv);
                    }
                }
                __syncwarp();
                double avg = thr;
                if (glob) {
                    avg = val[0];
                    for (int k = 1; k < P.glob_K; ++k) avg = fmax(avg, val[k]);
                }
                p = warp_qpart_ef_vals<kPartCap / 32>(pl, val, pos, d, avg, P.ef_min, lane);
                __syncwarp();
#pragma unroll
                for (int c = 0; c < kPartCap / 32; ++c) {  // only the positions the swaps changed
                    const int k = c * 32 + lane;
                    if (k < d && pl[k] != q0[c]) {
                        list[k] = pl[k];
                        I.pslot[r0 + k] = I.slot[r0 + pl[k]];
                    }
                }
                __syncwarp();
            } else if (lane == 0) {
                double avg = thr;
                if (glob) {
                    const double hv = H[v];
                    avg = pdv(I, r0, 0, v, H, hv);
                    for (int k = 1; k < P.glob_K; ++k) avg = fmax(avg, pdv(I, r0, k, v, H, hv));
                }
                p = qpart_ef_la(I, r0, v, H, d, avg, P.ef_min);
            }
            if (lane == 0) G.efc[v] = p;
        }
        __syncthreads();
    }

    __device__ double check_opt() {
        partition_own(false, P.ef_thr);
        rebuild_ef();
        checks++;
        return grad_max();
    }
    // cuda_block_EF: N steps, or check_every when the gradient at entry is
    // already below error_B (the count check breaks there).  Every call
    // follows a check_OPT whose max |grad| was taken over the same
    // potentials and active sets, so that value is the entry gradient MA.
    __device__ void block_ef(int N, double MA) {
        steps(MA < P.error_B ? min(N, P.check_every) : N);
    }
    __device__ void block_glob() {
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            G.efc[v] = min(deg(v), P.glob_K);
        }
        rebuild_ef();
        for (int go = 0; go < P.glob_rounds && !dead; ++go) {
            steps(P.glob_inner);
            partition_own(true, 0.0);
            rebuild_ef();
            if (grad_max() < P.glob_tol) break;
        }
    }
    __device__ double run_start() {
        block_glob();
        double M = check_opt();
        int factor = P.factor0;
        for (int go = 1; go <= P.max_rounds && !dead; ++go) {
            block_ef(factor, M);
            M = check_opt();
            if (factor < P.factor_cap) factor += P.factor_step;
            if (M < P.error_B) break;
            if (iters > P.max_iters) { capped = true; break; }
        }
        return M;
    }
    __device__ double run_fix() {
        double M = check_opt();
        for (int go = 1; go <= P.fix_rounds && !dead; ++go) {
            block_ef(P.fix_factor, M);
            M = check_opt();
            if (M < P.error_B) break;
            if (iters > P.max_iters) { capped = true; break; }
        }
        return M;
    }
    __device__ void combs_and_primal(double M, bool accumulate) {
        const int V = I.V;
        const double porog = P.porog;
        int* ccnt = G.scratch;
        int* lab = G.scratch + V;
        for (int i = threadIdx.x; i < nown(); i += kGT) {  // cuda_partition_v3
            const int v = node(i);
            ccnt[v] = qpart_b_pair(I, I.row[v], v, hc(), G.efc[v], P.comb_thr);
        }
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            const int64_t r0 = I.row[v];
            const double hv = hc()[v];
            bool has = false;
            for (int k = 0; k < ccnt[v] && !has; ++k) {
                const double d = pdv(I, r0, k, v, hc(), hv);
                has = (d >= -porog && d <= porog);
            }
            lab[v] = has ? v : INT_MAX;
            G.irr[v] = 0;
        }
        sync();
        // components of half edges, rooted at their smallest id
        volatile int* vlab = lab;
        for (int round = 0; round < V + 1 && !dead; ++round) {
            long long changed = 0;
            for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
                int m = vlab[v];
                if (m == INT_MAX) continue;
                const int64_t r0 = I.row[v];
                const double hv = hc()[v];
                for (int k = 0; k < ccnt[v]; ++k) {
                    const Slot s = I.pslot[r0 + k];
                    const double d = red_d(s, v, hc(), hv);
                    if (d >= -porog && d <= porog) m = min(m, vlab[s.nbr]);
                }
                if (m < vlab[v]) { vlab[v] = m; changed = 1; }
            }
            if (gsum_ll(changed) == 0) break;
        }
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            B.F[I.base + v] = 2.0 * hc()[v];
            B.efcnt[I.base + v] = G.efc[v];
            B.ccnt[I.base + v] = ccnt[v];
        }
        volatile int* virr = G.irr;
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            const int l = vlab[v];
            if (l == INT_MAX) continue;
            const int64_t r0 = I.row[v], r1 = I.row[v + 1];
            const double hv = hc()[v];
            int A = 0, Bc = 0;
            for (int64_t a = r0; a < r1; ++a) {
                const double d = red_d(I.slot[a], v, hc(), hv);
                if (d < porog) { if (d > -porog) Bc++; else A++; }
            }
            if (4 - 2 * A - Bc != 0) virr[l] = 1;
        }
        sync();
        long long nc = 0, ni = 0;
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            if (vlab[v] == v) { nc++; ni += virr[v]; }
        }
        nc = gsum_ll(nc);
        ni = gsum_ll(ni);
        // irregular combs: Ax=b on the device (comb::solve_AxB,
        // comb_thread.cpp:272-304), a thread per comb -- the thread owning
        // its root.  The members of irregular combs are listed first as
        // (root, node) keys in the ownership-sort buffer (free by now); each
        // root's thread picks its own from that short list, in ascending
        // node order, and builds the system in the slice arena (unused by
        // this solver), handed out by an atomic counter.  The first solve
        // only: after a repair shift the host driver runs the comb stage
        // itself.  The instance goes to the host stage when a system does not
        // converge within 900 steps or the arena is full.
        bool solved = (ni == 0);
        if (ni > 0 && !accumulate && !dead) {
            unsigned long long* used = G.axb_used;      // [0] arena doubles, [1] listed members
            for (int i = threadIdx.x; i < nown(); i += kGT) {
                const int v = node(i);
                const int l = vlab[v];
                if (l == INT_MAX || !virr[l]) continue;
                const unsigned long long k = atomicAdd(used + 1, 1ull);
                G.okey[k] = ((unsigned long long)(unsigned)l << 32) | (unsigned)v;
            }
            sync();
            const long long nm = (long long)*(volatile unsigned long long*)(used + 1);
            long long bad = 0;
            for (int i = threadIdx.x; i < nown() && !dead; i += kGT) {
                const int r = node(i);
                if (vlab[r] != r || !virr[r]) continue;
                int m = 0, z = 0;
                for (long long k = 0; k < nm; ++k) {
                    const unsigned long long key = __ldcg(G.okey + k);
                    if ((int)(key >> 32) != r) continue;
                    m++;
                    z += count_b(I.slot, I.row, hc(), (int)(unsigned)key, porog);
                }
                const unsigned long long need = (unsigned long long)axb_comb_doubles(m, z);
                const unsigned long long off = atomicAdd(used, need);
                if (off + need > (unsigned long long)B.S_cap) { bad = 1; continue; }
                double* w = B.selD + off;
                int* mem = reinterpret_cast<int*>(w);
                int c = 0;
                for (long long k = 0; k < nm && c < m; ++k) {  // members, insertion-sorted
                    const unsigned long long key = __ldcg(G.okey + k);
                    if ((int)(key >> 32) != r) continue;
                    const int u = (int)(unsigned)key;
                    int p = c++;
                    while (p > 0 && mem[p - 1] > u) { mem[p] = mem[p - 1]; --p; }
                    mem[p] = u;
                }
                bad |= axb_comb(I.slot, I.row, row0, B.mirror, hc(), vlab, mem, m, z, r, porog,
                                w + (m + 1) / 2 + 1, B.xval);
            }
            solved = gsum_ll(bad) == 0;
        }
        double lp = 0.0, dual_neg = 0.0, fsum = 0.0;
        long long maxr = -1, viol = 0;
        for (int i = threadIdx.x; i < nown(); i += kGT) {
            const int v = node(i);
            const int64_t r0 = I.row[v], r1 = I.row[v + 1];
            const double hv = hc()[v];
            fsum += 2.0 * hv;
            float degsum = 0.0f;
            bool any = false;
            for (int64_t a = r0; a < r1; ++a) {
                const Slot s = I.slot[a];
                const double d = red_d(s, v, hc(), hv);
                double x = (d < porog) ? ((d > -porog) ? 0.5 : 1.0) : 0.0;
                uint8_t code = (uint8_t)(x == 1.0 ? 2 : (x == 0.5 ? 1 : 0));
                if (ni > 0 && solved && code == 1) {  // the edge's larger-root comb decides
                    const int l1 = vlab[v], l2 = vlab[s.nbr];
                    const int c = (l2 == INT_MAX) ? l1 : (l1 == INT_MAX ? l2 : ::max(l1, l2));
                    if (c != INT_MAX && virr[c]) { x = (double)__ldcg(B.xval + a); code = 3; }
                }
                B.xcode[a] = code;
                const bool in_x = (x != 0.0) || code == 3;  // every comb edge enters graph::X
                degsum += (float)x;
                any |= in_x;
                if (s.nbr > v) {
                    lp += x * B.s_cost[a];
                    dual_neg += fmin(0.0, d);
                    if (in_x) maxr = ::max(maxr, (long long)::min((int)(a - r0), B.mirror[a]));
                }
            }
            if (any && !(degsum > 2.0f - 1e-2f && degsum < 2.0f + 1e-2f)) viol++;
        }
        lp = gsum(lp);
        dual_neg = gsum(dual_neg);
        fsum = gsum(fsum);
        maxr = gmax_ll(maxr);
        viol = gsum_ll(viol);
        const long long wsum = gsum_ll(wslots);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            B.work_slots[b] = (accumulate ? B.work_slots[b] : 0) + wsum;
            B.work_pad[b] = (accumulate ? B.work_pad[b] : 0) + wsum;
            const double dmin = __longlong_as_double((long long)B.dmin_bits[b]);
            B.n_edges[b] = (int32_t)((I.row[V] - I.row[0]) / 2);
            B.n_combs[b] = (int32_t)nc;
            B.n_irr[b] = (int32_t)ni;
            B.max_rank[b] = (int32_t)maxr;
            B.deg_viol[b] = (int32_t)viol;
            B.iters[b] = (accumulate ? B.iters[b] : 0) + iters;
            B.work_nodes[b] = (accumulate ? B.work_nodes[b] : 0) + iters * (long long)V;
            B.checks[b] = (accumulate ? B.checks[b] : 0) + checks;
            B.max_grad[b] = M;
            B.dual[b] = dmin * (-fsum + dual_neg);
            if (dead) { B.status[b] = F2M_ERR_CUDA; B.lp[b] = NAN; }
            else if (capped) { B.status[b] = F2M_ERR_NOT_CONVERGED; B.lp[b] = NAN; }
            else if (!solved) { B.status[b] = kNeedsHost; B.lp[b] = NAN; }
            else { B.status[b] = F2M_OK; B.lp[b] = lp; }
        }
    }
};


__global__ void __launch_bounds__(kGT, 1) k_solve_grid(Batch B, DevParams P, GridState G, int b, int refit,
                                                     int cap, int nl, int ne, int kmax) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sred[kGT / 32];
    __shared__ long long sredl[kGT / 32];
    __shared__ int swarp[kGT / 32 + 1];
    __shared__ unsigned long long sbc[1];
    __shared__ int sflag[1];
    __shared__ int slend[kMaxBlk + 1];
    __shared__ int scnt[2];
    __shared__ int ssb[kMaxNl / 32 + 1];
    __shared__ int shist[kGT];
    __shared__ int snb[kGridMaxCtas];
    __shared__ int snbn[1];
    __shared__ unsigned swm[kGridNbWords];
    const Inst I = make_inst(B, b);
    const int V = I.V;
    const int o0 = (int)(((long long)V * blockIdx.x) / gridDim.x);
    const int o1 = (int)(((long long)V * (blockIdx.x + 1)) / gridDim.x);
    const int nv = o1 - o0;
    // shared layout: own offsets | own EF cache (cap) | halo potentials (2 nl)
    // | halo map (nl) | halo list lengths (nl+1) | halo entries (ne)
    int* sefo = reinterpret_cast<int*>(smem_raw);
    size_t off = (((size_t)nv + 1) * 4 + 15) / 16 * 16;
    double* eD = reinterpret_cast<double*>(smem_raw + off);
    off += (size_t)cap * 8;
    uint32_t* eW = reinterpret_cast<uint32_t*>(smem_raw + off);
    off += ((size_t)cap * 4 + 15) / 16 * 16;
    GridSolver S{B, P, G, I, b, o0, o1, I.row[0], G.Ha, G.Hb, eD, eW, cap, sefo, sred, sredl, swarp, sbc, sflag,
                 snb, snbn, swm};
    if (threadIdx.x == 0) snbn[0] = 0;
    S.L.h = reinterpret_cast<double*>(smem_raw + off);
    off += (size_t)nl * 16;
    S.L.map = reinterpret_cast<int*>(smem_raw + off);
    off += (size_t)nl * 4;
    S.L.nn = reinterpret_cast<int*>(smem_raw + off);
    off += (((size_t)nl + 1) * 4 + 15) / 16 * 16;
    S.L.D = reinterpret_cast<double*>(smem_raw + off);
    off += (size_t)ne * 8;
    S.L.W = reinterpret_cast<uint32_t*>(smem_raw + off);
    S.L.lend = slend;
    S.L.cnt = scnt;
    S.L.sb = ssb;
    S.L.hist = shist;
    S.L.nl = nl;
    S.L.ne = ne;
    S.L.kmax = min(kmax, kMaxBlk);
    double M;
    for (int i = threadIdx.x; i < nv; i += kGT) G.owner[S.node(i)] = (int32_t)blockIdx.x;
    // the own nodes' slots in list order (the host paths upload slot and perm)
    for (int i = threadIdx.x; i < nv; i += kGT) {
        const int v = S.node(i);
        const int64_t r0 = I.row[v];
        gather_slots(I.slot + r0, I.perm + r0, I.pslot + r0, I.row[v + 1] - r0);
    }
    if (!refit) {
        for (int i = threadIdx.x; i < nv; i += kGT) {
            const int v = S.node(i);
            G.Ha[v] = B.F0 ? 0.5 * B.F0[I.base + v] : 0.0;  // F = 0 or warm
        }
        S.sync();
        M = B.F0 ? S.run_fix() : S.run_start();  // a resumed descent skips the global phase
    } else {
        // cuda_IRREGULAR_B_recompute (graph_cuda_comb.hpp:542-574)
        for (int i = threadIdx.x; i < nv; i += kGT) {
            const int v = S.node(i);
            G.Ha[v] = 0.5 * (B.F[I.base + v] + B.shift[I.base + v]);
            G.efc[v] = B.efcnt[I.base + v];
        }
        // the EF lists of the last update_EF are in the slot-indexed arena
        S.own_offsets();
        for (int i = threadIdx.x; i < nv; i += kGT) {
            const int v = S.node(i);
            const int n = G.efc[v], lo = sefo[i];
            const int64_t go = I.row[v] - I.row[0];
            if (lo + n <= cap)
                for (int k = 0; k < n; ++k) { eD[lo + k] = G.gD[go + k]; eW[lo + k] = G.gW[go + k]; }
        }
        S.sync();
        for (int go = 0; go < P.frozen_iters && !S.dead; ++go) S.step<true>();
        M = S.run_fix();
    }
    S.combs_and_primal(M, refit != 0);
}

// Shared memory of one CTA: own-node offsets, the own EF cache (3 entries per
// node; longer lists are read from the arena), and the halo (nl local nodes
// at 24 B, the rest of the opt-in limit as 12-B entries).  nl is the power of
// two >= 3x the own nodes, 1,024-2,048; CTAs with more than 2,048 own nodes
// get no halo and step with one barrier per step.
// Kilobytes of the SM's shared-memory carve-out left to L1 (F2M_GRID_L1_KB
// overrides): this 64-register kernel spills, and its local loads miss an L1
// squeezed by a full shared-memory allocation.  The halo needs far fewer
// entries than a full allocation gives it on 10^5-point instances (100k
// points: 0 / 32 / 48 / 56 / 64 / 72 / 80 KB gave 39.8 / 35.9 / 35.9 / 35.9 /
// 34.9-35.2 / 38.5 / 39.4 ms: past 64 KB the halo of the long phases stops
// fitting).
static int grid_l1_reserve_kb() {
    static int kb = -1;
    if (kb < 0) {
        const char* e = getenv("F2M_GRID_L1_KB");
        kb = e ? atoi(e) : 64;
        if (kb < 0) kb = 0;
        if (kb > 160) kb = 160;
    }
    return kb;
}

static size_t grid_smem_bytes(int32_t V, int grid, int* cap, int* nl, int* ne) {
    const int nv = (V + grid - 1) / grid + 1;
    size_t off = (((size_t)nv + 1) * 4 + 15) / 16 * 16;
    int dev = 0, lim = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // static shared memory and alignment, and the L1 reserve
    const long long room = (long long)lim - 8192 - 1024LL * grid_l1_reserve_kb();
    int l = 1024;
    while (l < 3 * nv && l < kMaxNl) l *= 2;
    if (nv > kMaxNl) l = 0;
    long long c = l ? (long long)nv * 3 : (room - (long long)off) / 12;
    const long long halo_nodes = l ? (long long)l * 24 + 16 : 0;
    long long e = l ? (room - (long long)off - c * 12 - 16 - halo_nodes) / 12 : 0;
    if (l && e < std::max(2LL * l, (long long)kPartScratchEntries)) {  // not enough room for a useful halo
        l = 0;
        e = 0;
        c = (room - (long long)off) / 12;
    }
    if (c < 0) c = 0;
    *cap = (int)c;
    *nl = l;
    *ne = (int)e;
    off += (size_t)c * 8 + ((size_t)c * 4 + 15) / 16 * 16;
    if (l) off += (size_t)l * 16 + (size_t)l * 4 + (((size_t)l + 1) * 4 + 15) / 16 * 16 + (size_t)e * 12;
    return off;
}

// Jacobi steps per grid barrier at most (F2M_GRID_BLOCK overrides; 0 = one
// barrier per step).  Deeper blocks recompute more halo nodes per step.
static int grid_block_steps() {
    static int k = -1;
    if (k < 0) {
        const char* e = getenv("F2M_GRID_BLOCK");
        k = e ? atoi(e) : 4;
        if (k < 0) k = 0;
        if (k > kMaxBlk) k = kMaxBlk;
    }
    return k;
}

cudaError_t launch_solve_grid(const Batch& B, const DevParams& P, const GridState& G, int b, int V,
                              bool refit, cudaStream_t s, int64_t* launches) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = sms;
    int cap = 0, nl = 0, ne = 0;
    size_t smem = grid_smem_bytes(V, grid, &cap, &nl, &ne);
    cudaError_t e = cudaFuncSetAttribute(k_solve_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_grid, kGT, smem);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (per_sm > 2) per_sm = 2;
    grid = sms * per_sm;
    if (grid > kGridMaxCtas) grid = kGridMaxCtas;
    smem = grid_smem_bytes(V, grid, &cap, &nl, &ne);
    if ((e = cudaMemsetAsync(G.bar, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(G.axb_used, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(G.err, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(G.prog, 0, kGridMaxCtas * sizeof(unsigned), s)) != cudaSuccess) return e;
    Batch Bc = B;
    DevParams Pc = P;
    GridState Gc = G;
    int bb = b, rf = refit ? 1 : 0, cp = cap, l = nl, en = ne, km = grid_block_steps();
    if (km == 0) l = 0;
    void* args[] = {&Bc, &Pc, &Gc, &bb, &rf, &cp, &l, &en, &km};
    e = cudaLaunchCooperativeKernel((const void*)k_solve_grid, dim3(grid), dim3(kGT), args, smem, s);
    ++*launches;
    return e;
}

/* ------------------------------------------------------------------ */
/* ownership order: Morton order of the points                          */
/* ------------------------------------------------------------------ */
__device__ __forceinline__ unsigned spread16(unsigned v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// key = Morton code of the point on a 2^16 x 2^16 lattice over the square
// that holds the instance's cell grid, then the node id (ties, and the
// order itself when spatial == 0).  n >= the instance's node count; the
// entries past it take the largest code and sort last.
__global__ void k_own_keys(Batch B, int b, int n, const int32_t* point_of, int spatial, unsigned long long* key) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    unsigned m = 0;
    if (v >= B.Vn[b]) {
        m = 0xffffffffu;
    } else if (spatial) {
        const int p = point_of ? point_of[v] : v;
        const double2 q = B.P[B.offs[b] + p];
        const double w = B.gh[b] * (double)max(B.gnx[b], B.gny[b]);
        const double fx = fmin(fmax((q.x - B.gx0[b]) / w, 0.0), 1.0) * 65535.0;
        const double fy = fmin(fmax((q.y - B.gy0[b]) / w, 0.0), 1.0) * 65535.0;
        m = spread16((unsigned)fx) | (spread16((unsigned)fy) << 1);
    }
    key[v] = ((unsigned long long)m << 32) | (unsigned)v;
}
__global__ void k_own_take(const unsigned long long* key, int n, int32_t* own) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) own[i] = (int32_t)(unsigned)key[i];
}

size_t grid_order_temp_bytes(int64_t n) { return radix_sort_temp_bytes(n); }

cudaError_t launch_grid_order(const Batch& B, const GridState& G, int b, int V, const int32_t* point_of,
                              bool spatial, cudaStream_t s, int64_t* launches) {
    if (V <= 0) return cudaSuccess;
    const int T = 256, nb = (V + T - 1) / T;
    k_own_keys<<<nb, T, 0, s>>>(B, b, V, point_of, spatial ? 1 : 0, G.okey);
    ++*launches;
    unsigned long long* sorted = G.okey;
    if (spatial) {
        // by the code (bits 32-63); the sort is stable, so equal codes keep
        // the node order
        cudaError_t e = radix_sort(G.okey, G.okey2, nullptr, nullptr, V, 32, 64, G.otmp, G.otmp_bytes, s,
                                   launches, &sorted, nullptr);
        if (e != cudaSuccess) return e;
    }
    k_own_take<<<nb, T, 0, s>>>(sorted, V, G.own);
    ++*launches;
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* the reference's edge order of one instance                           */
/* ------------------------------------------------------------------ */
// Per slot of node v: keys (emitter << 32 | partner) and the cost's bits
// (costs are non-negative, so their bits order as the values) for a slot
// whose neighbour is the higher id, all ones (last) otherwise.
__global__ void k_edge_keys(Batch B, int b, int V, unsigned long long* k1, uint32_t* v1) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int64_t base = B.offs[b];
    const int64_t s0 = B.row[base];
    for (int64_t a = B.row[base + v]; a < B.row[base + v + 1]; ++a) {
        const bool up = B.slot[a].nbr > v;
        k1[a - s0] = up ? (((unsigned long long)(unsigned)B.s_em[a] << 32) | (unsigned)B.s_oth[a]) : ~0ull;
        v1[a - s0] = (uint32_t)(a - s0);
    }
}
__global__ void k_edge_cost_keys(Batch B, int b, int64_t S, const unsigned long long* k1, const uint32_t* v1,
                                 unsigned long long* k2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S) return;
    const int64_t s0 = B.row[B.offs[b]];
    k2[i] = k1[i] == ~0ull ? ~0ull : (unsigned long long)__double_as_longlong(B.s_cost[s0 + v1[i]]);
}

size_t edge_order_temp_bytes(int64_t S) { return radix_sort_temp_bytes(S); }

cudaError_t launch_edge_order(const Batch& B, int b, int V, int64_t S, const EdgeSort& E, const uint32_t** order,
                              cudaStream_t s, int64_t* launches) {
    if (V <= 0 || S <= 0) { *order = E.v2; return cudaSuccess; }
    const int T = 256;
    k_edge_keys<<<(V + T - 1) / T, T, 0, s>>>(B, b, V, E.k1, E.v1);
    ++*launches;
    // LSD: by (emitter, partner), then stably by cost
    unsigned long long* ks = nullptr;
    uint32_t* vs = nullptr;
    cudaError_t e = radix_sort(E.k1, E.k2, E.v1, E.v2, S, 0, 64, E.tmp, E.tmp_bytes, s, launches, &ks, &vs);
    if (e != cudaSuccess) return e;
    unsigned long long* kc = (ks == E.k1) ? E.k2 : E.k1;  // the free key buffer
    uint32_t* vfree = (vs == E.v1) ? E.v2 : E.v1;
    k_edge_cost_keys<<<(unsigned)((S + T - 1) / T), T, 0, s>>>(B, b, S, ks, vs, kc);
    ++*launches;
    e = radix_sort(kc, ks, vs, vfree, S, 0, 64, E.tmp, E.tmp_bytes, s, launches, &ks, &vs);
    if (e != cudaSuccess) return e;
    *order = vs;
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* the result arrays in the reference's edge order                      */
/* ------------------------------------------------------------------ */
EdgeExport edge_export_view(void* xout, int64_t E) {
    EdgeExport X;
    double* d = static_cast<double*>(xout);
    X.Do = d;
    X.D = d + E;
    X.x = d + 2 * E;
    int32_t* i = reinterpret_cast<int32_t*>(d + 3 * E);
    X.ev1 = i;
    X.ev2 = i + E;
    X.el1 = i + 2 * E;
    X.el2 = i + 3 * E;
    return X;
}

// Edge e of the order is the slot order[e] of its lower-id endpoint (found
// by binary search over the instance's row offsets); x follows the slot's
// primal code (graph::X, F2M.h:161), the labels the points' labels.
__global__ void k_export_edges(Batch B, int b, int V, const uint32_t* order, int64_t E, EdgeExport X) {
    const int64_t base = B.offs[b];
    const int64_t* row = B.row + base;
    const int64_t s0 = row[0];
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = s0 + order[e];
        int lo = 0, hi = V - 1;  // the last node whose list starts at or before a
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (row[mid] <= a) lo = mid; else hi = mid - 1;
        }
        const int v = lo;
        const Slot s = B.slot[a];
        const int u = s.nbr;
        const uint8_t c = B.xcode[a];
        X.ev1[e] = v;
        X.ev2[e] = u;
        const bool vlow = B.K[base + v] < B.K[base + u];
        X.el1[e] = vlow ? v : u;
        X.el2[e] = vlow ? u : v;
        X.Do[e] = B.s_cost[a];
        X.D[e] = s.D;
        X.x[e] = c == 3 ? (double)B.xval[a] : (c == 2 ? 1.0 : (c == 1 ? 0.5 : 0.0));
    }
}

cudaError_t launch_export_edges(const Batch& B, int b, int V, const uint32_t* order, int64_t E,
                                const EdgeExport& X, cudaStream_t s, int64_t* launches) {
    if (E <= 0) return cudaSuccess;
    const int T = 256;
    const int64_t blocks = std::min<int64_t>((E + T - 1) / T, 148 * 16);
    k_export_edges<<<(unsigned)blocks, T, 0, s>>>(B, b, V, order, E, X);
    ++*launches;
    return cudaGetLastError();
}

}  // namespace f2m
