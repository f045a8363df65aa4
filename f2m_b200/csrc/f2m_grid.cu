// Grid-wide solver: one large instance over every SM of the GPU.
//
// The same schedule as the per-team solver (graph_cuda.cu:163-430 and the
// comb stage, graph_cuda_comb.hpp:415-475), for instances whose potentials no
// longer fit one SM's shared memory (10^5+ nodes).  Each CTA owns a
// contiguous range of nodes; H = F/2 (double-buffered) and the comb labels
// live in global memory and are read through L2 (ld.volatile) because other
// SMs write them; a CTA's EF lists are cached in its shared memory.  A
// bounded software grid barrier separates the Jacobi steps; the launch is
// cooperative, so all CTAs are resident.  A barrier that waits too long sets
// an error flag and every CTA returns.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "f2m_device.cuh"
#include "f2m_internal.h"

namespace f2m {

constexpr int kGT = 1024;              // threads per CTA (one CTA per SM: fewer barrier arrivals)
constexpr long long kSpinLimit = 1LL << 26;  // ~seconds of waiting before giving up

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

// Potentials written by other SMs are read through L2 (ld.global.cg): the
// grid barrier orders the writes, and bypassing L1 keeps a stale line of an
// earlier iteration out (the two buffers alternate every step).
struct L2Ptr {
    const double* p;
    __device__ __forceinline__ double operator[](int64_t i) const { return __ldcg(p + i); }
};

struct GridSolver {
    const Batch& B;
    const DevParams& P;
    const GridState& G;
    const Inst& I;
    int b;
    int v0, v1;            // this CTA's nodes
    int64_t row0;          // first slot of the instance
    double* Hc;
    double* Hn;
    double* eD;            // shared-memory EF cache of this CTA
    uint32_t* eW;
    int cap;
    int* sefo;             // shared: local offset of each own node's EF list (v1-v0+1)
    double* sred;
    long long* sredl;
    int* swarp;
    unsigned long long* sbcv;  // shared broadcast slot of the grid reductions
    int* sflag;                // shared: barrier error flag of this CTA
    int phase = 0;
    long long iters = 0, wslots = 0;
    int checks = 0;
    bool capped = false;
    bool dead = false;     // a barrier timed out

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
                        if (spins > kSpinLimit) { atomicExch(G.err, 1); bad = 1; break; }
                    }
                }
            }
            *sflag = bad;
        }
        __syncthreads();
        dead = *sflag != 0;
        return !dead;
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

    // grad/2 of an own node over its EF list (the first efcnt slots of its
    // list, held in shared memory or in the slot-indexed arena).  The
    // neighbours' potentials come from L2; they are loaded four at a time
    // ahead of the compare chain, so one L2 latency covers four entries.
    __device__ double hgrad(int v) const {
        const int n = G.efc[v];
        const int lo = sefo[v - v0];
        const bool sm = lo + n <= cap;
        const int64_t go = I.row[v] - row0;
        const double* Dp = sm ? eD + lo : G.gD + go;
        const uint32_t* Wp = sm ? eW + lo : G.gW + go;
        const L2Ptr H = hc();
        const double hv = H[v];
        constexpr int CH = 4;
        double x0 = 0.0, x1 = 1e6, x2 = 1e6;
        bool chain = false;
        for (int k0 = 0; k0 < n; k0 += CH) {
            double hw[CH], dd[CH];
            uint32_t ww[CH];
#pragma unroll
            for (int j = 0; j < CH; ++j) {
                ww[j] = 0u;
                hw[j] = 0.0;
                dd[j] = 0.0;
                if (k0 + j < n) {
                    ww[j] = Wp[k0 + j];
                    dd[j] = Dp[k0 + j];
                    hw[j] = H[ww[j] & 0x7fffffffu];
                }
            }
#pragma unroll
            for (int j = 0; j < CH; ++j) {
                if (k0 + j >= n) break;
                const bool first = (ww[j] >> 31) != 0;
                const double x = (dd[j] + (first ? hw[j] : hv)) + (first ? hv : hw[j]);
                if (k0 + j == 0) {  // cuda_get_Nodes_grad_R: chain unless the first is below 1e6
                    x0 = x;
                    chain = !(x0 < 1e6);
                } else if (!chain) {
                    top3_insert(x, x0, x1, x2);
                } else {
                    if (x < x0) { x2 = x1; x1 = x0; x0 = x; continue; }
                    if (x < x1) { x2 = x1; x1 = x; continue; }
                    if (x < x2) { x2 = x; }
                }
            }
        }
        return (-(x1 + x2) / 2) * 0.5;
    }
    __device__ void swap_h() { double* t = Hc; Hc = Hn; Hn = t; }
    template <bool MASKED>
    __device__ void step() {
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            const double g = hgrad(v);
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
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) m = fmax(m, fabs(hgrad(v)));
        return 2.0 * gmax(m);
    }
    // update_EF for this CTA's nodes: local offsets, shared cache, arena copy
    __device__ void rebuild_ef() {
        __syncthreads();
        int carry = 0;
        for (int r = v0; r < v1; r += kGT) {
            const int v = r + threadIdx.x;
            const int c = (v < v1) ? G.efc[v] : 0;
            int tot;
            const int ex = block_excl_scan<kGT>(c, swarp, &tot);
            if (v < v1) sefo[v - v0] = carry + ex;
            carry += tot;
        }
        if (threadIdx.x == 0) sefo[v1 - v0] = carry;
        __syncthreads();
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            const int64_t r0 = I.row[v];
            const int n = G.efc[v], lo = sefo[v - v0];
            const int64_t go = r0 - row0;
            const bool sm = lo + n <= cap;
            for (int k = 0; k < n; ++k) {
                const Slot s = I.slot[r0 + I.perm[r0 + k]];
                const uint32_t w = (uint32_t)s.nbr | (s.nbr < v ? 0x80000000u : 0u);
                G.gD[go + k] = s.D;
                G.gW[go + k] = w;
                if (sm) { eD[lo + k] = s.D; eW[lo + k] = w; }
            }
        }
        __syncthreads();
    }
    __device__ double check_opt() {
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            const int d = deg(v);
            G.efc[v] = (d < P.ef_small_deg) ? d : qpart_ef(I, I.row[v], v, hc(), d, P.ef_thr, P.ef_min);
        }
        rebuild_ef();
        checks++;
        return grad_max();
    }
    __device__ void block_ef(int N) {
        const double MA = grad_max();
        int count_M = 0;
        for (int it = 0; it < N && !dead; ++it) {
            step<false>();
            if (++count_M >= P.check_every) {
                if (MA < P.error_B) break;
                count_M = 0;
            }
        }
    }
    __device__ void block_glob() {
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) G.efc[v] = min(deg(v), P.glob_K);
        rebuild_ef();
        for (int go = 0; go < P.glob_rounds && !dead; ++go) {
            for (int it = 0; it < P.glob_inner && !dead; ++it) step<false>();
            for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
                const int d = deg(v);
                if (d < P.glob_K) { G.efc[v] = d; continue; }
                const int64_t r0 = I.row[v];
                const double hv = hc()[v];
                double avg = pdv(I, r0, I.perm + r0, 0, v, hc(), hv);
                for (int k = 1; k < P.glob_K; ++k) avg = fmax(avg, pdv(I, r0, I.perm + r0, k, v, hc(), hv));
                G.efc[v] = qpart_ef(I, r0, v, hc(), d, avg, P.ef_min);
            }
            rebuild_ef();
            if (grad_max() < P.glob_tol) break;
        }
    }
    __device__ double run_start() {
        block_glob();
        double M = check_opt();
        int factor = P.factor0;
        for (int go = 1; go <= P.max_rounds && !dead; ++go) {
            block_ef(factor);
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
            block_ef(P.fix_factor);
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
        for (int v = v0 + threadIdx.x; v < v1; v += kGT)  // cuda_partition_v3
            ccnt[v] = qpart_b(I, I.row[v], v, hc(), G.efc[v], P.comb_thr);
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            const int64_t r0 = I.row[v];
            const double hv = hc()[v];
            bool has = false;
            for (int k = 0; k < ccnt[v] && !has; ++k) {
                const double d = pdv(I, r0, I.perm + r0, k, v, hc(), hv);
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
            for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
                int m = vlab[v];
                if (m == INT_MAX) continue;
                const int64_t r0 = I.row[v];
                const double hv = hc()[v];
                for (int k = 0; k < ccnt[v]; ++k) {
                    const Slot s = I.slot[r0 + I.perm[r0 + k]];
                    const double d = red_d(s, v, hc(), hv);
                    if (d >= -porog && d <= porog) m = min(m, vlab[s.nbr]);
                }
                if (m < vlab[v]) { vlab[v] = m; changed = 1; }
            }
            if (gsum_ll(changed) == 0) break;
        }
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            B.F[I.base + v] = 2.0 * hc()[v];
            B.efcnt[I.base + v] = G.efc[v];
            B.ccnt[I.base + v] = ccnt[v];
        }
        volatile int* virr = G.irr;
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
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
        for (int v = v0 + threadIdx.x; v < v1; v += kGT)
            if (vlab[v] == v) { nc++; ni += virr[v]; }
        nc = gsum_ll(nc);
        ni = gsum_ll(ni);
        double lp = 0.0, dual_neg = 0.0, fsum = 0.0;
        long long maxr = -1, viol = 0;
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            const int64_t r0 = I.row[v], r1 = I.row[v + 1];
            const double hv = hc()[v];
            fsum += 2.0 * hv;
            float degsum = 0.0f;
            bool any = false;
            for (int64_t a = r0; a < r1; ++a) {
                const Slot s = I.slot[a];
                const double d = red_d(s, v, hc(), hv);
                const double x = (d < porog) ? ((d > -porog) ? 0.5 : 1.0) : 0.0;
                B.xcode[a] = (uint8_t)(x == 1.0 ? 2 : (x == 0.5 ? 1 : 0));
                degsum += (float)x;
                any |= (x != 0.0);
                if (s.nbr > v) {
                    lp += x * B.s_cost[a];
                    dual_neg += fmin(0.0, d);
                    if (x != 0.0) maxr = ::max(maxr, (long long)::min((int)(a - r0), B.mirror[a]));
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
            else if (ni > 0) { B.status[b] = kNeedsHost; B.lp[b] = NAN; }
            else { B.status[b] = F2M_OK; B.lp[b] = lp; }
        }
    }
};

__global__ void __launch_bounds__(kGT, 1) k_solve_grid(Batch B, DevParams P, GridState G, int b, int refit,
                                                     int cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sred[kGT / 32];
    __shared__ long long sredl[kGT / 32];
    __shared__ int swarp[kGT / 32 + 1];
    __shared__ unsigned long long sbc[1];
    __shared__ int sflag[1];
    const Inst I = make_inst(B, b);
    const int V = I.V;
    const int v0 = (int)(((long long)V * blockIdx.x) / gridDim.x);
    const int v1 = (int)(((long long)V * (blockIdx.x + 1)) / gridDim.x);
    const int nv = v1 - v0;
    int* sefo = reinterpret_cast<int*>(smem_raw);
    const size_t head = (((size_t)nv + 1) * 4 + 15) / 16 * 16;
    double* eD = reinterpret_cast<double*>(smem_raw + head);
    uint32_t* eW = reinterpret_cast<uint32_t*>(eD + cap);
    GridSolver S{B, P, G, I, b, v0, v1, I.row[0], G.Ha, G.Hb, eD, eW, cap, sefo, sred, sredl, swarp, sbc, sflag};
    double M;
    if (!refit) {
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) G.Ha[v] = B.F0 ? 0.5 * B.F0[I.base + v] : 0.0;  // F = 0 or warm
        S.sync();
        M = B.F0 ? S.run_fix() : S.run_start();  // a resumed descent skips the global phase
    } else {
        // cuda_IRREGULAR_B_recompute (graph_cuda_comb.hpp:542-574)
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            G.Ha[v] = 0.5 * (B.F[I.base + v] + B.shift[I.base + v]);
            G.efc[v] = B.efcnt[I.base + v];
        }
        // the EF lists of the last update_EF are in the slot-indexed arena
        __syncthreads();
        int carry = 0;
        for (int r = v0; r < v1; r += kGT) {
            const int v = r + threadIdx.x;
            const int c = (v < v1) ? G.efc[v] : 0;
            int tot;
            const int ex = block_excl_scan<kGT>(c, swarp, &tot);
            if (v < v1) sefo[v - v0] = carry + ex;
            carry += tot;
        }
        if (threadIdx.x == 0) sefo[nv] = carry;
        __syncthreads();
        for (int v = v0 + threadIdx.x; v < v1; v += kGT) {
            const int n = G.efc[v], lo = sefo[v - v0];
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

static size_t grid_smem_bytes(int32_t V, int grid, int* cap) {
    const int nv = (V + grid - 1) / grid + 1;
    const size_t head = (((size_t)nv + 1) * 4 + 15) / 16 * 16;
    // EF lists of a CTA's nodes: about 4 per node in the active phase, 5 in
    // the first phase; lists beyond the cache are read from the arena
    int dev = 0, lim = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const long long room = ((long long)lim - 4096 - (long long)head) / 12;
    long long c = (long long)nv * 8;
    if (c > room) c = room > 0 ? room : 0;
    *cap = (int)c;
    return head + (size_t)c * 12;
}

cudaError_t launch_solve_grid(const Batch& B, const DevParams& P, const GridState& G, int b, int V,
                              bool refit, cudaStream_t s, int64_t* launches) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = sms;
    int cap = 0;
    size_t smem = grid_smem_bytes(V, grid, &cap);
    cudaError_t e = cudaFuncSetAttribute(k_solve_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_grid, kGT, smem);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (per_sm > 2) per_sm = 2;
    grid = sms * per_sm;
    if (grid > kGridMaxCtas) grid = kGridMaxCtas;
    smem = grid_smem_bytes(V, grid, &cap);
    if ((e = cudaMemsetAsync(G.bar, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(G.err, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
    Batch Bc = B;
    DevParams Pc = P;
    GridState Gc = G;
    int bb = b, rf = refit ? 1 : 0, cp = cap;
    void* args[] = {&Bc, &Pc, &Gc, &bb, &rf, &cp};
    e = cudaLaunchCooperativeKernel((const void*)k_solve_grid, dim3(grid), dim3(kGT), args, smem, s);
    ++*launches;
    return e;
}


}  // namespace f2m
