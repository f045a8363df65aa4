// Entropically smoothed F2M dual bound and its adjoint, for batches of
// instances (no counterpart in the reference, which solves the LP only).
//
// Graph: the union over points of each point's N nearest neighbours by FP32
// Euclidean distance c = sqrt(dx*dx + dy*dy) (round-to-nearest, no FMA), ties
// by index; node lists ascending in neighbour index.
//
// Bound: with z_e = (u_a + u_b - c_e)/tau and sigma the logistic function,
//   L(u) = 2 sum_v u_v - tau sum_e softplus(z_e),
// the dual of the entropy-smoothed fractional 2-matching LP, so L(u) bounds
// that LP from below for every u.  Forward: T damped Jacobi coordinate-ascent
// steps from u = 0 (s_v = root of sum_{e=(v,w)} sigma((s + u_w - c_e)/tau) = 2,
// u_v <- (1 - omega) u_v + omega s_v), then L(u^T).  Backward: the exact
// adjoint of those steps (implicit function theorem at each root), with the
// iterates recomputed from checkpoints every K steps instead of stored, then
// chained through c_e = |p_a - p_b| to the coordinates.  All dual arithmetic
// is FP64; coordinates and costs are FP32.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "f2m_device.cuh"
#include "f2m_internal.h"

namespace f2m {

constexpr int kST = 512;  // threads of a solver CTA (one instance at a time)

__device__ __forceinline__ float sdist(float x0, float y0, float x1, float y1) {
    const float dx = __fsub_rn(x0, x1), dy = __fsub_rn(y0, y1);
    return __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
}

__device__ __forceinline__ int find_inst(const int64_t* offs, int n_inst, int64_t g) {
    int lo = 0, hi = n_inst - 1;  // last b with offs[b] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* ---------------- kNN: warp per point, brute force over its instance ---- */
// Each warp keeps the point's best N keys (cost bits << 32 | local index; the
// cost is non-negative, so the unsigned order is (cost, index)) as a sorted
// list spread over two registers per lane (elements l and 32 + l).
__global__ void __launch_bounds__(256) k_sknn(SmoothBatch S) {
    const int lane = threadIdx.x & 31;
    const int64_t g = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (g >= S.n_total) return;
    const int b = find_inst(S.offs, S.n_inst, g);
    const int64_t base = S.offs[b];
    const int V = (int)(S.offs[b + 1] - base);
    const int N = min(S.N, V - 1);
    const int i = (int)(g - base);
    const float xi = S.x[g], yi = S.y[g];
    unsigned long long A = ~0ull, Bk = ~0ull;
    unsigned long long thr = ~0ull;  // element N-1
    for (int j0 = 0; j0 < V; j0 += 32) {
        const int j = j0 + lane;
        unsigned long long key = ~0ull;
        if (j < V && j != i) {
            const float c = sdist(xi, yi, S.x[base + j], S.y[base + j]);
            key = ((unsigned long long)__float_as_uint(c) << 32) | (unsigned)j;
        }
        unsigned m = __ballot_sync(0xffffffffu, key < thr);
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const unsigned long long k = __shfl_sync(0xffffffffu, key, src);
            if (k >= thr) continue;
            const int pos = __popc(__ballot_sync(0xffffffffu, A < k)) +
                            __popc(__ballot_sync(0xffffffffu, Bk < k));
            const unsigned long long pa = __shfl_up_sync(0xffffffffu, A, 1);
            const unsigned long long pb = __shfl_up_sync(0xffffffffu, Bk, 1);
            const unsigned long long a31 = __shfl_sync(0xffffffffu, A, 31);
            const unsigned long long nA = lane < pos ? A : (lane == pos ? k : pa);
            const int hb = 32 + lane;
            const unsigned long long nB = hb < pos ? Bk : (hb == pos ? k : (lane == 0 ? a31 : pb));
            A = nA;
            Bk = nB;
            thr = (N - 1 < 32) ? __shfl_sync(0xffffffffu, A, N - 1) : __shfl_sync(0xffffffffu, Bk, N - 33);
        }
    }
    unsigned long long* out = S.top + g * S.N;
    if (lane < S.N) out[lane] = lane < N ? A : ~0ull;
    if (32 + lane < S.N) out[32 + lane] = 32 + lane < N ? Bk : ~0ull;
}

// reverse counts: rdeg[w] = number of points that keep w
__global__ void k_srdeg(SmoothBatch S) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= S.n_total * S.N) return;
    const unsigned long long k = S.top[t];
    if (k == ~0ull) return;
    const int64_t g = t / S.N;
    const int b = find_inst(S.offs, S.n_inst, g);
    atomicAdd(&S.rdeg[S.offs[b] + (unsigned)(k & 0xffffffffu)], 1);
}

__global__ void k_stcap(SmoothBatch S) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.n_total) return;
    S.deg[g] = S.N + S.rdeg[g];
    S.tcur[g] = 0;
}

__global__ void k_sfill(SmoothBatch S) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= S.n_total * S.N) return;
    const int64_t g = t / S.N;
    const int k = (int)(t % S.N);
    const unsigned long long key = S.top[t];
    int32_t w = -1;
    if (key != ~0ull) w = (int32_t)(key & 0xffffffffu);
    S.tnbr[S.tcap[g] + k] = w;  // own list (-1 = none)
    if (w < 0) return;
    const int b = find_inst(S.offs, S.n_inst, g);
    const int64_t gw = S.offs[b] + w;
    const int p = atomicAdd(&S.tcur[gw], 1);
    S.tnbr[S.tcap[gw] + S.N + p] = (int32_t)(g - S.offs[b]);
}

// sort each temporary list by neighbour, drop repeats and the -1 fillers
__global__ void k_ssort(SmoothBatch S) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.n_total) return;
    int32_t* a = S.tnbr + S.tcap[g];
    const int n = S.N + S.rdeg[g];
    for (int i = 1; i < n; ++i) {
        const int32_t v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
        a[j + 1] = v;
    }
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (a[i] >= 0 && (m == 0 || a[m - 1] != a[i])) a[m++] = a[i];
    S.deg[g] = m;
}

__global__ void k_scopy(SmoothBatch S) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.n_total) return;
    const int b = find_inst(S.offs, S.n_inst, g);
    const int64_t base = S.offs[b];
    const int32_t* a = S.tnbr + S.tcap[g];
    const int64_t r0 = S.row[g];
    const int n = (int)(S.row[g + 1] - r0);
    for (int k = 0; k < n; ++k) {
        const int32_t w = a[k];
        S.nbr[r0 + k] = w;
        S.c[r0 + k] = sdist(S.x[g], S.y[g], S.x[base + w], S.y[base + w]);
    }
}

__global__ void k_smirror(SmoothBatch S) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= S.n_total) return;
    const int b = find_inst(S.offs, S.n_inst, g);
    const int64_t base = S.offs[b];
    const int32_t v = (int32_t)(g - base);
    for (int64_t k = S.row[g]; k < S.row[g + 1]; ++k) {
        const int64_t gw = base + S.nbr[k];
        int64_t lo = S.row[gw], hi = S.row[gw + 1] - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (S.nbr[mid] < v) lo = mid + 1; else hi = mid;
        }
        S.mirror[k] = lo;
    }
}

/* ---------------- the bound and its adjoint: one CTA per instance ------- */
__device__ __forceinline__ double sigm(double z) {
    if (z >= 0) return 1.0 / (1.0 + exp(-z));
    const double e = exp(z);
    return e / (1.0 + e);
}
__device__ __forceinline__ double softplus(double z) { return fmax(z, 0.0) + log1p(exp(-fabs(z))); }

// Root s of sum_k sigma((s + u[nbr_k] - c_k)/tau) = 2 by Newton's method kept
// inside a bracket (bisection when a step leaves it).  The bracket is the
// smallest a_k - 40 tau (every term below 5e-18) and the third smallest
// a_k + 40 tau (three terms above 1 - 5e-18), a_k = c_k - u[nbr_k].
__device__ double node_root(const int32_t* nb, const float* c, int n, const double* u, double tau,
                            double s0, int max_it) {
    double m0 = INFINITY, m1 = INFINITY, m2 = INFINITY;
    for (int k = 0; k < n; ++k) {
        const double a = (double)c[k] - u[nb[k]];
        if (a < m0) { m2 = m1; m1 = m0; m0 = a; }
        else if (a < m1) { m2 = m1; m1 = a; }
        else if (a < m2) { m2 = a; }
    }
    double lo = m0 - 40 * tau, hi = m2 + 40 * tau;
    double s = fmin(fmax(s0, lo), hi);
    for (int it = 0; it < max_it; ++it) {
        double g = -2.0, gp = 0.0;
        for (int k = 0; k < n; ++k) {
            const double sg = sigm((s - ((double)c[k] - u[nb[k]])) / tau);
            g += sg;
            gp += sg * (1.0 - sg);
        }
        gp /= tau;
        if (g > 0) hi = s; else lo = s;
        if (fabs(g) <= 1e-13 || hi - lo <= 1e-15 * (1.0 + fabs(s))) break;
        double sn = (gp > 0) ? s - g / gp : 0.5 * (lo + hi);
        if (!(sn > lo && sn < hi)) sn = 0.5 * (lo + hi);
        if (sn == s) break;
        s = sn;
    }
    return s;
}

struct SInst {
    int V;
    int64_t base;
    const int64_t* row;  // row + base
    int64_t r0;
};

// One damped Jacobi step u -> un; writes the roots to s_out when given.
__device__ __forceinline__ void sjacobi(const SmoothBatch& S, const SInst& I, const double* u,
                                        double* un, double* s_out) {
    for (int v = threadIdx.x; v < I.V; v += kST) {
        const int64_t a = I.row[v], e = I.row[v + 1];
        const double s = node_root(S.nbr + a, S.c + a, (int)(e - a), u, S.tau, u[v], S.newton_max);
        if (s_out) s_out[v] = s;
        un[v] = (1.0 - S.omega) * u[v] + S.omega * s;
    }
}

__device__ double sbound(const SmoothBatch& S, const SInst& I, const double* u, double* sred) {
    double su = 0.0, sp = 0.0;
    for (int v = threadIdx.x; v < I.V; v += kST) {
        su += 2.0 * u[v];
        for (int64_t k = I.row[v]; k < I.row[v + 1]; ++k) {
            const int w = S.nbr[k];
            if (w > v) sp += softplus((u[v] + u[w] - (double)S.c[k]) / S.tau);
        }
    }
    su = block_sum<kST>(su, sred);
    sp = block_sum<kST>(sp, sred);
    return su - S.tau * sp;
}

template <bool GRAD>
__global__ void __launch_bounds__(kST) k_sbound(SmoothBatch S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sred[kST / 32];
    __shared__ int sitem;
    double* Ha = reinterpret_cast<double*>(smem_raw);
    for (;;) {
        if (threadIdx.x == 0) sitem = atomicAdd(S.queue, 1);
        __syncthreads();
        const int b = sitem;
        __syncthreads();
        if (b >= S.n_inst) return;
        SInst I;
        I.base = S.offs[b];
        I.V = (int)(S.offs[b + 1] - I.base);
        I.row = S.row + I.base;
        I.r0 = I.row[0];
        double* Hb = Ha + I.V;
        const int T = S.iters, K = S.ckpt;
        double* ck = S.ck + I.base * S.n_ck;
        for (int v = threadIdx.x; v < I.V; v += kST) Ha[v] = 0.0;
        __syncthreads();
        double* u = Ha;
        double* un = Hb;
        for (int t = 0; t < T; ++t) {
            if (GRAD && t % K == 0)
                for (int v = threadIdx.x; v < I.V; v += kST) ck[(t / K) * I.V + v] = u[v];
            sjacobi(S, I, u, un, nullptr);
            __syncthreads();
            double* tt = u; u = un; un = tt;
        }
        const double L = sbound(S, I, u, sred);
        if (threadIdx.x == 0) S.L[b] = L;
        if (!GRAD) { __syncthreads(); continue; }
        // adjoint of L(u^T) with respect to u^T and (explicitly) c; the
        // explicit sigma_e is split evenly over the edge's two slots
        const double up = S.dL[b];
        double* lam = S.lam + I.base;
        double* lam2 = S.lam2 + I.base;
        for (int v = threadIdx.x; v < I.V; v += kST) {
            double d = 2.0;
            for (int64_t k = I.row[v]; k < I.row[v + 1]; ++k) {
                const double sg = sigm((u[v] + u[S.nbr[k]] - (double)S.c[k]) / S.tau);
                d -= sg;
                S.gc[k] = up * (0.5 * sg);
            }
            lam[v] = up * d;
        }
        __syncthreads();
        double* su_ = S.segu + I.base * K;
        double* ss_ = S.segs + I.base * K;
        const int nseg = (T + K - 1) / K;
        for (int seg = nseg - 1; seg >= 0; --seg) {
            const int t0 = seg * K, t1 = min(T, t0 + K);
            for (int v = threadIdx.x; v < I.V; v += kST) Ha[v] = ck[seg * I.V + v];
            __syncthreads();
            u = Ha;
            un = Hb;
            for (int t = t0; t < t1; ++t) {  // recompute the segment's iterates
                double* ut = su_ + (t - t0) * I.V;
                for (int v = threadIdx.x; v < I.V; v += kST) ut[v] = u[v];
                sjacobi(S, I, u, un, ss_ + (t - t0) * I.V);
                __syncthreads();
                double* tt = u; u = un; un = tt;
            }
            for (int t = t1 - 1; t >= t0; --t) {
                const double* ut = su_ + (t - t0) * I.V;
                const double* st = ss_ + (t - t0) * I.V;
                // pass 1: mu_v = omega lam_v / D_v; q = mu_v p_e on v's slots
                for (int v = threadIdx.x; v < I.V; v += kST) {
                    const int64_t a = I.row[v], e = I.row[v + 1];
                    double D = 0.0;
                    for (int64_t k = a; k < e; ++k) {
                        const double sg = sigm((st[v] + ut[S.nbr[k]] - (double)S.c[k]) / S.tau);
                        const double p = sg * (1.0 - sg) / S.tau;
                        S.q[k] = p;
                        D += p;
                    }
                    const double mu = D > 0 ? S.omega * lam[v] / D : 0.0;  // D == 0: all saturated
                    for (int64_t k = a; k < e; ++k) {
                        const double qk = mu * S.q[k];
                        S.q[k] = qk;
                        S.gc[k] += qk;
                    }
                }
                __syncthreads();
                // pass 2: lam_w <- (1 - omega) lam_w - sum over w's edges of the
                // neighbour's q on the same edge
                for (int w = threadIdx.x; w < I.V; w += kST) {
                    double l = (1.0 - S.omega) * lam[w];
                    for (int64_t k = I.row[w]; k < I.row[w + 1]; ++k) l -= S.q[S.mirror[k]];
                    lam2[w] = l;
                }
                __syncthreads();
                double* tt = lam; lam = lam2; lam2 = tt;
            }
        }
        // dL/dc_e = both slots' sums; chain through c_e = |p_v - p_w|
        for (int v = threadIdx.x; v < I.V; v += kST) {
            const int64_t gv = I.base + v;
            const double xv = S.x[gv], yv = S.y[gv];
            double gx = 0.0, gy = 0.0;
            for (int64_t k = I.row[v]; k < I.row[v + 1]; ++k) {
                const double ce = (double)S.c[k];
                if (ce == 0.0) continue;
                const int64_t gw = I.base + S.nbr[k];
                const double dc = S.gc[k] + S.gc[S.mirror[k]];
                gx += dc * (xv - (double)S.x[gw]) / ce;
                gy += dc * (yv - (double)S.y[gw]) / ce;
            }
            S.gx[gv] = (float)gx;
            S.gy[gv] = (float)gy;
        }
        __syncthreads();
    }
}

/* ---------------- host launchers ---------------------------------------- */
static unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t launch_smooth_graph(SmoothBatch& S, int64_t* scan_scratch, cudaStream_t s,
                                int64_t* launches) {
    cudaError_t e;
    const int64_t nN = S.n_total * S.N;
    if ((e = cudaMemsetAsync(S.rdeg, 0, sizeof(int32_t) * S.n_total, s)) != cudaSuccess) return e;
    k_sknn<<<nblk(S.n_total, 8), 256, 0, s>>>(S);
    k_srdeg<<<nblk(nN, 256), 256, 0, s>>>(S);
    k_stcap<<<nblk(S.n_total, 256), 256, 0, s>>>(S);
    *launches += 3;
    if ((e = launch_scan(S.deg, S.tcap, S.n_total, scan_scratch, s, launches)) != cudaSuccess) return e;
    k_sfill<<<nblk(nN, 256), 256, 0, s>>>(S);
    k_ssort<<<nblk(S.n_total, 128), 128, 0, s>>>(S);
    *launches += 2;
    if ((e = launch_scan(S.deg, S.row, S.n_total, scan_scratch, s, launches)) != cudaSuccess) return e;
    k_scopy<<<nblk(S.n_total, 128), 128, 0, s>>>(S);
    k_smirror<<<nblk(S.n_total, 128), 128, 0, s>>>(S);
    *launches += 2;
    return cudaGetLastError();
}

int32_t smooth_max_nodes() {
    int dev = 0, lim = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return (lim - 1024) / 16;
}

cudaError_t launch_smooth_bound(SmoothBatch& S, int32_t max_v, bool grad, cudaStream_t s,
                                int64_t* launches) {
    const size_t dyn = (size_t)max_v * 16;
    const void* fn = grad ? (const void*)k_sbound<true> : (const void*)k_sbound<false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kST, dyn);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid = sms * per_sm;
    if (grid > S.n_inst) grid = S.n_inst;
    if ((e = cudaMemsetAsync(S.queue, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
    if (grad) k_sbound<true><<<grid, kST, dyn, s>>>(S);
    else k_sbound<false><<<grid, kST, dyn, s>>>(S);
    ++*launches;
    return cudaGetLastError();
}

}  // namespace f2m
