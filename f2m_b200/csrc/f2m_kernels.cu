// f2m_b200 CUDA kernels for sm_100a.
//
// Pipeline of one batched call (one CTA = one instance unless noted):
//   k_prep      1e-3 rounding, de-duplication, compaction, bbox   (FXY.hpp:231-309)
//   k_grid_*    per-instance cell grid (counting sort of the points)
//   k_cutoff    per-node ring cut-off radius (stat pass)          (FXY.hpp:441-534)
//   k_select    per-node first-N neighbours by (d, emitter, partner)
//                                                    (FXY.hpp:347-437 + graph_tour.hpp:28-90)
//   k_graph_*   union-of-kNN CSR in edge order, mirror slots, D = Do/d_min
//                                     (graph_tour.hpp:28-98, graph_cuda_init.hpp:3-96)
//   k_solve     persistent CTA per instance: the whole descent schedule
//               (graph_cuda.cu:163-430), partitions (graph_cuda_partition.hpp),
//               comb extraction (graph_cuda_comb.hpp:201-475), the comb check
//               (comb_thread.cpp:180-195) and the primal value
//               (graph_cuda.cu:135-147, graph_tour.hpp:165-184).
//
// All solver arithmetic is FP64 and evaluates exactly the reference's
// expressions, so a node's potential F follows the reference's trajectory
// bit for bit (given the same node ids).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>

#include "f2m_device.cuh"
#include "f2m_internal.h"

namespace f2m {

constexpr int kT = 256;       // width of the node-parallel kernels
constexpr int kTile = 1024;   // points per shared-memory tile (16 KB)
constexpr int kMaxPasses = 64;

__device__ __forceinline__ double round3(double x) {
    double r = round(x * 1000.0);  // std::round: half away from zero, as FXY.hpp:252
    return r / 1000.0;
}

/* ------------------------------------------------------------------ */
/* k_prep: rounding, de-duplication, compaction, bbox (FXY.hpp:231-309)  */
/* ------------------------------------------------------------------ */
__global__ void __launch_bounds__(kT) k_prep(Batch B) {
    const int b = blockIdx.x;
    const int64_t base = B.offs[b];
    const int n = (int)(B.offs[b + 1] - base);
    __shared__ double2 tile[kTile];
    __shared__ int swarp[kT / 32 + 1];
    __shared__ int s_carry;
    __shared__ double sred[kT / 32];

    for (int i = threadIdx.x; i < n; i += kT) {
        B.Pr[base + i] = make_double2(round3(B.X_in[base + i]), round3(B.Y_in[base + i]));
        B.dup_of[base + i] = -1;
    }
    __syncthreads();
    // a point is dropped if an earlier point has identical rounded
    // coordinates; it maps to the first such point (FXY.hpp:260-265)
    for (int t0 = 0; t0 < n && !B.skip_dedup; t0 += kTile) {
        const int cnt = min(kTile, n - t0);
        for (int k = threadIdx.x; k < cnt; k += kT) tile[k] = B.Pr[base + t0 + k];
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kT) {
            if (i <= t0 || B.dup_of[base + i] >= 0) continue;
            const double2 p = B.Pr[base + i];
            const int jmax = min(cnt, i - t0);
            for (int k = 0; k < jmax; ++k)
                if (tile[k].x == p.x && tile[k].y == p.y) { B.dup_of[base + i] = t0 + k; break; }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int r = 0; r < n; r += kT) {
        const int i = r + threadIdx.x;
        const int keep = (i < n && B.dup_of[base + i] < 0) ? 1 : 0;
        int tot;
        const int ex = block_excl_scan<kT>(keep, swarp, &tot);
        if (keep) {
            const int id = s_carry + ex;
            B.P[base + id] = B.Pr[base + i];
            B.K[base + id] = B.K_in ? B.K_in[base + i] : i + 1;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += tot;
        __syncthreads();
    }
    const int V = s_carry;
    double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
    for (int i = threadIdx.x; i < V; i += kT) {
        const double2 p = B.P[base + i];
        mnx = fmin(mnx, p.x); mxx = fmax(mxx, p.x);
        mny = fmin(mny, p.y); mxy = fmax(mxy, p.y);
    }
    mnx = block_min<kT>(mnx, sred);
    mxx = block_max<kT>(mxx, sred);
    mny = block_min<kT>(mny, sred);
    mxy = block_max<kT>(mxy, sred);
    if (threadIdx.x == 0) {
        // FXY.hpp:305-306 with the area widened to 64 bits; a zero x-span
        // falls back to the y-span (the reference never terminates there)
        const double sx = mxx - mnx, sy = mxy - mny;
        int st = F2M_OK;
        double spn = 0.0;
        if (V < 4 || !(sx * sx < 9.0e18) || !(sy * sy < 9.0e18)) {
            st = F2M_ERR_INPUT;
        } else {
            long long area = (long long)(sx * sx);
            if (area == 0) area = (long long)(sy * sy);
            if (area == 0) st = F2M_ERR_INPUT;
            else spn = sqrt((double)area / (double)V);
        }
        // cell grid: cells of the ring unit 2*size_per_node, enlarged until
        // there are at most n cells (they are indexed inside the instance's
        // point range)
        double h = 2.0 * spn;
        if (!(h > 0.0)) h = fmax(fmax(sx, sy), 1.0);
        long long gx = 1, gy = 1;
        for (int t = 0; t < 64; ++t) {
            gx = (long long)(sx / h) + 1;
            gy = (long long)(sy / h) + 1;
            if (gx * gy <= (long long)max(n, 1)) break;
            h *= 1.5;
        }
        B.gx0[b] = mnx;
        B.gy0[b] = mny;
        B.gh[b] = h;
        B.gnx[b] = (int)gx;
        B.gny[b] = (int)gy;
        B.Vn[b] = V;
        B.spn[b] = spn;
        B.status[b] = st;
        B.dmin_bits[b] = 0x7ff0000000000000ull;  // +inf
    }
}

/* ------------------------------------------------------------------ */
/* cell grid of each instance (a counting sort of the points by cell)    */
/* ------------------------------------------------------------------ */
__device__ __forceinline__ int cell_coord(double v, double v0, double h, int n) {
    double c = floor((v - v0) / h);
    c = fmin(fmax(c, 0.0), (double)(n - 1));
    return (int)c;
}

__global__ void __launch_bounds__(kT) k_grid_count(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int i = B.chunk_start[c] + threadIdx.x;
    if (i >= B.Vn[b]) return;
    const int64_t base = B.offs[b];
    const double2 p = B.P[base + i];
    const int nx = B.gnx[b], ny = B.gny[b];
    const int cell = cell_coord(p.y, B.gy0[b], B.gh[b], ny) * nx + cell_coord(p.x, B.gx0[b], B.gh[b], nx);
    B.pcell[base + i] = cell;
    atomicAdd(reinterpret_cast<unsigned long long*>(&B.cellcnt[base + cell]), 1ull);
}

__global__ void __launch_bounds__(kT) k_grid_scatter(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int i = B.chunk_start[c] + threadIdx.x;
    if (i >= B.Vn[b]) return;
    const int64_t base = B.offs[b];
    const int cell = B.pcell[base + i];
    const int pos = atomicAdd(&B.cellcur[base + cell], 1);
    const int64_t k = B.cellstart[base + cell] + pos;
    B.sidx[k] = i;
    B.spt[k] = B.P[base + i];
}

// Cell rows of the box [x-R, x+R] x [y-R, y+R], one cell of margin.
struct Box {
    int cx0, cx1, cy0, cy1;
};
__device__ __forceinline__ Box box_of(const Batch& B, int b, double x, double y, double R) {
    const double h = B.gh[b];
    const int nx = B.gnx[b], ny = B.gny[b];
    Box r;
    r.cx0 = max(cell_coord(x - R, B.gx0[b], h, nx) - 1, 0);
    r.cx1 = min(cell_coord(x + R, B.gx0[b], h, nx) + 1, nx - 1);
    r.cy0 = max(cell_coord(y - R, B.gy0[b], h, ny) - 1, 0);
    r.cy1 = min(cell_coord(y + R, B.gy0[b], h, ny) + 1, ny - 1);
    return r;
}

/* ------------------------------------------------------------------ */
/* k_cutoff: ring counting with radius doubling (FXY.hpp:441-534)       */
/* one warp per node, candidates from the cell grid                     */
/* ------------------------------------------------------------------ */
__global__ void __launch_bounds__(kT) k_cutoff(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int V = B.Vn[b];
    const int i0 = B.chunk_start[c];
    if (i0 >= V) return;
    const int64_t base = B.offs[b];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int N = min(B.N_cut, V - 1);  // FXY.hpp:77
    const double s = 2.0 * B.spn[b];    // FXY.hpp:78
    const int nx = B.gnx[b];
    for (int qi = w; qi < kT && i0 + qi < V; qi += kT / 32) {
        const int i = i0 + qi;
        const double2 me = B.P[base + i];
        int L = 0, st = 0, passes = 0;
        double cut = 0.0;
        for (;;) {
            const double sL = s * (double)L;
            double lim[5], lo[5], hi[5];
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                lim[j] = fma(s, (double)j, sL);  // nvcc's contraction of s*j + s*L
                const double l2 = lim[j] * lim[j];
                lo[j] = l2 * (1.0 - 0x1p-40);
                hi[j] = l2 * (1.0 + 0x1p-40);
            }
            int cnt1 = 0, cnt2 = 0, cnt3 = 0, cnt4 = 0;
            const Box bx = box_of(B, b, me.x, me.y, lim[4]);
            for (int cy = bx.cy0; cy <= bx.cy1; ++cy) {
                const int64_t k0 = B.cellstart[base + cy * nx + bx.cx0];
                const int64_t k1 = B.cellstart[base + cy * nx + bx.cx1 + 1];
                for (int64_t k = k0 + lane; k < k1; k += 32) {
                    const double2 p = B.spt[k];
                    const double dX = fabs(me.x - p.x), dY = fabs(me.y - p.y);
                    const double q = fma(dY, dY, dX * dX);
                    if (q >= hi[4] || B.sidx[k] == i) continue;
                    // counts[j] = #{ sqrt(q) < lim[j] } (FXY.hpp:479-482); the
                    // square root is taken only inside the rounding band
                    double d = -1.0;
                    bool in;
#define F2M_RING(J, CNT)                                             \
    if (q < lo[J]) in = true;                                        \
    else if (q >= hi[J]) in = false;                                 \
    else { if (d < 0.0) d = sqrt(q); in = d < lim[J]; }              \
    if (!in) continue;                                               \
    CNT++;
                    F2M_RING(4, cnt4)
                    F2M_RING(3, cnt3)
                    F2M_RING(2, cnt2)
                    F2M_RING(1, cnt1)
#undef F2M_RING
                }
            }
            const int cnts[5] = {0, (int)__reduce_add_sync(0xffffffffu, cnt1),
                                 (int)__reduce_add_sync(0xffffffffu, cnt2),
                                 (int)__reduce_add_sync(0xffffffffu, cnt3),
                                 (int)__reduce_add_sync(0xffffffffu, cnt4)};
            st = 0;
            cut = lim[0];
#pragma unroll
            for (int j = 1; j < 5; ++j) {  // FXY.hpp:486-502
                st = cnts[j];
                cut = lim[j];
                if (cnts[j] > N) break;
            }
            if (st >= N || ++passes >= kMaxPasses) break;
            L = (L == 0) ? 5 : 2 * L;  // FXY.hpp:526-531
        }
        if (lane == 0) {
            B.cut[base + i] = cut;
            B.stat[base + i] = st;
            if (st < N) B.status[b] = F2M_ERR_CAPACITY;
        }
    }
}

/* ------------------------------------------------------------------ */
/* k_select: first-N incident candidates of each node                   */
/* ------------------------------------------------------------------ */
// Key of the pair (i,j) at distance d in the reference's global candidate
// order: thrust::sort by d, ties in emission order, where the pair a<b is
// emitted by a when d <= cut[a] and by b otherwise (FXY.hpp:388-432).
__device__ __forceinline__ bool key_less(double d1, int e1, int o1, double d2, int e2, int o2) {
    if (d1 != d2) return d1 < d2;
    if (e1 != e2) return e1 < e2;
    return o1 < o2;
}

// One warp per node keeps the sorted first-N list distributed over its
// lanes (position lane*RPL + r); candidates come from the cells within the
// node's cut-off radius, which holds all of its first N (their distances are
// below the cut-off, FXY.hpp:486-502).  Insertion is a warp-wide shift.
// Edge cost of a candidate at FP64 distance d: the reference's raw distance,
// or TSPLIB EUC_2D nint(d) (the oracle's ORC_COST_NINT).
__device__ __forceinline__ double cand_cost(double d, int mode) {
    return mode == F2M_COST_NINT ? (double)(long long)(d + 0.5) : d;
}

template <int RPL>
__global__ void __launch_bounds__(kT) k_select(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int V = B.Vn[b];
    const int i0 = B.chunk_start[c];
    if (i0 >= V) return;
    const int64_t base = B.offs[b];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int N = min(B.N, V - 1);
    const int nx = B.gnx[b];
    const int mode = B.cost_mode;
    const unsigned FULL = 0xffffffffu;
    for (int qi = w; qi < kT && i0 + qi < V; qi += kT / 32) {
        const int i = i0 + qi;
        const double2 me = B.P[base + i];
        const double cut_i = B.cut[base + i];
        double kd[RPL];
        int ke[RPL], ko[RPL];
#pragma unroll
        for (int r = 0; r < RPL; ++r) { kd[r] = INFINITY; ke[r] = INT_MAX; ko[r] = INT_MAX; }
        int cnt = 0;
        double worst_hi = INFINITY;
        // Pass 0 scans the cells around the node's own cut-off radius, where its
        // first N candidates lie.  With nint costs a candidate out to
        // (N-th cost + 0.5) can tie with the N-th, so pass 1 scans the cells of
        // that wider box that pass 0 did not.
        Box bx0 = box_of(B, b, me.x, me.y, cut_i);
        for (int pass = 0; pass < 2; ++pass) {
            Box bx = bx0;
            if (pass == 1) {
                if (mode != F2M_COST_NINT || cnt < N) break;
                const int wl = (N - 1) / RPL, wr = (N - 1) % RPL;
                double mineD = 0.0;
#pragma unroll
                for (int r = 0; r < RPL; ++r)
                    if (r == wr) mineD = kd[r];
                const double R2 = __shfl_sync(FULL, mineD, wl) + 0.5;
                if (!(R2 > cut_i)) break;
                bx = box_of(B, b, me.x, me.y, R2);
            }
            for (int cy = bx.cy0; cy <= bx.cy1; ++cy) {
                for (int cx0 = bx.cx0; cx0 <= bx.cx1;) {
                    // a run of cells on this row (pass 1: outside pass 0's box)
                    int cx1 = bx.cx1;
                    if (pass == 1 && cy >= bx0.cy0 && cy <= bx0.cy1) {
                        if (cx0 >= bx0.cx0 && cx0 <= bx0.cx1) { cx0 = bx0.cx1 + 1; continue; }
                        if (cx0 < bx0.cx0) cx1 = min(cx1, bx0.cx0 - 1);
                    }
                    const int64_t k0 = B.cellstart[base + cy * nx + cx0];
                    const int64_t k1 = B.cellstart[base + cy * nx + cx1 + 1];
                    cx0 = cx1 + 1;
                    for (int64_t kb = k0; kb < k1; kb += 32) {
                        const int64_t k = kb + lane;
                        bool take = false;
                        double cd_ = 0.0;
                        int em = 0, oth = 0;
                        if (k < k1) {
                            const int j = B.sidx[k];
                            const double2 p = B.spt[k];
                            const double dX = fabs(me.x - p.x), dY = fabs(me.y - p.y);
                            const double q = fma(dY, dY, dX * dX);
                            if (j != i && (cnt < N || q <= worst_hi)) {
                                const double d = sqrt(q);
                                const double cut_j = B.cut[base + j];
                                // a candidate of the reference (FXY.hpp:388-432):
                                // within either endpoint's cut-off; the lower id
                                // emits it if within its own cut-off
                                take = d <= cut_i || d <= cut_j;
                                const int a = min(i, j), bb = max(i, j);
                                const double cut_a = (a == i) ? cut_i : cut_j;
                                em = (d <= cut_a) ? a : bb;
                                oth = (em == a) ? bb : a;
                                cd_ = cand_cost(d, mode);
                            }
                        }
                        unsigned mask = __ballot_sync(FULL, take);
                        while (mask) {
                            const int src = __ffs(mask) - 1;
                            mask &= mask - 1;
                            const double cd = __shfl_sync(FULL, cd_, src);
                            const int ce = __shfl_sync(FULL, em, src);
                            const int co = __shfl_sync(FULL, oth, src);
                            int mine = 0;
#pragma unroll
                            for (int r = 0; r < RPL; ++r)
                                if (lane * RPL + r < cnt && key_less(kd[r], ke[r], ko[r], cd, ce, co)) mine++;
                            const int pos = (int)__reduce_add_sync(FULL, mine);
                            if (pos >= N) continue;
                            const double pd = __shfl_up_sync(FULL, kd[RPL - 1], 1);
                            const int pe = __shfl_up_sync(FULL, ke[RPL - 1], 1);
                            const int po = __shfl_up_sync(FULL, ko[RPL - 1], 1);
#pragma unroll
                            for (int r = RPL - 1; r >= 0; --r) {
                                const int g = lane * RPL + r;
                                if (g > pos) {
                                    if (r > 0) { kd[r] = kd[r - 1]; ke[r] = ke[r - 1]; ko[r] = ko[r - 1]; }
                                    else { kd[r] = pd; ke[r] = pe; ko[r] = po; }
                                } else if (g == pos) {
                                    kd[r] = cd; ke[r] = ce; ko[r] = co;
                                }
                            }
                            cnt = min(cnt + 1, N);
                            if (cnt == N) {
                                const int wl = (N - 1) / RPL, wr = (N - 1) % RPL;
                                double mineD = 0.0;
#pragma unroll
                                for (int r = 0; r < RPL; ++r)
                                    if (r == wr) mineD = kd[r];
                                const double wd = __shfl_sync(FULL, mineD, wl);
                                // squared-distance bound of a key that can still
                                // enter (raw: <= wd; nint: < wd + 0.5)
                                const double wr_ = (mode == F2M_COST_NINT) ? wd + 0.5 : wd;
                                worst_hi = wr_ * wr_ * (1.0 + 0x1p-40);
                            }
                        }
                    }
                }
            }
        }
        const int64_t o = (base + i) * (int64_t)B.N;
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
            const int g = lane * RPL + r;
            if (g < cnt) {
                B.top_nbr[o + g] = (ke[r] == i) ? ko[r] : ke[r];
                B.top_cost[o + g] = kd[r];
                B.top_em[o + g] = ke[r];
                B.top_oth[o + g] = ko[r];
            }
        }
        if (lane == 0) B.ntop[base + i] = cnt;
    }
}

/* ------------------------------------------------------------------ */
/* graph build: union of the per-node lists (graph_tour.hpp:28-98)      */
/* ------------------------------------------------------------------ */
__device__ __forceinline__ bool in_top(const Batch& B, int64_t base, int j, int i) {
    const int64_t o = (base + j) * (int64_t)B.N;
    const int n = B.ntop[base + j];
    for (int m = 0; m < n; ++m)
        if (B.top_nbr[o + m] == i) return true;
    return false;
}

__global__ void __launch_bounds__(kT) k_graph_rev(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int V = B.Vn[b];
    const int i = B.chunk_start[c] + threadIdx.x;
    if (i >= V) return;
    const int64_t base = B.offs[b];
    const int64_t o = (base + i) * (int64_t)B.N;
    const int nt = B.ntop[base + i];
    for (int k = 0; k < nt; ++k) {
        const int j = B.top_nbr[o + k];
        const bool dup = in_top(B, base, j, i);
        B.tdup[o + k] = dup;
        if (!dup) atomicAdd(&B.rev[base + j], 1);
    }
    // d_min over kept edges (graph_tour.hpp:70): the smallest cost of a
    // node's list is its first entry; positive doubles order like their bits
    if (nt > 0) {
        atomicMin(&B.dmin_bits[b], (unsigned long long)__double_as_longlong(B.top_cost[o]));
        // a zero-cost edge (nint of a distance below 0.5) leaves D undefined
        if (B.top_cost[o] == 0.0) B.status[b] = F2M_ERR_INPUT;
    }
}

// degree per input position (0 for dropped duplicates and padding)
__global__ void __launch_bounds__(kT) k_graph_deg(Batch B, int64_t* deg) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    const int i = B.chunk_start[c] + threadIdx.x;
    const int64_t base = B.offs[b];
    const int n = (int)(B.offs[b + 1] - base);
    if (i >= n) return;
    int64_t d = 0;
    if (B.status[b] == F2M_OK && i < B.Vn[b]) d = B.ntop[base + i] + B.rev[base + i];
    deg[base + i] = d;
}

__global__ void __launch_bounds__(kT) k_graph_fill(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int V = B.Vn[b];
    const int i = B.chunk_start[c] + threadIdx.x;
    if (i >= V) return;
    const int64_t base = B.offs[b];
    const int64_t o = (base + i) * (int64_t)B.N;
    const int nt = B.ntop[base + i];
    const int64_t r = B.row[base + i];
    for (int k = 0; k < nt; ++k) {
        const int j = B.top_nbr[o + k];
        const double cost = B.top_cost[o + k];
        const int em = B.top_em[o + k], oth = B.top_oth[o + k];
        B.s_nbr[r + k] = j; B.s_cost[r + k] = cost; B.s_em[r + k] = em; B.s_oth[r + k] = oth;
        if (!B.tdup[o + k]) {
            const int p = atomicAdd(&B.cursor[base + j], 1);
            const int64_t s2 = B.row[base + j] + B.ntop[base + j] + p;
            B.s_nbr[s2] = i; B.s_cost[s2] = cost; B.s_em[s2] = em; B.s_oth[s2] = oth;
        }
    }
}

// Sort each node's slots by the global edge order; the result is the
// reference's per-node list (edges pushed in edge-id order, graph_tour.hpp:87-88).
__global__ void __launch_bounds__(kT) k_graph_sort(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int V = B.Vn[b];
    const int i = B.chunk_start[c] + threadIdx.x;
    if (i >= V) return;
    const int64_t base = B.offs[b];
    const int64_t r0 = B.row[base + i], r1 = B.row[base + i + 1];
    if (r1 - r0 > 65535) { B.status[b] = F2M_ERR_CAPACITY; return; }
    constexpr int kLocal = 48;  // lists up to this long are sorted in registers/local memory
    const int n = (int)(r1 - r0);
    if (n <= kLocal) {
        double kd[kLocal];
        int ke[kLocal], ko[kLocal], kn[kLocal];
        for (int a = 0; a < n; ++a) {
            const double d = B.s_cost[r0 + a];
            const int e = B.s_em[r0 + a], o2 = B.s_oth[r0 + a], nb = B.s_nbr[r0 + a];
            int p = a;
            while (p > 0 && key_less(d, e, o2, kd[p - 1], ke[p - 1], ko[p - 1])) {
                kd[p] = kd[p - 1]; ke[p] = ke[p - 1]; ko[p] = ko[p - 1]; kn[p] = kn[p - 1];
                --p;
            }
            kd[p] = d; ke[p] = e; ko[p] = o2; kn[p] = nb;
        }
        for (int a = 0; a < n; ++a) {
            B.s_cost[r0 + a] = kd[a]; B.s_em[r0 + a] = ke[a];
            B.s_oth[r0 + a] = ko[a]; B.s_nbr[r0 + a] = kn[a];
        }
    } else {
    for (int64_t a = r0 + 1; a < r1; ++a) {
        const double kd = B.s_cost[a];
        const int ke = B.s_em[a], ko = B.s_oth[a], kn = B.s_nbr[a];
        int64_t p = a;
        while (p > r0 && key_less(kd, ke, ko, B.s_cost[p - 1], B.s_em[p - 1], B.s_oth[p - 1])) {
            B.s_cost[p] = B.s_cost[p - 1]; B.s_em[p] = B.s_em[p - 1];
            B.s_oth[p] = B.s_oth[p - 1]; B.s_nbr[p] = B.s_nbr[p - 1];
            --p;
        }
        B.s_cost[p] = kd; B.s_em[p] = ke; B.s_oth[p] = ko; B.s_nbr[p] = kn;
    }
    }
    const double dmin = __longlong_as_double((long long)B.dmin_bits[b]);
    for (int64_t a = r0; a < r1; ++a) {
        Slot s;
        s.D = B.s_cost[a] / dmin;  // F2M.h:101
        s.nbr = B.s_nbr[a];
        s.aux = (int32_t)(a - r0);
        B.slot[a] = s;
        B.perm[a] = (uint16_t)(a - r0);
        B.pslot[a] = s;
    }
}

__global__ void __launch_bounds__(kT) k_graph_mirror(Batch B) {
    const int c = blockIdx.x;
    const int b = B.chunk_inst[c];
    if (B.status[b] != F2M_OK) return;
    const int V = B.Vn[b];
    const int i = B.chunk_start[c] + threadIdx.x;
    if (i >= V) return;
    const int64_t base = B.offs[b];
    const int64_t r0 = B.row[base + i], r1 = B.row[base + i + 1];
    for (int64_t a = r0; a < r1; ++a) {
        // the same edge carries the same key in both lists, and both lists
        // are sorted by key: binary search
        const int j = B.s_nbr[a];
        const double kd = B.s_cost[a];
        const int ke = B.s_em[a], ko = B.s_oth[a];
        int64_t lo = B.row[base + j], hi = B.row[base + j + 1];
        const int64_t q0 = lo;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (key_less(B.s_cost[mid], B.s_em[mid], B.s_oth[mid], kd, ke, ko)) lo = mid + 1; else hi = mid;
        }
        B.mirror[a] = (lo < B.row[base + j + 1] && B.s_nbr[lo] == i) ? (int)(lo - q0) : -1;
    }
}

/* ------------------------------------------------------------------ */
/* exclusive scan of int64 (row offsets)                                */
/* ------------------------------------------------------------------ */
constexpr int kScanPer = 4;
constexpr int kScanBlock = kT * kScanPer;

__global__ void __launch_bounds__(kT) k_scan_local(const int64_t* in, int64_t* out, int64_t n,
                                                   int64_t* sums) {
    __shared__ long long swarp[kT / 32 + 1];
    const int64_t o = (int64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
    long long v[kScanPer];
    long long tsum = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = (o + k < n) ? in[o + k] : 0;
        tsum += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long inc = tsum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
    }
    if (lane == 31) swarp[w] = inc;
    __syncthreads();
    if (w == 0) {
        long long s = (lane < kT / 32) ? swarp[lane] : 0;
        long long incs = s;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, incs, off);
            if (lane >= off) incs += y;
        }
        if (lane < kT / 32) swarp[lane] = incs - s;
        if (lane == kT / 32 - 1) swarp[kT / 32] = incs;
    }
    __syncthreads();
    long long run = swarp[w] + inc - tsum;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (o + k < n) out[o + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = swarp[kT / 32];
}

// single CTA: exclusive scan of the block sums (in place)
__global__ void __launch_bounds__(kT) k_scan_sums(int64_t* sums, int64_t nb) {
    __shared__ long long swarp[kT / 32 + 1];
    __shared__ long long s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t r = 0; r < nb; r += kT) {
        const int64_t k = r + threadIdx.x;
        const long long x = (k < nb) ? sums[k] : 0;
        long long inc = x;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, inc, off);
            if (lane >= off) inc += y;
        }
        if (lane == 31) swarp[w] = inc;
        __syncthreads();
        if (w == 0) {
            long long s = (lane < kT / 32) ? swarp[lane] : 0;
            long long incs = s;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                long long y = __shfl_up_sync(0xffffffffu, incs, off);
                if (lane >= off) incs += y;
            }
            if (lane < kT / 32) swarp[lane] = incs - s;
            if (lane == kT / 32 - 1) swarp[kT / 32] = incs;
        }
        __syncthreads();
        if (k < nb) sums[k] = s_carry + swarp[w] + inc - x;
        __syncthreads();
        if (threadIdx.x == 0) s_carry += swarp[kT / 32];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = s_carry;
}

__global__ void __launch_bounds__(kT) k_scan_add(int64_t* out, int64_t n, const int64_t* sums) {
    const int64_t o = (int64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
    const int64_t add = sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanPer; ++k)
        if (o + k < n) out[o + k] += add;
}

int64_t scan_scratch_elems(int64_t n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

// out[0..n) = exclusive scan of in[0..n); out[n] = total.
cudaError_t launch_scan(const int64_t* in, int64_t* out, int64_t n, int64_t* scratch,
                        cudaStream_t s, int64_t* launches) {
    const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb == 0) return cudaMemsetAsync(out, 0, sizeof(int64_t), s);
    k_scan_local<<<(unsigned)nb, kT, 0, s>>>(in, out, n, scratch);
    k_scan_sums<<<1, kT, 0, s>>>(scratch, nb);
    k_scan_add<<<(unsigned)nb, kT, 0, s>>>(out, n, scratch);
    // total
    cudaError_t e = cudaMemcpyAsync(out + n, scratch + nb, sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
    *launches += 3;
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* the solver: a team of threads runs one instance's whole schedule      */
/* ------------------------------------------------------------------ */
// A CTA holds TEAMS independent teams of TEAM threads.  Each team takes
// instances from a work counter and keeps, per instance, the potentials F
// (double-buffered for the Jacobi step) and the EF lists (D as FP64,
// neighbour as u16) in its slice of shared memory.  Team barriers are named
// barriers (barrier.sync id, TEAM).
template <int TEAM>
struct Team {
    int tid, id;
    double* sred;       // TEAM/32
    long long* sredl;   // TEAM/32
    int* swarp;         // TEAM/32 + 1
    int* sint;          // 4 ints
    // barrier.sync without .aligned: a team may reach it with a diverged warp
    // (after `if (tid == 0) {...}`), which the aligned form (bar.sync) forbids
    __device__ __forceinline__ void sync() const {
        asm volatile("barrier.sync %0, %1;" ::"r"(id + 1), "r"(TEAM) : "memory");
    }
    __device__ double max(double x) const {
        const int lane = tid & 31, w = tid >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sred[w] = x;
        sync();
        double r = -INFINITY;
        for (int k = 0; k < TEAM / 32; ++k) r = fmax(r, sred[k]);
        sync();
        return r;
    }
    __device__ double sum(double x) const {
        const int lane = tid & 31, w = tid >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sred[w] = x;
        sync();
        double r = 0.0;
        for (int k = 0; k < TEAM / 32; ++k) r += sred[k];  // same order in every thread
        sync();
        return r;
    }
    __device__ long long sum_ll(long long x) const {
        const int lane = tid & 31, w = tid >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sredl[w] = x;
        sync();
        long long r = 0;
        for (int k = 0; k < TEAM / 32; ++k) r += sredl[k];
        sync();
        return r;
    }
    __device__ long long max_ll(long long x) const {
        const int lane = tid & 31, w = tid >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = ::max(x, (long long)__shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) sredl[w] = x;
        sync();
        long long r = LLONG_MIN;
        for (int k = 0; k < TEAM / 32; ++k) r = ::max(r, sredl[k]);
        sync();
        return r;
    }
    // exclusive scan in team-thread order; *total = team sum
    __device__ int excl_scan(int x, int* total) const {
        const int lane = tid & 31, w = tid >> 5;
        int inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) swarp[w] = inc;
        sync();
        int before = 0, tot = 0;
        for (int k = 0; k < TEAM / 32; ++k) {
            const int v = swarp[k];
            if (k < w) before += v;
            tot += v;
        }
        sync();
        *total = tot;
        return before + inc - x;
    }
};

// Shared-memory slice of one team.  H = F/2 is kept instead of F: halving is
// exact, so H_new = H + grad/2 equals F_new/2 bit for bit and a reduced cost
// D + 0.5*F[v1] + 0.5*F[v2] is (D + H[v1]) + H[v2] with the same rounding.
//
// The EF lists are stored SELL-32: after each update_EF the nodes are ordered
// by list length (counting sort, longest first), cut into slices of 32 nodes
// (one warp), and each slice holds its nodes' entries column-major
// (entry k of lane l at 32*k + l), padded with +inf to the slice's longest
// list.  A warp then reads its slice with unit stride and all lanes run the
// same trip count.  Padding cannot change the three smallest values (it is
// above the compare chain's 1e6 sentinels).  Slices are cached in shared
// memory in order; the rest live in the same layout in the instance's part of
// a global arena (coalesced, L2-resident), and a slice that fits in neither
// reads each node's list from the node-indexed copy.
struct TeamMem {
    double* Ha;
    double* Hb;
    uint16_t* ord;   // 32*NS: nodes in slice order
    int* soff;       // NS: >= 0 shared offset; kSelGlobal + g: global offset g; kSelNode: node copy
    int* swid;       // NS: slice width (longest list)
    int* hist;       // 258: counting-sort buckets; hist[256] = total list length,
                     // hist[257] = SELL entries incl. padding (32 x slice width, summed)
    double* eD;      // cap entries: D
    uint16_t* eW;    // cap entries: neighbour | 0x8000 when the neighbour is the lower id
    double* gsD;     // gcap entries in global memory
    uint16_t* gsW;
    int* cnt;        // V: EF list length per node (cuda_EF_NodesStat), global
    int cap;
    int gcap;
    int NS;
};
constexpr int kSelGlobal = -(1 << 30);  // soff in [kSelGlobal, -1]: global SELL
constexpr int kSelNode = INT_MIN;

__device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

__device__ __forceinline__ TeamMem carve_team(unsigned char* base, size_t bytes, const Batch& B, int b,
                                              int V) {
    TeamMem M;
    M.NS = (V + 31) / 32;
    size_t o = 0;
    M.Ha = reinterpret_cast<double*>(base + o); o += (size_t)V * 8;
    M.Hb = reinterpret_cast<double*>(base + o); o = align16(o + (size_t)V * 8);
    M.soff = reinterpret_cast<int*>(base + o); o = align16(o + (size_t)M.NS * 4);
    M.swid = reinterpret_cast<int*>(base + o); o = align16(o + (size_t)M.NS * 4);
    M.hist = reinterpret_cast<int*>(base + o); o = align16(o + 258 * 4);
    M.ord = reinterpret_cast<uint16_t*>(base + o); o = align16(o + (size_t)M.NS * 32 * 2);
    M.eD = reinterpret_cast<double*>(base + o);
    const long long rest = (long long)bytes - (long long)o;
    int cap = rest > 0 ? (int)(rest / 10) : 0;
    cap &= ~31;
    M.eW = reinterpret_cast<uint16_t*>(M.eD + cap);
    M.cap = cap;
    const int64_t p0 = B.offs[b], p1 = B.offs[b + 1];
    M.gsD = B.selD + B.sel_stride * p0;
    M.gsW = B.selW + B.sel_stride * p0;
    const int64_t gcap = B.sel_stride * (p1 - p0);
    M.gcap = (int)(gcap < ((int64_t)1 << 29) ? gcap : ((int64_t)1 << 29));
    M.cnt = B.efcnt + p0;
    return M;
}
__device__ __host__ inline size_t team_fixed_bytes(int V) {
    const int NS = (V + 31) / 32;
    return (size_t)V * 16 + (size_t)NS * 8 + 258 * 4 + (size_t)NS * 64 + 5 * 16;
}

__device__ __forceinline__ uint16_t ef_word(int v, int nbr) {
    return (uint16_t)(nbr | (nbr < v ? 0x8000 : 0));
}

// The reduced cost of an EF entry (D, word) of node v.
__device__ __forceinline__ double ef_d(double D, uint16_t w, double hv, const double* __restrict__ H) {
    const double a = H[w & 0x7fff];
    const bool lo = (w & 0x8000) != 0;
    return (D + (lo ? a : hv)) + (lo ? hv : a);
}

// cuda_get_Nodes_grad_R (graph_cuda_grad.hpp:321-340): grad = -(v1+v2)/2 over
// the 2nd and 3rd smallest of {first, rest.., 1e6, 1e6}.  While the first value
// is below 1e6 the reference's compare chain keeps v0<=v1<=v2 and is a sorted
// insertion (top3_insert, branch-free compares and selects); otherwise the chain
// itself runs (it can then leave v0 > v1).  Returns grad/2, the step of H.
template <class Get>
__device__ __forceinline__ double half_grad(int n, Get get) {
    double v0 = get(0), v1 = 1e6, v2 = 1e6;
    if (v0 < 1e6) {
#pragma unroll 4
        for (int k = 1; k < n; ++k) top3_insert(get(k), v0, v1, v2);
    } else {
        for (int k = 1; k < n; ++k) {
            const double x = get(k);
            if (x < v0) { v2 = v1; v1 = v0; v0 = x; continue; }
            if (x < v1) { v2 = v1; v1 = x; continue; }
            if (x < v2) { v2 = x; }
        }
    }
    return (-(v1 + v2) / 2) * 0.5;
}

// Copies of the active sets (update_EF), with restrict pointers so that the
// compiler may issue the loads of an unrolled group before its stores.
// node v's list prefix (n slots in list order) -> its node-indexed copy
__device__ __forceinline__ void copy_ef_prefix(const Slot* __restrict__ ps, double* __restrict__ gD,
                                               uint16_t* __restrict__ gN, int n, int v) {
#pragma unroll 4
    for (int k = 0; k < n; ++k) {
        const Slot sl = ps[k];
        gD[k] = sl.D;
        gN[k] = (uint16_t)(sl.nbr | (sl.nbr < v ? 0x8000 : 0));
    }
}
// one lane's column of a SELL-32 slice of width wdt from a node-indexed list
// of n entries (padding: +inf, word 0)
__device__ __forceinline__ void fill_slice_lane(const double* __restrict__ gD, const uint16_t* __restrict__ gN,
                                                int n, int wdt, double* __restrict__ dD, uint16_t* __restrict__ dW) {
#pragma unroll 4
    for (int k = 0; k < wdt; ++k) {
        const bool real = k < n;
        dD[32 * k] = real ? gD[k] : INFINITY;
        dW[32 * k] = real ? gN[k] : (uint16_t)0;
    }
}

template <int TEAM>
struct Solver {
    static constexpr int WARPS = TEAM / 32;
    const Batch& B;
    const DevParams& P;
    const Inst& I;
    const Team<TEAM>& T;
    TeamMem M;
    double* Hc;   // H = F/2, current
    double* Hn;   // next (Jacobi double buffer)
    int64_t row0;
    long long iters = 0;
    long long wslots = 0;  // active slots read, summed over iterations
    long long wpad = 0;    // SELL entries the warps sweep (padding included), summed over iterations
    int checks = 0;
    bool capped = false;

    __device__ Solver(const Batch& b, const DevParams& p, const Inst& i, const Team<TEAM>& t, TeamMem m)
        : B(b), P(p), I(i), T(t), M(m), Hc(m.Ha), Hn(m.Hb), row0(i.row[0]) {}

    __device__ int deg(int v) const { return (int)(I.row[v + 1] - I.row[v]); }
    __device__ void swap_f() { double* t = Hc; Hc = Hn; Hn = t; }

    // grad/2 of the node in lane `lane` of slice s; v = that node (or -1)
    __device__ __forceinline__ double slice_hgrad(int s, int lane, int& v, double& hv) const {
        const int p = s * 32 + lane;
        v = (p < I.V) ? (int)M.ord[p] : -1;
        const int vv = v < 0 ? (int)M.ord[s * 32] : v;  // padding lanes shadow lane 0
        hv = Hc[vv];
        const int off = M.soff[s];
        if (off >= 0) {
            const double* Dp = M.eD + off + lane;
            const uint16_t* Wp = M.eW + off + lane;
            return half_grad(M.swid[s], [&](int k) { return ef_d(Dp[32 * k], Wp[32 * k], hv, Hc); });
        }
        if (off != kSelNode) {
            const double* Dp = M.gsD + (off - kSelGlobal) + lane;
            const uint16_t* Wp = M.gsW + (off - kSelGlobal) + lane;
            return half_grad(M.swid[s], [&](int k) { return ef_d(Dp[32 * k], Wp[32 * k], hv, Hc); });
        }
        const int64_t go = I.row[vv] - row0;
        const double* Dp = I.gD + go;
        const uint16_t* Wp = I.gN + go;
        return half_grad(M.cnt[vv], [&](int k) { return ef_d(Dp[k], Wp[k], hv, Hc); });
    }
    // one Jacobi step: F += grad(F) (graph_cuda.cu:293-304), as H += grad/2;
    // frozen nodes keep F (block_EF_iter_BLOCK, graph_cuda.cu:278-289)
    template <bool MASKED>
    __device__ __forceinline__ void step() {
        const int w = T.tid >> 5, lane = T.tid & 31;
        for (int s = w; s < M.NS; s += WARPS) {
            int v;
            double hv;
            const double g = slice_hgrad(s, lane, v, hv);
            if (v >= 0) Hn[v] = (MASKED && B.shift[I.base + v] != 0.0) ? hv : hv + g;
        }
        wslots += M.hist[256];
        wpad += M.hist[257];
        T.sync();
        swap_f();
        iters++;
    }
    __device__ void jacobi() { step<false>(); }
    __device__ void jacobi_masked() { step<true>(); }
    // max |grad| (max_node_grad, graph_cuda_maxmin.hpp:29-37)
    __device__ double grad_max() const {
        const int w = T.tid >> 5, lane = T.tid & 31;
        double m = 0.0;
        for (int s = w; s < M.NS; s += WARPS) {
            int v;
            double hv;
            const double g = slice_hgrad(s, lane, v, hv);
            if (v >= 0) m = fmax(m, fabs(g));
        }
        return 2.0 * T.max(m);
    }
    // update_EF (graph_cuda.cu:229-252).  from_perm: copy each node's list
    // prefix (cnt[v] entries in the order of its permuted list) to the
    // node-indexed global copy; then build the SELL-32 cache from that copy.
    __device__ void rebuild_ef(bool from_perm) {
        const int V = I.V;
        long long tot = 0;
        for (int v = T.tid; v < V; v += TEAM) tot += M.cnt[v];
        if (from_perm) {
            for (int v = T.tid; v < V; v += TEAM) {
                const int64_t r0 = I.row[v];
                const int64_t go = r0 - row0;
                const int n = M.cnt[v];
                copy_ef_prefix(I.pslot + r0, I.gD + go, I.gN + go, n, v);
            }
        }
        // counting sort by list length, longest first (bucket 255 = 255 or more)
        for (int k = T.tid; k < 257; k += TEAM) M.hist[k] = 0;
        tot = T.sum_ll(tot);  // (also orders the hist reset before its use)
        if (T.tid == 0) M.hist[256] = (int)tot;
        // (lanes with the same bucket add once per warp: few buckets, many nodes)
        for (int v0 = T.tid & ~31; v0 < V; v0 += TEAM) {
            const int v = v0 + (T.tid & 31);
            const int key = v < V ? 255 - min(M.cnt[v], 255) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            if (key >= 0 && (T.tid & 31) == __ffs(peers) - 1) atomicAdd(&M.hist[key], __popc(peers));
        }
        T.sync();
        if (T.tid < 32) {  // exclusive scan of the 256 buckets, 8 per lane
            const int l = T.tid;
            int c[8], run = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) { c[j] = M.hist[8 * l + j]; run += c[j]; }
            int inc = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (l >= o) inc += y;
            }
            int base = inc - run;
#pragma unroll
            for (int j = 0; j < 8; ++j) { M.hist[8 * l + j] = base; base += c[j]; }
        }
        T.sync();
        for (int v0 = T.tid & ~31; v0 < V; v0 += TEAM) {
            const int lane_ = T.tid & 31, v = v0 + lane_;
            const int key = v < V ? 255 - min(M.cnt[v], 255) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const int leader = __ffs(peers) - 1;
            int base = 0;
            if (key >= 0 && lane_ == leader) base = atomicAdd(&M.hist[key], __popc(peers));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (key >= 0) M.ord[base + __popc(peers & ((1u << lane_) - 1u))] = (uint16_t)v;
        }
        T.sync();
        // slice widths (longest list of the slice) and offsets in the cache
        const int w = T.tid >> 5, lane = T.tid & 31;
        for (int s = w; s < M.NS; s += WARPS) {
            const int p = s * 32 + lane;
            const int c = (p < V) ? M.cnt[M.ord[p]] : 0;
            const int mx = __reduce_max_sync(0xffffffffu, c);
            if (lane == 0) M.swid[s] = max(mx, 1);
        }
        T.sync();
        // slice positions in slice order: the leading slices that fit go to
        // shared memory, the rest to the global arena (from its start)
        int carry = 0;
        long long lead = 0;
        for (int r = 0; r < M.NS; r += TEAM) {
            const int s = r + T.tid;
            const int size = (s < M.NS) ? 32 * M.swid[s] : 0;
            int t;
            const int ex = T.excl_scan(size, &t);
            if (s < M.NS) {
                M.soff[s] = carry + ex;
                if (carry + ex + size <= M.cap) lead = ::max(lead, (long long)(carry + ex + size));
            }
            carry += t;
        }
        if (T.tid == 0) M.hist[257] = carry;  // read after the barriers below
        lead = T.max_ll(lead);
        for (int s = T.tid; s < M.NS; s += TEAM) {
            const int pos = M.soff[s], size = 32 * M.swid[s];
            if (pos + size <= M.cap) continue;
            const int g = pos - (int)lead;
            M.soff[s] = (g + size <= M.gcap) ? kSelGlobal + g : kSelNode;
        }
        T.sync();
        // fill the slices from the node-indexed copy
        for (int s = w; s < M.NS; s += WARPS) {
            const int off = M.soff[s];
            if (off == kSelNode) continue;
            double* dD = (off >= 0) ? M.eD + off : M.gsD + (off - kSelGlobal);
            uint16_t* dW = (off >= 0) ? M.eW + off : M.gsW + (off - kSelGlobal);
            const int p = s * 32 + lane;
            const int v = (p < V) ? (int)M.ord[p] : -1;
            const int n = (v >= 0) ? M.cnt[v] : 0;
            const int64_t go = (v >= 0) ? I.row[v] - row0 : 0;
            fill_slice_lane(I.gD + go, I.gN + go, n, M.swid[s], dD + lane, dW + lane);
        }
        T.sync();
    }
    __device__ void finish_partition() {
        T.sync();
        rebuild_ef(true);
    }
    // check_OPT + update_EF (graph_cuda.cu:229-271) with cuda_partition_v2
    __device__ double check_opt() {
        for (int v = T.tid; v < I.V; v += TEAM) {
            const int d = deg(v);
            M.cnt[v] = (d < P.ef_small_deg) ? d : qpart_ef_pair(I, I.row[v], v, Hc, d, P.ef_thr, P.ef_min);
        }
        finish_partition();
        checks++;
        return grad_max();
    }
    // block_EF (graph_cuda.cu:308-338).  Every call follows a check_OPT whose
    // max |grad| was taken over the same potentials and active sets, so that
    // value is the entry gradient MA.
    __device__ void block_ef(int N, double MA) {
        int count_M = 0;
        for (int it = 0; it < N; ++it) {
            jacobi();
            if (++count_M >= P.check_every) {
                if (MA < P.error_B) break;
                count_M = 0;
            }
        }
    }
    // block_GLOB (graph_cuda.cu:363-430)
    __device__ void block_glob() {
        for (int v = T.tid; v < I.V; v += TEAM) M.cnt[v] = min(deg(v), P.glob_K);  // setvalue2V
        finish_partition();
        for (int go = 0; go < P.glob_rounds; ++go) {
            for (int it = 0; it < P.glob_inner; ++it) jacobi();
            // cuda_partition_v4 (graph_cuda_partition.hpp:89-115)
            for (int v = T.tid; v < I.V; v += TEAM) {
                const int d = deg(v);
                if (d < P.glob_K) { M.cnt[v] = d; continue; }
                const int64_t r0 = I.row[v];
                const double hv = Hc[v];
                double avg = pdv(I, r0, 0, v, Hc, hv);
                for (int k = 1; k < P.glob_K; ++k) avg = fmax(avg, pdv(I, r0, k, v, Hc, hv));
                M.cnt[v] = qpart_ef_pair(I, r0, v, Hc, d, avg, P.ef_min);
            }
            finish_partition();
            if (grad_max() < P.glob_tol) break;
        }
    }
    // run_start_cuda (graph_cuda.cu:163-199)
    __device__ double run_start() {
        block_glob();
        double M_ = check_opt();
        int factor = P.factor0;
        for (int go = 1; go <= P.max_rounds; ++go) {
            block_ef(factor, M_);
            M_ = check_opt();
            if (factor < P.factor_cap) factor += P.factor_step;
            if (M_ < P.error_B) break;
            if (iters > P.max_iters) { capped = true; break; }
        }
        return M_;
    }
    // run_fix_cuda (graph_cuda.cu:204-226)
    __device__ double run_fix() {
        double M_ = check_opt();
        for (int go = 1; go <= P.fix_rounds; ++go) {
            block_ef(P.fix_factor, M_);
            M_ = check_opt();
            if (M_ < P.error_B) break;
            if (iters > P.max_iters) { capped = true; break; }
        }
        return M_;
    }
    // Comb extraction (graph_cuda_comb.hpp:415-475), the device comb check and
    // the primal; writes the per-node state for the host and the results.
    __device__ void combs_and_primal(int b, double M_, bool accumulate) {
        const int V = I.V;
        const double porog = P.porog;
        int* ccnt = reinterpret_cast<int*>(Hn);  // Hn is free: room for 2V ints
        int* lab = ccnt + V;
        for (int v = T.tid; v < V; v += TEAM)  // cuda_partition_v3
            ccnt[v] = qpart_b_pair(I, I.row[v], v, Hc, M.cnt[v], P.comb_thr);
        T.sync();
        for (int v = T.tid; v < V; v += TEAM) {
            const int64_t r0 = I.row[v];
            const double hv = Hc[v];
            bool has = false;
            for (int k = 0; k < ccnt[v] && !has; ++k) {
                const double d = pdv(I, r0, k, v, Hc, hv);
                has = (d >= -porog && d <= porog);
            }
            lab[v] = has ? v : INT_MAX;
        }
        T.sync();
        // a comb is a connected component of half edges rooted at its
        // smallest node id (get_cuda_comb_size, graph_cuda_comb.hpp:320-392);
        // min-label propagation over the half-edge frontier finds them
        volatile int* vlab = lab;
        for (;;) {
            int changed = 0;
            for (int v = T.tid; v < V; v += TEAM) {
                int m = vlab[v];
                if (m == INT_MAX) continue;
                const int64_t r0 = I.row[v];
                const double hv = Hc[v];
                for (int k = 0; k < ccnt[v]; ++k) {
                    const Slot s = I.pslot[r0 + k];
                    const double d = red_d(s, v, Hc, hv);
                    if (d >= -porog && d <= porog) m = min(m, vlab[s.nbr]);
                }
                if (m < vlab[v]) { vlab[v] = m; changed = 1; }
            }
            if (T.sum_ll(changed) == 0) break;
        }
        // state for the host comb check (and a later repair step); the EF
        // lengths are in B.efcnt already
        for (int v = T.tid; v < V; v += TEAM) {
            B.F[I.base + v] = 2.0 * Hc[v];
            B.ccnt[I.base + v] = ccnt[v];
        }
        T.sync();
        // comb check (comb::solve_simple, comb_thread.cpp:180-195) with the
        // host's A/B rule (node::get_statusAB, node.cpp:49-57)
        int* irr = ccnt;  // saved in B.ccnt
        for (int v = T.tid; v < V; v += TEAM) irr[v] = 0;
        T.sync();
        for (int v = T.tid; v < V; v += TEAM) {
            if (lab[v] == INT_MAX) continue;
            const int64_t r0 = I.row[v], r1 = I.row[v + 1];
            const double hv = Hc[v];
            int A = 0, Bc = 0;
            for (int64_t a = r0; a < r1; ++a) {
                const double d = red_d(I.slot[a], v, Hc, hv);
                if (d < porog) { if (d > -porog) Bc++; else A++; }
            }
            if (4 - 2 * A - Bc != 0) irr[lab[v]] = 1;
        }
        T.sync();
        long long nc = 0, ni = 0;
        for (int v = T.tid; v < V; v += TEAM)
            if (lab[v] == v) { nc++; ni += irr[v]; }
        nc = T.sum_ll(nc);
        ni = T.sum_ll(ni);
        // irregular combs of the first solve: k_axb, launched after this
        // kernel, solves their Ax=b on the device and redoes the primal from
        // the comb labels saved here (a separate kernel keeps the system
        // solver's registers out of this one).  After a repair shift the host
        // driver runs the comb stage itself.
        const bool axb = ni > 0 && !accumulate;
        if (axb)
            for (int v = T.tid; v < V; v += TEAM) {
                B.clab[I.base + v] = lab[v];
                B.cirr[I.base + v] = irr[v];
            }
        // primal (graph_cuda.cu:135-147): x = 1 on A edges, 1/2 on the B edges
        // of regular combs; OVAL = sum x*Do, MAX edge rank (graph_tour.hpp:165-184)
        PrimalSums ps;
        for (int v = T.tid; v < V; v += TEAM)
            primal_node(B, I, Hc, (const int*)nullptr, (const int*)nullptr, false, v, porog, ps);
        double lp = ps.lp, dual_neg = ps.dual_neg, fsum = ps.fsum;
        long long maxr = ps.maxr, viol = ps.viol;
        lp = T.sum(lp);
        dual_neg = T.sum(dual_neg);
        fsum = T.sum(fsum);
        maxr = T.max_ll(maxr);
        viol = T.sum_ll(viol);
        if (T.tid == 0) {
            const double dmin = __longlong_as_double((long long)B.dmin_bits[b]);
            B.n_edges[b] = (int32_t)((I.row[V] - I.row[0]) / 2);
            B.n_combs[b] = (int32_t)nc;
            B.n_irr[b] = (int32_t)ni;
            B.max_rank[b] = (int32_t)maxr;
            B.deg_viol[b] = (int32_t)viol;
            B.iters[b] = (accumulate ? B.iters[b] : 0) + iters;
            B.work_nodes[b] = (accumulate ? B.work_nodes[b] : 0) + iters * (long long)V;
            B.work_slots[b] = (accumulate ? B.work_slots[b] : 0) + wslots;
            B.work_pad[b] = (accumulate ? B.work_pad[b] : 0) + wpad;
            B.checks[b] = (accumulate ? B.checks[b] : 0) + checks;
            B.max_grad[b] = M_;
            B.dual[b] = dmin * (-fsum + dual_neg);
            if (capped) { B.status[b] = F2M_ERR_NOT_CONVERGED; B.lp[b] = NAN; }
            else if (ni > 0) { B.status[b] = axb ? kNeedsAxb : kNeedsHost; B.lp[b] = NAN; }
            else { B.status[b] = F2M_OK; B.lp[b] = lp; }
        }
        T.sync();
    }
};

// Persistent CTAs; each team takes instances from `items` (largest first).
template <int TEAM, int TEAMS, bool REFIT>
__global__ void __launch_bounds__(TEAM* TEAMS) k_solve(Batch B, DevParams P, const int32_t* items,
                                                       int n_items, int32_t* queue, int vcap,
                                                       int team_bytes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_red[TEAMS][TEAM / 32];
    __shared__ long long s_redl[TEAMS][TEAM / 32];
    __shared__ int s_warp[TEAMS][TEAM / 32 + 1];
    __shared__ int s_int[TEAMS][4];
    const int id = threadIdx.x / TEAM;
    Team<TEAM> T{(int)(threadIdx.x % TEAM), id, s_red[id], s_redl[id], s_warp[id], s_int[id]};
    unsigned char* mine = smem_raw + (size_t)id * team_bytes;
    for (;;) {
        if (T.tid == 0) T.sint[0] = atomicAdd(queue, 1);
        T.sync();
        const int item = T.sint[0];
        T.sync();
        if (item >= n_items) return;
        const int b = items[item];
        const int st = B.status[b];
        if (REFIT ? (st != F2M_OK && st != kNeedsHost) : (st != F2M_OK)) continue;
        const Inst I = make_inst(B, b);
        if (I.V > vcap || team_fixed_bytes(I.V) > (size_t)team_bytes) {
            if (T.tid == 0) B.status[b] = F2M_ERR_CAPACITY;
            T.sync();
            continue;
        }
        const TeamMem M = carve_team(mine, team_bytes, B, b, I.V);  // sized for this instance
        init_pslot(I, T.tid, TEAM);  // the host paths upload slot and perm only
        Solver<TEAM> S(B, P, I, T, M);
        double Mg;
        if (!REFIT) {
            // F = 0 (graph_cuda_init.hpp:183), or a warm start
            // (resuming from given potentials skips the global phase: run_fix,
            // the schedule the reference runs after a repair shift)
            for (int v = T.tid; v < I.V; v += TEAM) M.Ha[v] = B.F0 ? 0.5 * B.F0[I.base + v] : 0.0;
            T.sync();
            Mg = B.F0 ? S.run_fix() : S.run_start();
        } else {
            // cuda_IRREGULAR_B_recompute (graph_cuda_comb.hpp:542-574): shift the
            // potentials of irregular combs, 20 frozen iterations, run_fix; the
            // EF lists of the last update_EF are in the node-indexed copy
            for (int v = T.tid; v < I.V; v += TEAM) M.Ha[v] = 0.5 * (B.F[I.base + v] + B.shift[I.base + v]);
            T.sync();
            S.rebuild_ef(false);
            for (int go = 0; go < P.frozen_iters; ++go) S.jacobi_masked();
            Mg = S.run_fix();
        }
        S.combs_and_primal(b, Mg, REFIT);
    }
}

/* ------------------------------------------------------------------ */
/* k_axb: Ax=b of irregular combs, then the primal                      */
/* ------------------------------------------------------------------ */
// comb::solve_AxB (comb_thread.cpp:272-304) for every irregular comb of an
// instance the solver left with status kNeedsAxb, on the device: a thread
// per comb (roots r = tid, tid + kAxT, ...), its system in the instance's
// part of the global slice arena (free once the descent is over).  The rows
// are the comb's nodes in ascending id (the reference takes them in its hash
// map's order; the solution does not depend on the order, its last bits
// may).  Each B edge takes x (as FP32, as comb::XB holds it) from the comb
// the host applies last: graph::X is filled comb by comb in root order, so
// the comb with the larger root of the edge's two ends.  When a system does
// not converge within 900 steps (the reference allows 999: near that limit
// the order could decide) or the arena cannot hold the systems, the instance
// goes to the host stage (kNeedsHost), which also runs the repair loop
// (graph_cuda.cu:69-126); otherwise the primal is redone with the Ax=b
// values and the instance is solved.  The potentials come from the saved F.
constexpr int kAxT = 256;
__global__ void __launch_bounds__(kAxT) k_axb(Batch B, DevParams P) {
    const int b = blockIdx.x;
    if (B.status[b] != kNeedsAxb) return;
    __shared__ int swarp[kAxT / 32 + 1];
    __shared__ double sred[kAxT / 32];
    __shared__ long long sredl[kAxT / 32];
    const Inst I = make_inst(B, b);
    const int V = I.V;
    const double porog = P.porog;
    const int64_t row0 = I.row[0];
    const HalfF H{B.F + I.base};
    const int* lab = B.clab + I.base;
    const int* irr = B.cirr + I.base;
    long long need = 0;
    for (int r = threadIdx.x; r < V; r += kAxT) {
        if (lab[r] != r || !irr[r]) continue;
        long long m = 0, z = 0;
        for (int u = 0; u < V; ++u)
            if (lab[u] == r) { m++; z += count_b(I.slot, I.row, H, u, porog); }
        need += axb_comb_doubles(m, z);
    }
    int total = 0;  // (a thread's share is clamped so that the block sum fits an int)
    const int off = block_excl_scan<kAxT>((int)::min(need, (long long)1 << 20), swarp, &total);
    const int64_t p0 = B.offs[b], p1 = B.offs[b + 1];
    const long long gcap = ::min((long long)(B.sel_stride * (p1 - p0)), (long long)1 << 29);
    long long bad = (need >= ((long long)1 << 20) || total > gcap) ? 1 : 0;
    if (total <= gcap) {
        double* w = B.selD + B.sel_stride * p0 + off;
        for (int r = threadIdx.x; r < V && !bad; r += kAxT) {
            if (lab[r] != r || !irr[r]) continue;
            int* mem = reinterpret_cast<int*>(w);
            int m = 0, z = 0;
            for (int u = 0; u < V; ++u)
                if (lab[u] == r) { mem[m++] = u; z += count_b(I.slot, I.row, H, u, porog); }
            double* sys = w + (m + 1) / 2 + 1;
            w += axb_comb_doubles(m, z);
            bad = axb_comb(I.slot, I.row, row0, B.mirror, H, lab, mem, m, z, r, porog, sys, B.xval);
        }
    }
    if (block_sum_ll<kAxT>(bad, sredl) != 0) {
        if (threadIdx.x == 0) { B.status[b] = kNeedsHost; B.lp[b] = NAN; }
        return;
    }
    PrimalSums ps;  // __syncthreads inside the sum above orders the xval writes
    for (int v = threadIdx.x; v < V; v += kAxT) primal_node(B, I, H, lab, irr, true, v, porog, ps);
    const double lp = block_sum<kAxT>(ps.lp, sred);
    const double dual_neg = block_sum<kAxT>(ps.dual_neg, sred);
    const double fsum = block_sum<kAxT>(ps.fsum, sred);
    const long long maxr = block_max_ll<kAxT>(ps.maxr, sredl);
    const long long viol = block_sum_ll<kAxT>(ps.viol, sredl);
    if (threadIdx.x == 0) {
        const double dmin = __longlong_as_double((long long)B.dmin_bits[b]);
        B.max_rank[b] = (int32_t)maxr;
        B.deg_viol[b] = (int32_t)viol;
        B.dual[b] = dmin * (-fsum + dual_neg);
        B.status[b] = F2M_OK;
        B.lp[b] = lp;
    }
}

cudaError_t launch_axb(const Batch& B, const DevParams& P, cudaStream_t s, int64_t* launches) {
    if (B.n_inst <= 0) return cudaSuccess;
    k_axb<<<B.n_inst, kAxT, 0, s>>>(B, P);
    ++*launches;
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* host launchers                                                       */
/* ------------------------------------------------------------------ */
cudaError_t launch_prep(const Batch& B, cudaStream_t s, int64_t* launches) {
    k_prep<<<B.n_inst, kT, 0, s>>>(B);
    ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_knn(const Batch& B, int64_t* scan_scratch, cudaStream_t s, int64_t* launches) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(B.cellcnt, 0, sizeof(int64_t) * (B.n_total + 1), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(B.cellcur, 0, sizeof(int32_t) * B.n_total, s)) != cudaSuccess) return e;
    k_grid_count<<<B.n_chunks, kT, 0, s>>>(B);
    ++*launches;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_scan(B.cellcnt, B.cellstart, B.n_total, scan_scratch, s, launches)) != cudaSuccess) return e;
    k_grid_scatter<<<B.n_chunks, kT, 0, s>>>(B);
    k_cutoff<<<B.n_chunks, kT, 0, s>>>(B);
    *launches += 2;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (B.N <= 32) k_select<1><<<B.n_chunks, kT, 0, s>>>(B);
    else if (B.N <= 64) k_select<2><<<B.n_chunks, kT, 0, s>>>(B);
    else if (B.N <= 128) k_select<4><<<B.n_chunks, kT, 0, s>>>(B);
    else k_select<8><<<B.n_chunks, kT, 0, s>>>(B);
    ++*launches;
    return cudaGetLastError();
}

cudaError_t launch_graph(const Batch& B, int64_t* deg, int64_t* scan_scratch, cudaStream_t s,
                         int64_t* launches) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(B.rev, 0, sizeof(int32_t) * B.n_total, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(B.cursor, 0, sizeof(int32_t) * B.n_total, s)) != cudaSuccess) return e;
    k_graph_rev<<<B.n_chunks, kT, 0, s>>>(B);
    k_graph_deg<<<B.n_chunks, kT, 0, s>>>(B, deg);
    *launches += 2;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_scan(deg, B.row, B.n_total, scan_scratch, s, launches)) != cudaSuccess) return e;
    k_graph_fill<<<B.n_chunks, kT, 0, s>>>(B);
    k_graph_sort<<<B.n_chunks, kT, 0, s>>>(B);
    k_graph_mirror<<<B.n_chunks, kT, 0, s>>>(B);
    *launches += 3;
    return cudaGetLastError();
}

// Solver classes: instances are routed by point count to a (team width,
// teams per CTA) shape; every CTA is 1024 threads wide and takes the whole
// shared memory of an SM, split evenly among its teams.
struct SolveClass {
    int team, teams, max_n;
};
// Size classes: instances of at most max_n points go to the first class that
// takes them.  The bounds are tunable per process (solve_set_bounds); the
// defaults came from timing the batched workload on a B200.
static SolveClass kClasses[] = {
    {128, 8, 448}, {256, 4, 896}, {512, 2, 1792}, {1024, 1, 1 << 30}};
constexpr int kNumClasses = 4;

// Largest instance whose fixed shared-memory part fits a team of class c.
static int class_capacity(int c);

int solve_set_bounds(const int32_t* max_n) {
    int prev = 3;
    for (int c = 0; c < kNumClasses - 1; ++c) {
        if (max_n[c] <= prev || max_n[c] > class_capacity(c)) return -1;
        prev = max_n[c];
    }
    for (int c = 0; c < kNumClasses - 1; ++c) kClasses[c].max_n = max_n[c];
    return 0;
}
void solve_get_bounds(int32_t* max_n) {
    for (int c = 0; c < kNumClasses - 1; ++c) max_n[c] = kClasses[c].max_n;
}

int32_t solve_max_nodes() { return 10000; }
int solve_num_classes() { return kNumClasses; }
int solve_class_of(int32_t n) {
    for (int c = 0; c < kNumClasses; ++c)
        if (n <= kClasses[c].max_n) return c;
    return kNumClasses - 1;
}

// Shared memory of the solver CTAs.  A CTA does not take the whole opt-in
// limit: what it leaves stays L1 cache, which then holds the list slices
// that did not fit in shared memory (read from global memory every Jacobi
// step) and the slot records the partitions scan.  On the batched workload
// a 132 KB CTA (124 KB of L1) solves faster than a 227 KB one (about 5%).
// F2M_SOLVE_SMEM_KB overrides the target (read once per process; 0 = the
// whole opt-in limit; f2m_set_solver_smem_kb sets it at run time, as the
// autotuner does).  A launch whose largest instance needs more than the
// target for its fixed part (potentials, slice tables) takes what it needs.
constexpr int kSolveSmemKB = 132;
static size_t smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return (size_t)v;
}
static int g_smem_kb = -1;  // process-wide target (solve_set_smem_kb); -1: not read yet
int solve_get_smem_kb() {
    if (g_smem_kb < 0) {
        const char* e = getenv("F2M_SOLVE_SMEM_KB");
        g_smem_kb = e ? atoi(e) : kSolveSmemKB;
        if (g_smem_kb < 0) g_smem_kb = 0;
    }
    return g_smem_kb;
}
int solve_set_smem_kb(int kb) {
    if (kb < 0 || kb > 4096) return -1;
    g_smem_kb = kb;
    return 0;
}
static size_t smem_target() {
    const int kb = solve_get_smem_kb();
    const size_t optin = smem_optin();
    return (kb > 0 && (size_t)kb * 1024 < optin) ? (size_t)kb * 1024 : optin;
}
template <int TEAM, int TEAMS>
static size_t solve_static_smem() {
    return sizeof(double) * TEAMS * (TEAM / 32) * 2 + sizeof(int) * TEAMS * (TEAM / 32 + 5) + 64;
}
// dynamic bytes of a CTA of TEAMS teams out of `total` shared memory, and
// each team's share
static size_t dyn_of(size_t total, size_t stat) { return (total - stat) & ~(size_t)255; }
static int team_share(size_t dyn, int teams) { return (int)((dyn / teams) & ~(size_t)15); }

static int team_bytes_of(int team, int teams) {  // at the opt-in limit (class capacities)
    const size_t stat = sizeof(double) * teams * (team / 32) * 2 + sizeof(int) * teams * (team / 32 + 5) + 64;
    return team_share(dyn_of(smem_optin(), stat), teams);
}
static int class_capacity(int c) {
    const int tb = team_bytes_of(kClasses[c].team, kClasses[c].teams);
    int lo = 4, hi = 32767;  // node ids are 15-bit in the EF words
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (team_fixed_bytes(mid) <= (size_t)tb) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int TEAM, int TEAMS, bool R>
static cudaError_t launch_one(const Batch& B, const DevParams& P, const int32_t* items, int n_items,
                              int32_t* queue, int vcap, cudaStream_t s, int64_t* launches) {
    const size_t stat = solve_static_smem<TEAM, TEAMS>();
    const size_t optin = smem_optin();
    // the target, or what the largest instance's fixed part needs (with 4 KB
    // of slice cache per team), if more
    const size_t need = stat + 256 + (size_t)TEAMS * (team_fixed_bytes(vcap) + 16 + 4096);
    const size_t total = std::min(optin, std::max(smem_target(), need));
    const size_t dyn = dyn_of(total, stat);
    const int team_bytes = team_share(dyn, TEAMS);
    if (team_fixed_bytes(vcap) > (size_t)team_bytes) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(k_solve<TEAM, TEAMS, R>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve<TEAM, TEAMS, R>, TEAM * TEAMS, dyn);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid = sms * per_sm;
    const int need_ctas = (n_items + TEAMS - 1) / TEAMS;
    if (grid > need_ctas) grid = need_ctas;
    if ((e = cudaMemsetAsync(queue, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
    k_solve<TEAM, TEAMS, R><<<grid, TEAM * TEAMS, dyn, s>>>(B, P, items, n_items, queue, vcap, team_bytes);
    ++*launches;
    return cudaGetLastError();
}

template <bool R>
static cudaError_t launch_class(int c, const Batch& B, const DevParams& P, const int32_t* items,
                                int n_items, int32_t* queue, int vcap, cudaStream_t s,
                                int64_t* launches) {
    if (n_items <= 0) return cudaSuccess;
    switch (c) {
        case 0: return launch_one<128, 8, R>(B, P, items, n_items, queue, vcap, s, launches);
        case 1: return launch_one<256, 4, R>(B, P, items, n_items, queue, vcap, s, launches);
        case 2: return launch_one<512, 2, R>(B, P, items, n_items, queue, vcap, s, launches);
        default: return launch_one<1024, 1, R>(B, P, items, n_items, queue, vcap, s, launches);
    }
}

cudaError_t launch_solve_class(int c, const Batch& B, const DevParams& P, const int32_t* items,
                               int n_items, int32_t* queue, int vcap, cudaStream_t s,
                               int64_t* launches) {
    return launch_class<false>(c, B, P, items, n_items, queue, vcap, s, launches);
}
cudaError_t launch_refit_class(int c, const Batch& B, const DevParams& P, const int32_t* items,
                               int n_items, int32_t* queue, int vcap, cudaStream_t s,
                               int64_t* launches) {
    return launch_class<true>(c, B, P, items, n_items, queue, vcap, s, launches);
}

}  // namespace f2m
