// Internal declarations shared by the CUDA kernels (f2m_kernels.cu) and the
// host runtime (f2m_runtime.cu).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/f2m.h"

namespace f2m {

// Internal status: the instance needs the host comb solve (Ax=b) because at
// least one comb violates 2A+B=4 (comb_thread.cpp:180-195).
constexpr int32_t kNeedsHost = 100;
// Internal status between the solver and k_axb: the instance has irregular
// combs whose Ax=b the device solves next (comb_thread.cpp:272-304).
constexpr int32_t kNeedsAxb = 101;

// One CSR slot as the solver reads it: normalised cost D and neighbour id.
// `aux` holds the slot's original position in its node's list (the edge's
// rankDo at that endpoint, node.cpp:18).
struct __align__(16) Slot {
    double D;
    int32_t nbr;
    int32_t aux;
};

// Device-side constants of one solve call (the reference's constants).
struct DevParams {
    double error_B, porog, glob_tol, ef_thr, comb_thr;
    int32_t glob_K, glob_rounds, glob_inner;
    int32_t factor0, factor_step, factor_cap, max_rounds;
    int32_t fix_rounds, fix_factor, check_every, frozen_iters;
    int32_t ef_small_deg, ef_min;
    int64_t max_iters;
    int64_t spin_limit;     // grid barrier polls before giving up (whole-GPU solver)
};

// Pointers of one batched call.  Node g of instance b lives at index
// offs[b] + local id; slots of node g are [row[g], row[g+1]).
struct Batch {
    int32_t n_inst;
    int32_t N;              // neighbours selected per node (top_k, E_max)
    int32_t N_cut;          // top_k of the cut-off pass (FXY.hpp:77-78); normally N
    int32_t skip_dedup;     // points were de-duplicated on the host already
    int32_t cost_mode;      // f2m_cost_mode of the edge costs
    int32_t n_total;        // points over all instances (before de-duplication)
    const int64_t* offs;    // [n_inst+1]
    const double* X_in;     // raw coordinates [n_total]
    const double* Y_in;
    const int32_t* K_in;    // labels or nullptr (then label = local index + 1)
    double2* Pr;            // rounded, not compacted [n_total]
    double2* P;             // rounded, de-duplicated, compacted [n_total]
    int32_t* K;             // labels of P [n_total]
    int32_t* dup_of;        // [n_total] input index -> local id of the kept copy, -1 if kept
    int32_t* Vn;            // [n_inst]
    double* spn;            // size_per_node [n_inst]
    unsigned long long* dmin_bits;  // [n_inst] min edge cost (as ordered bits)
    int32_t* status;        // [n_inst]
    // cell grid per instance
    double* gx0;            // [n_inst]
    double* gy0;
    double* gh;
    int32_t* gnx;
    int32_t* gny;
    int32_t* pcell;         // [n_total] cell of each point
    int64_t* cellcnt;       // [n_total+1] points per cell (cells of b at offs[b] + cell)
    int64_t* cellstart;     // [n_total+1] exclusive scan of cellcnt
    int32_t* cellcur;       // [n_total]
    int32_t* sidx;          // [n_total] points sorted by cell (local ids)
    double2* spt;           // [n_total] their coordinates
    // kNN
    double* cut;            // [n_total]
    int32_t* stat;          // [n_total]
    int32_t* ntop;          // [n_total]
    int32_t* top_nbr;       // [n_total*N]
    double* top_cost;       // [n_total*N]
    int32_t* top_em;        // [n_total*N]
    int32_t* top_oth;       // [n_total*N]
    // graph
    int32_t* rev;           // [n_total]
    int32_t* cursor;        // [n_total]
    uint8_t* tdup;          // [n_total * N] the top entry's neighbour also keeps this node
    int64_t* row;           // [n_total+1]
    int32_t* s_nbr;         // [S]
    double* s_cost;         // [S] raw cost Do
    int32_t* s_em;          // [S]
    int32_t* s_oth;         // [S]
    Slot* slot;             // [S]
    uint16_t* perm;         // [S] per-node list order (local positions)
    Slot* pslot;            // [S] the slots in list order: pslot[r+k] = slot[r + perm[r+k]]
    int32_t* mirror;        // [S] position of the same edge in the neighbour's list
    double* efD;            // [S] active-set arena (update_EF copies): D
    uint16_t* efN;          // [S] active-set arena: neighbour
    uint8_t* xcode;         // [S] 0, 1 (= 1/2), 2 (= 1), 3 (= xval: an Ax=b solution)
    float* xval;            // [S] x of the B edges of combs solved by Ax=b on the device
    int32_t* clab;          // [n_total] comb root of each node (INT_MAX outside combs), for k_axb
    int32_t* cirr;          // [n_total] 1 at the root of an irregular comb, for k_axb
    double* selD;           // [S] SELL-32 slices that do not fit in shared memory: D
    uint16_t* selW;         // [S] ... neighbour word; instance b owns sel_stride * offs[b] ..
    int64_t sel_stride;     //     sel_stride * offs[b+1] (S / n_total entries per point)
    int64_t S_cap;
    // per-node state kept between the solve and the host comb check
    double* F;              // [n_total] potentials
    int32_t* efcnt;         // [n_total] EF list length (cuda_EF_NodesStat)
    int32_t* ccnt;          // [n_total] comb prefix length (cuda_COMB_NodesStat)
    const double* shift;    // [n_total] repair shift per node (k_refit input; 0 = none)
    const double* F0;       // [n_total] starting potentials (warm start), or null for F = 0
    // per-instance results
    double* lp;
    int32_t* n_edges;
    int32_t* n_combs;
    int32_t* n_irr;
    int32_t* max_rank;
    int32_t* deg_viol;
    int64_t* iters;
    int64_t* work_nodes;    // sum over Jacobi iterations of V
    int64_t* work_slots;    // sum over Jacobi iterations of active slots
    int64_t* work_pad;      // sum over Jacobi iterations of the entries swept incl. SELL padding
    int32_t* checks;
    double* max_grad;
    double* dual;
    // work lists
    const int32_t* chunk_inst;  // node-parallel work items
    const int32_t* chunk_start;
    int32_t n_chunks;
    const int32_t* order;       // instances to run, largest first
    int32_t n_items;            // entries of `order`
    int32_t* queue;             // persistent-kernel work counter
};

// Global state of the grid-wide solver for one large instance (f2m_grid.cu).
struct GridState {
    double* Ha;             // [V] H = F/2, two buffers
    double* Hb;
    int32_t* efc;           // [V] EF list length of each node
    double* gD;             // [S] EF lists at their nodes' slot positions (D)
    uint32_t* gW;           // [S] (neighbour | 1<<31 when it is the lower id)
    int32_t* scratch;       // [2V] comb prefix lengths + labels
    int32_t* irr;           // [V]
    unsigned* bar;          // [2] grid barrier: arrivals, generation
    int32_t* err;           // [1] set when a barrier timed out
    unsigned long long* axb_used;  // [2] slice-arena doubles handed to Ax=b systems, comb members listed
    double* part;           // [2*grid] partial reductions
    long long* partl;       // [2*grid]
    int32_t* own;           // [V] nodes in ownership order (CTA c owns a contiguous run)
    int32_t* owner;         // [V] CTA owning each node
    int32_t* rd;            // [V] nonzero: some other CTA's halo reads the node
    unsigned* prog;         // [kGridMaxCtas] halo blocks each CTA has completed (neighbour waits)
    unsigned* nbm;          // [kGridMaxCtas * kGridNbWords] bit d of row c: CTA d reads c's nodes
    unsigned long long* okey;   // [V] ownership sort keys (Morton code << 32 | node)
    unsigned long long* okey2;  // [V]
    void* otmp;             // radix-sort scratch
    size_t otmp_bytes;
};
constexpr int kGridMaxCtas = 2 * 160;
constexpr int kGridNbWords = kGridMaxCtas / 32;  // words of one neighbour-mask row

// Host-side launchers (f2m_kernels.cu, f2m_grid.cu).
cudaError_t launch_solve_grid(const Batch& B, const DevParams& P, const GridState& G, int b, int V,
                              bool refit, cudaStream_t s, int64_t* launches);
// Ownership order of the grid solver's nodes: Morton order of the points
// (point_of[v] = point of node v, or nullptr when node = point), or the node
// order itself when the instance has no coordinates (spatial = false).
cudaError_t launch_grid_order(const Batch& B, const GridState& G, int b, int V, const int32_t* point_of,
                              bool spatial, cudaStream_t s, int64_t* launches);
size_t grid_order_temp_bytes(int64_t n);

// Buffers of the device edge order of one instance (single-instance calls).
struct EdgeSort {
    unsigned long long* k1;  // [S] keys
    unsigned long long* k2;  // [S]
    uint32_t* v1;            // [S] slot offsets within the instance
    uint32_t* v2;            // [S]
    void* tmp;               // radix-sort scratch
    size_t tmp_bytes;
    void* xout;              // [S * 20 bytes] the exported edge arrays (EdgeExport)
};
size_t edge_order_temp_bytes(int64_t S);
// The result arrays of one solved instance in the reference's edge order,
// written on the device: internal ids of the lower/higher-id endpoint, of
// the lower/higher-label endpoint, raw and normalised cost, primal x.
struct EdgeExport {
    int32_t *ev1, *ev2, *el1, *el2;
    double *Do, *D, *x;
};
EdgeExport edge_export_view(void* xout, int64_t E);
cudaError_t launch_export_edges(const Batch& B, int b, int V, const uint32_t* order, int64_t E,
                                const EdgeExport& X, cudaStream_t s, int64_t* launches);
// The reference's edge order (ascending cost, then emitter, then partner:
// graph_tour.hpp:28-98) of instance b's edges, each as the offset of its slot
// in the lower-id endpoint's list (within the instance's slots); the first
// S/2 entries of *order are the edges in order.
cudaError_t launch_edge_order(const Batch& B, int b, int V, int64_t S, const EdgeSort& E, const uint32_t** order,
                              cudaStream_t s, int64_t* launches);
// FP64 pipe throughput probe (f2m_probe.cu): kind 0 DADD chains, kind 1 DSETP.
cudaError_t launch_fp64_probe(int kind, int blocks, int iters, double* out, cudaStream_t s);
double fp64_probe_ops(int kind, int blocks, int iters);
cudaError_t launch_partition_check(int n_cases, unsigned long long seed, unsigned long long* bad,
                                   cudaStream_t s);
cudaError_t launch_prep(const Batch& B, cudaStream_t s, int64_t* launches);
// Ax=b of the irregular combs and the primal of every instance the solver
// left with status kNeedsAxb (one CTA per instance of the batch).
cudaError_t launch_axb(const Batch& B, const DevParams& P, cudaStream_t s, int64_t* launches);
cudaError_t launch_knn(const Batch& B, int64_t* scan_scratch, cudaStream_t s, int64_t* launches);
cudaError_t launch_graph(const Batch& B, int64_t* deg_scratch, int64_t* scan_scratch,
                         cudaStream_t s, int64_t* launches);
// Persistent solver over items[0..n_items) of size class c (largest first);
// queue is a device counter.  REFIT variant: F += shift, frozen iterations,
// run_fix (graph_cuda_comb.hpp:542-574).
cudaError_t launch_solve_class(int c, const Batch& B, const DevParams& P, const int32_t* items,
                               int n_items, int32_t* queue, int vcap, cudaStream_t s,
                               int64_t* launches);
cudaError_t launch_refit_class(int c, const Batch& B, const DevParams& P, const int32_t* items,
                               int n_items, int32_t* queue, int vcap, cudaStream_t s,
                               int64_t* launches);
int solve_num_classes();
int solve_class_of(int32_t n);
int solve_set_bounds(const int32_t* max_n);  // 3 increasing bounds; -1 if rejected
void solve_get_bounds(int32_t* max_n);
int solve_set_smem_kb(int kb);                // shared-memory target of a solver CTA (0 = all)
int solve_get_smem_kb();
// Smoothed-bound batch (f2m_smooth.cu).  Node g of instance b is offs[b] +
// local id; neighbour ids in nbr are local; slots are global (row).
struct SmoothBatch {
    int32_t n_inst = 0, N = 0;
    int64_t n_total = 0;
    const int64_t* offs = nullptr;
    const float* x = nullptr;
    const float* y = nullptr;
    unsigned long long* top = nullptr;  // [n_total * N] (cost bits << 32 | local index)
    int32_t* rdeg = nullptr;            // [n_total]
    int32_t* tcur = nullptr;            // [n_total]
    int64_t* tcap = nullptr;            // [n_total + 1] temporary list offsets
    int32_t* tnbr = nullptr;            // [2 * n_total * N]
    int64_t* deg = nullptr;             // [n_total] scan input
    int64_t* row = nullptr;             // [n_total + 1]
    int32_t* nbr = nullptr;             // [S]
    int64_t* mirror = nullptr;          // [S] slot of the same edge in the neighbour's list
    float* c = nullptr;                 // [S]
    double tau = 0, omega = 0;
    int32_t iters = 0, newton_max = 0, ckpt = 1, n_ck = 1;
    double* L = nullptr;                // [n_inst]
    const double* dL = nullptr;         // [n_inst] upstream gradient
    int32_t solver = 0;                 // 1: one CTA per instance, 2: one launch per step
    double* ck = nullptr;               // [n_total * n_ck] checkpoints of u
    double* ua = nullptr;               // [n_total] potentials (per-step path)
    double* ub = nullptr;               // [n_total]
    double* Lp = nullptr;               // [n_total] per-node terms of L (per-step path)
    double* segu = nullptr;             // [n_total * ckpt] recomputed iterates
    double* segs = nullptr;             // [n_total * ckpt] their roots
    double* lam = nullptr;              // [n_total]
    double* lam2 = nullptr;             // [n_total]
    double* q = nullptr;                // [S]
    double* gc = nullptr;               // [S] dL/dc accumulated per slot
    float* gx = nullptr;                // [n_total]
    float* gy = nullptr;                // [n_total]
    int32_t* queue = nullptr;
    unsigned long long* work = nullptr; // [1] logistic terms evaluated by the persistent kernel
};
cudaError_t launch_smooth_graph(SmoothBatch& S, int64_t* scan_scratch, cudaStream_t s,
                                int64_t* launches);
cudaError_t launch_smooth_bound(SmoothBatch& S, int32_t max_v, bool grad, cudaStream_t s,
                                int64_t* launches);
cudaError_t launch_smooth_steps(SmoothBatch& S, bool grad, cudaStream_t s, int64_t* launches);
int32_t smooth_max_nodes();
// Rate probe of the smoothed bound's logistic term (one exp and two
// divisions, the Newton sums' unit of work), and its work per launch.
cudaError_t launch_logit_probe(int blocks, int iters, double* out, cudaStream_t s);
double logit_probe_terms(int blocks, int iters);

cudaError_t launch_scan(const int64_t* in, int64_t* out, int64_t n, int64_t* scratch,
                        cudaStream_t s, int64_t* launches);
// Stable LSD radix sort of 64-bit keys (values optional) by bits [begin_bit,
// end_bit) (f2m_sort.cu); the result ends in keys/vals or kbuf/vbuf (*kres, *vres).
size_t radix_sort_temp_bytes(int64_t n);
cudaError_t radix_sort(unsigned long long* keys, unsigned long long* kbuf, uint32_t* vals, uint32_t* vbuf,
                       int64_t n, int begin_bit, int end_bit, void* temp, size_t temp_bytes, cudaStream_t s,
                       int64_t* launches, unsigned long long** kres, uint32_t** vres);
int64_t scan_scratch_elems(int64_t n);
int32_t solve_max_nodes();

}  // namespace f2m
