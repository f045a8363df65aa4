/*
 * f2m_b200 -- C ABI of the B200-native F2M (fractional 2-matching) solver.
 *
 * Plain pointers and sizes only; no torch or CUDA types cross this boundary.
 * Every entry point returns an f2m_status; nothing calls exit().  Host arrays
 * belong to the caller; device buffers belong to the context.  One context
 * per host thread (a context owns one CUDA stream on one device).
 *
 * Each entry point names the reference interface it replaces
 * (aav-antonov/F2M, paths relative to that project).
 */
#ifndef F2M_B200_H
#define F2M_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum f2m_status {
    F2M_OK = 0,
    F2M_ERR_INPUT = 1,          /* bad file/arguments (reference: exit(0), FXY.hpp:221-226) */
    F2M_ERR_CAPACITY = 2,       /* instance exceeds a compiled limit */
    F2M_ERR_NOT_CONVERGED = 3,  /* "ERROR: Optimal Solution not Found" (graph_tour.hpp:236-239) */
    F2M_ERR_CUDA = 4,           /* a CUDA call failed (reference: cudaCheckErrors exit(1)) */
    F2M_ERR_NO_DEVICE = 5       /* no CUDA device / the kernels are not loadable */
} f2m_status;

typedef enum f2m_cost_mode {
    F2M_COST_REF_EUCLID = 0,    /* raw FP64 sqrt(dx^2+dy^2), as FXY.hpp:382 */
    F2M_COST_NINT = 1           /* TSPLIB EUC_2D nint(sqrt(dx^2+dy^2)) as the edge cost */
} f2m_cost_mode;

/* The reference's hard-coded constants, now parameters (defaults equal the
 * reference; graph_cuda.cu:56-57,178-186,214-216,370-394,
 * graph_cuda_partition.hpp:50,62, graph_cuda_comb.hpp:420,556). */
typedef struct f2m_params {
    double error_B;        /* 1e-7: convergence on max|grad| */
    double error_B_comb;   /* 1e2: half-edge band = error_B * error_B_comb */
    int32_t glob_K;        /* 5 */
    int32_t glob_rounds;   /* 200 */
    int32_t glob_inner;    /* 50 */
    double glob_tol;       /* 0.01 */
    int32_t factor0;       /* 100 */
    int32_t factor_step;   /* 300 */
    int32_t factor_cap;    /* 5000 */
    int32_t max_rounds;    /* 10000 */
    int32_t fix_rounds;    /* 100 */
    int32_t fix_factor;    /* 500 */
    int32_t check_every;   /* 50 */
    int32_t frozen_iters;  /* 20 */
    double ef_thr;         /* 1.0 */
    int32_t ef_small_deg;  /* 10 */
    int32_t ef_min;        /* 3 */
    double comb_thr;       /* 0.25 */
    double shift0;         /* 0.5 */
    double shift_max;      /* 32 */
    int64_t max_iters;     /* safety cap on Jacobi iterations per solve (not in the reference) */
    int32_t cost_mode;     /* f2m_cost_mode */
    int32_t solver;        /* 0 auto: a team per instance, the whole GPU above 10,000 points;
                              2: the whole-GPU solver for a single instance of any size */
    int64_t grid_spin_limit; /* the whole-GPU solver's grid barrier is a bounded wait: after
                              this many polls a CTA gives up, every CTA leaves the solve and
                              the call fails with F2M_ERR_CUDA (default 2^26, seconds of
                              waiting; the GPU context stays usable).  Not in the reference. */
} f2m_params;

typedef struct f2m_ctx f2m_ctx;

/* Fill *p with the reference's constants. */
void f2m_default_params(f2m_params* p);

/* Create a context on `device`.  Replaces the implicit CUDA context set-up of
 * graph_c::init_cuda (graph_cuda_init.hpp:102-193). */
f2m_status f2m_create(f2m_ctx** ctx, int device);
void f2m_destroy(f2m_ctx* ctx);
/* Last error message of this context (never NULL). */
const char* f2m_last_error(const f2m_ctx* ctx);
/* Kernels launched by this context since creation (diagnostics). */
int64_t f2m_kernel_launches(const f2m_ctx* ctx);

/* ------------------------------------------------------------------ */
/* Batched solve: many independent instances in one call.               */
/* The reference solves one file per process (RUN.cpp:12-31); this entry  */
/* is its batched replacement: per instance it runs FXY (FXY.hpp:23-144), */
/* the union-of-kNN graph build (graph_tour.hpp:28-98), the descent       */
/* (graph_cuda.cu:163-430), comb extraction (graph_cuda_comb.hpp:415-475) */
/* and the host comb check + primal (graph_cuda_comb.hpp:121-147,         */
/* graph_cuda.cu:135-147) and returns the report's Optimal Value.         */
/* ------------------------------------------------------------------ */
typedef struct f2m_batch_out {
    double* lp;            /* [n_inst] Optimal Value (sum x*Do); NaN when not found */
    int32_t* status;       /* [n_inst] f2m_status per instance */
    int32_t* n_nodes;      /* optional [n_inst]: nodes after de-duplication */
    int32_t* n_edges;      /* optional [n_inst] */
    int32_t* n_combs;      /* optional [n_inst] */
    int32_t* max_rank;     /* optional [n_inst] "MAX edge rank" */
    int64_t* iterations;   /* optional [n_inst] Jacobi iterations */
    int32_t* n_irregular;  /* optional [n_inst] combs failing 2A+B=4, whose x comes from Ax=b
                              (comb_thread.cpp:272-304) */
} f2m_batch_out;

/* Host arrays: offs[n_inst+1] (int64) into x[], y[] (FP64 coordinates,
 * rounded to 1e-3 and de-duplicated as get_KXY does, FXY.hpp:252-267). */
f2m_status f2m_solve_batch(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs,
                           const double* x, const double* y, int32_t top_k,
                           const f2m_params* params, f2m_batch_out* out);

/* Same, with offs/x/y already resident in device memory (d_ pointers); the
 * host copy h_offs plans the launch.  Outputs are device pointers too (lp,
 * status required; others optional), written on the context stream; the
 * call returns once they are enqueued (f2m_sync() waits for them). */
f2m_status f2m_solve_batch_device(f2m_ctx* ctx, int32_t n_inst, const int64_t* h_offs,
                                  const int64_t* d_offs, const double* d_x, const double* d_y,
                                  int32_t top_k, const f2m_params* params,
                                  f2m_batch_out* d_out);
f2m_status f2m_sync(f2m_ctx* ctx);

/* Work counters of the last batched call, summed over its instances. */
typedef struct f2m_work {
    int64_t node_iters;    /* sum over Jacobi iterations of the nodes updated */
    int64_t slot_iters;    /* sum over Jacobi iterations of the active slots read */
    int64_t slots;         /* CSR slots built (2 x edges) */
    int64_t points;        /* points after de-duplication */
    int64_t pad_iters;     /* sum over Jacobi iterations of the list entries the warps sweep,
                              padding of the 32-node slices included */
    int64_t lane_iters;    /* sum over Jacobi iterations of the lanes updating a node
                              (32 per slice of 32 nodes) */
} f2m_work;

/* Device time (CUDA events on the context stream) of the phases of the last
 * batched call: ms[0] rounding/de-duplication, ms[1] kNN, ms[2] graph build,
 * ms[3] the persistent solver (descent, combs, primal).  Diagnostics; no
 * reference counterpart (the reference prints gettimeofday phase times,
 * graph_cuda_define.hpp:29-34). */
f2m_status f2m_phase_times(f2m_ctx* ctx, float* ms, f2m_work* work);

/* Measured FP64 pipe rate of this context's GPU in FP64 lane operations per
 * second (diagnostics; no reference counterpart).  The dual descent issues
 * FP64 additions and compares, so this rate, not HBM bandwidth, is the
 * roofline of its persistent solver.  kind 0: independent DADD chains;
 * kind 1: DSETP compares (one DADD per eight); kind 2: logistic terms of the
 * smoothed bound per second (one FP64 exp and two divisions each, four
 * independent sums per thread), the roofline of its persistent kernel.
 * Best of `repeats` timed launches (CUDA events) over every SM at full
 * occupancy. */
f2m_status f2m_fp64_rate(f2m_ctx* ctx, int32_t kind, int32_t repeats, double* lane_ops_per_s);

/* Self-check of the warp-cooperative list partition (diagnostics; no
 * reference counterpart): runs n_cases seeded lists (0-128 entries, many
 * ties, thresholds that need the raise-by-one loop of qpart_ptr_EF,
 * graph_cuda_partition.hpp:27-54) through the serial partition and the warp
 * partition on the device and returns how many differ in order or count
 * (0 when they agree). */
f2m_status f2m_partition_selfcheck(f2m_ctx* ctx, int32_t n_cases, uint64_t seed, int64_t* mismatches);

/* Work of the last smoothed-bound call on this context (diagnostics; no
 * reference counterpart): the logistic terms (exp-based evaluations: Newton
 * sums, softplus, sigma and its derivative) its persistent one-CTA-per-
 * instance kernel evaluated, and that kernel's CUDA-event time in ms.
 * terms is -1 when the call took the one-launch-per-step path. */
f2m_status f2m_smooth_work(const f2m_ctx* ctx, int64_t* terms, float* kernel_ms);

/* ------------------------------------------------------------------ */
/* Single instance with full results (the F2M.h graph API).             */
/* ------------------------------------------------------------------ */
typedef struct f2m_result f2m_result;

/* Points in (labels optional: NULL = 1..n).  Node ids follow the
 * de-duplicated input order.  Replaces graph(file,N) + graph_c + RUN()
 * (F2M.h:181,320,175) for in-memory inputs. */
f2m_status f2m_solve_points(f2m_ctx* ctx, const double* x, const double* y,
                            const int32_t* labels, int32_t n, int32_t top_k,
                            const f2m_params* params, f2m_result** out);
/* Resume from stored potentials (no counterpart in the reference, which
 * always starts from F = 0, graph_cuda_init.hpp:183): as f2m_solve_points,
 * with the descent started from F0 (n_F0 values in the node order of a
 * result for the same points and top_k, f2m_result_nodes) and run with the
 * schedule the reference uses after a repair shift (run_fix,
 * graph_cuda.cu:204-226: active-set rounds until max|grad| < error_B), so
 * good potentials converge in far fewer iterations.  F2M_ERR_INPUT if n_F0
 * is not the node count. */
f2m_status f2m_solve_points_from(f2m_ctx* ctx, const double* x, const double* y,
                                 const int32_t* labels, int32_t n, int32_t top_k,
                                 const double* F0, int32_t n_F0, const f2m_params* params,
                                 f2m_result** out);
/* graph_c(graph*) + graph::RUN() (F2M.h:175,320) on a graph the caller
 * built: n_edges edges between node indices v1/v2 (either order) in the
 * reference's edge order (graph::E, ascending Do, graph_tour.hpp:28-98),
 * each node's list in that order (graph_cuda_init.hpp:42-63), normalised
 * costs D (Do / d_min) and raw costs Do; labels (n_nodes, NULL = 1..n) name
 * the nodes in the outputs.  Solves on the device and runs the host comb
 * stage, as f2m_solve_points. */
f2m_status f2m_solve_graph(f2m_ctx* ctx, int32_t n_nodes, int32_t n_edges, const int32_t* v1,
                           const int32_t* v2, const double* D, const double* Do,
                           const int32_t* labels, const f2m_params* params, f2m_result** out);
/* The kNN graph alone: FXY's candidate kNN (FXY.hpp:23-144, 313-534) and the
 * greedy union of graph::graph (graph_tour.hpp:28-98), without solving.  The
 * result carries the edges in the reference's edge order
 * (f2m_result_edges: endpoints, labels, Do and D = Do/d_min; x is 0), the
 * nodes (F is 0), status F2M_OK and an LP value of NaN. */
f2m_status f2m_knn(f2m_ctx* ctx, const double* x, const double* y, const int32_t* labels,
                   int32_t n, int32_t top_k, f2m_result** out);


/* `F2M.solver.exe file N` (RUN.cpp:12-31): parse the TSPLIB file, solve, and
 * when write_files != 0 write <file>.topN.F2M_report / .F2M_solution
 * (graph_tour.hpp:186-241), .DM (FXY.hpp:146-165) and <file>_duplicates
 * (FXY.hpp:168-183).  Node ids follow the reference's graph order
 * (graph_tour.hpp:95-97). */
f2m_status f2m_solve_file(f2m_ctx* ctx, const char* path, int32_t top_k,
                          const f2m_params* params, int32_t write_files,
                          f2m_result** out);

/* Allocation-free solve of one instance (no counterpart in the reference).
 * For callers that cannot allocate device memory while they run -- a host
 * application that owns the GPU through its own memory pool, or a
 * latency-bound loop that cannot afford cudaMalloc's synchronisation -- this
 * entry point allocates nothing: its scratch is one fixed 12 MiB array in
 * device memory that every GPU loading the library holds until exit.
 * Limits: n <= 2048 points, top_k <= 24, reference cost mode; larger inputs
 * return F2M_ERR_CAPACITY.  It always runs the per-instance team solver:
 * params->solver == 2 (the whole-GPU solver) returns F2M_ERR_INPUT.  d_x, d_y (n coordinates), d_lp and d_status (one
 * value each) are device pointers; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  The call only enqueues work on that stream and
 * returns; the results are ready once the stream is synchronised.  It runs
 * the device stages only: an instance whose combs need the host Ax=b stage
 * gets status F2M_ERR_CAPACITY (solve it with f2m_solve_points).
 * The first call on a device looks up the array's device address there
 * (cudaGetSymbolAddress) and, under CUDA's default lazy module loading, is
 * also the moment the array and the solver's kernels are loaded onto that
 * device -- the one time this entry point causes device allocations.  Make
 * one warm-up call on each device during your own set-up, before your pool
 * takes the GPU and before any stream capture (or set
 * CUDA_MODULE_LOADING=EAGER to load at library load).  A device reset
 * (cudaDeviceReset) makes the saved address stale: do not reset the device
 * between calls.
 * All calls share the one array and it keeps the previous call's contents
 * (the solver clears what must start at zero), so calls that overlap on the
 * GPU -- on different streams, or from different host threads -- race. */
f2m_status f2m_solve_points_noalloc(const double* d_x, const double* d_y, int32_t n,
                                    int32_t top_k, const f2m_params* params, double* d_lp,
                                    int32_t* d_status, void* stream);

void f2m_result_free(f2m_result* r);
int32_t f2m_result_status(const f2m_result* r);
int32_t f2m_result_n_nodes(const f2m_result* r);
int32_t f2m_result_n_edges(const f2m_result* r);
/* graph::OVAL and graph::MAXrankDo (graph_tour.hpp:165-184) */
double f2m_result_lp(const f2m_result* r);
int32_t f2m_result_max_rank(const f2m_result* r);
/* Seconds spent in the solve proper (the report's "Time:", graph_cuda.cu:51,131). */
double f2m_result_seconds(const f2m_result* r);
/* Edges in the graph's edge order: internal node ids (v1<v2), TSPLIB labels
 * of the lower/higher-label endpoint, raw cost Do, normalised cost D and the
 * primal value x (graph::X, F2M.h:161; 0 where absent).  Any pointer may be
 * NULL. */
void f2m_result_edges(const f2m_result* r, int32_t* v1, int32_t* v2, int32_t* lab1,
                      int32_t* lab2, double* Do, double* D, double* x);
/* Per node: TSPLIB label, dual potential F (graph::F, F2M.h:146). */
void f2m_result_nodes(const f2m_result* r, int32_t* label, double* F);

typedef struct f2m_stats {
    int64_t iterations;    /* all Jacobi iterations */
    int32_t checks;        /* check_OPT calls */
    int32_t n_combs;
    int32_t irr_a;         /* combs failing 2A+B=4 at the final check */
    int32_t irr_b;         /* combs whose Ax=b did not converge */
    int32_t repair_steps;
    int32_t degree_violations; /* nodes with |sum x - 2| >= 1e-2 (graph_tour.hpp:142-163) */
    double max_grad;       /* max|grad| at the last check */
    double d_min;
    double dual_value;     /* FP64 dual bound 2*sum(u) + sum(min(0,d)) with u=-F/2 */
} f2m_stats;
void f2m_result_stats(const f2m_result* r, f2m_stats* s);

/* ------------------------------------------------------------------------
 * Entropically smoothed F2M dual bound and its gradient.  No counterpart in
 * the reference (it solves the LP only); this is the differentiable
 * extension of the same method.  Per instance: the graph is the union of
 * each point's top_k nearest neighbours by FP32 Euclidean distance (ties by
 * index, no rounding or de-duplication); with z_e = (u_a + u_b - c_e)/tau,
 *   L(u) = 2 sum_v u_v - tau sum_e softplus(z_e)
 * bounds the entropy-smoothed fractional 2-matching LP from below for every
 * u.  u comes from `iters` damped Jacobi coordinate-ascent steps from 0; the
 * gradient is the exact adjoint of that computation (iterates recomputed
 * from checkpoints every `checkpoint` steps), chained through c_e = |p_a-p_b|.
 * At a stationary u, dL/dc_e = sigmoid(z_e), the smoothed x_e. */
typedef struct f2m_smooth_params {
    double tau;          /* temperature (> 0) */
    int32_t iters;       /* Jacobi steps (>= 0) */
    double damping;      /* omega in (0, 1]: u <- (1-omega) u + omega root */
    int32_t newton_max;  /* Newton steps per node root */
    int32_t checkpoint;  /* steps between stored iterates in the backward pass */
    int32_t solver;      /* 0 auto, 1 one CTA per instance, 2 one launch per step
                            (a warp per node over the whole batch) */
} f2m_smooth_params;
void f2m_default_smooth_params(f2m_smooth_params* p); /* 1e-3, 100, 0.5, 60, 16, 0 */

/* Forward: L[b] for each instance (offs has n_inst+1 entries into x/y, host
 * arrays; 3 <= top_k <= 64; at most f2m_smooth_max_nodes() points each). */
f2m_status f2m_smoothed_bound_fwd(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs,
                                  const float* x, const float* y, int32_t top_k,
                                  const f2m_smooth_params* p, double* L);
/* Backward: recomputes the forward pass, writes L and the gradient of
 * sum_b dL[b] * L[b] with respect to the coordinates (dL null = all ones). */
f2m_status f2m_smoothed_bound_bwd(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs,
                                  const float* x, const float* y, int32_t top_k,
                                  const f2m_smooth_params* p, const double* dL, double* L,
                                  float* dL_dx, float* dL_dy);
/* Backward with the edge-cost gradient exported: as f2m_smoothed_bound_bwd,
 * plus the graph's edges and dL/dc_e, the derivative of sum_b dL[b] * L[b]
 * with respect to each edge cost (at a stationary u, dL[b] * sigmoid(z_e):
 * the smoothed x_e, whose sums over each point's edges are 2).  Edges are
 * listed once, the lower global point index first (edge_a < edge_b, indices
 * into x/y), in the order of the lower endpoint's list; cost is c_e in FP32.
 * *n_edges receives the edge count; arrays of n_total * top_k entries always
 * suffice (each point adds at most top_k edges to the union), and a smaller
 * edge_cap returns F2M_ERR_CAPACITY with the count set.  Any edge array may
 * be NULL. */
f2m_status f2m_smoothed_bound_bwd_edges(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs,
                                        const float* x, const float* y, int32_t top_k,
                                        const f2m_smooth_params* p, const double* dL, double* L,
                                        float* dL_dx, float* dL_dy, int64_t edge_cap,
                                        int64_t* n_edges, int32_t* edge_a, int32_t* edge_b,
                                        float* cost, double* dL_dc);
int32_t f2m_smooth_max_nodes(void);

/* Size classes of the batched solver (no reference counterpart): an instance
 * of at most max_nodes[0] points runs on a 128-thread team (8 per CTA), up to
 * max_nodes[1] on 256 (4 per CTA), up to max_nodes[2] on 512 (2 per CTA),
 * larger ones on 1024 threads.  The potentials do not depend on the classes
 * (the LP value only through the order of its team-wide sum, ~1e-16
 * relative); f2m_b200/autotune.py times candidate bounds on a workload.  The
 * bounds are process-wide: set them before solving.  F2M_ERR_INPUT if not
 * increasing or a class's shared memory cannot hold an instance that size. */
f2m_status f2m_set_class_bounds(const int32_t* max_nodes); /* 3 values */
void f2m_get_class_bounds(int32_t* max_nodes);
/* Shared memory a CTA of the batched solver takes, in KB (no reference
 * counterpart; process-wide, like the class bounds).  What a CTA leaves
 * stays L1 cache, which holds the list slices that did not fit in shared
 * memory; 0 takes the whole opt-in limit.  A launch whose largest instance
 * needs more for its fixed part takes what it needs.  Default 132 (or
 * F2M_SOLVE_SMEM_KB); f2m_b200/autotune.py tunes it with the bounds. */
f2m_status f2m_set_solver_smem_kb(int32_t kb);
int32_t f2m_get_solver_smem_kb(void);

#ifdef __cplusplus
}
#endif
#endif
