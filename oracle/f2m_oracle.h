/*
 * CPU oracle for the F2M hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++17 FP64 restatement of the reference solver (aav-antonov/F2M):
 * TSPLIB parse, FXY kNN candidates, the greedy union-of-kNN graph build, the
 * dual descent schedule with its per-node partitions, comb extraction, the
 * host comb check (E/V/comb threads + Ax_b) and the primal/report stage.
 * Every function in f2m_oracle.cpp cites the reference file:line it follows.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library; the product path (f2m_b200) never calls it.
 */
#ifndef F2M_ORACLE_H
#define F2M_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (same values as include/f2m.h) */
#define ORC_OK 0
#define ORC_ERR_INPUT 1
#define ORC_ERR_CAPACITY 2
#define ORC_ERR_NOT_CONVERGED 3

/* cost modes */
#define ORC_COST_REF_EUCLID 0 /* raw FP64 sqrt(dx^2+dy^2) as the reference */
#define ORC_COST_NINT 1       /* TSPLIB EUC_2D nint(sqrt(dx^2+dy^2)) */

/* internal node-id orders */
#define ORC_ID_REF 0 /* libstdc++ unordered_map iteration order, as graph_tour.hpp:97 */
#define ORC_ID_FXY 1 /* deduplicated input order */

/* kNN formulations (identical output; literal is O(V^2) memory-heavy) */
#define ORC_KNN_LITERAL 0 /* stat/fill/stable-sort/cut + greedy union loop */
#define ORC_KNN_TOPN 1    /* per-node first-N by (d, emitter, partner) */

typedef struct orc_result orc_result;

typedef struct orc_stats {
    int64_t iters_glob;     /* Jacobi iterations in block_GLOB */
    int64_t iters_ef;       /* Jacobi iterations in block_EF (start phase) */
    int64_t iters_repair;   /* iterations inside the repair loop */
    int32_t checks;         /* check_OPT calls */
    int32_t glob_rounds;    /* block_GLOB outer rounds */
    int32_t ef_rounds;      /* run_start outer rounds */
    int32_t n_combs;        /* combs at the final extraction */
    int32_t irr_a;          /* irregular combs (2A+B != 4) at the final check */
    int32_t irr_b;          /* combs whose Ax=b did not converge (final) */
    int32_t repair_steps;   /* shift/refit steps taken */
    int64_t ef_slots;       /* active slots after the last update_EF */
    double max_grad;        /* |max grad| at the last check_OPT */
    double d_min;           /* normalisation distance */
} orc_stats;

/* Solve from a TSPLIB file exactly as `F2M.solver.exe file N`.  When
 * write_files != 0 the .topN.F2M_report / .F2M_solution / .DM /
 * _duplicates files are written next to `path`. */
int orc_solve_file(const char* path, int top_k, int cost_mode, int id_order,
                   int knn_mode, int write_files, int threads, orc_result** out);

/* Solve from point arrays (labels K, coordinates X/Y as given; the 1e-3
 * rounding and de-duplication of get_KXY are applied). */
int orc_solve_points(const int32_t* K, const double* X, const double* Y,
                     int32_t n, int top_k, int cost_mode, int id_order,
                     int knn_mode, int threads, orc_result** out);

/* kNN + graph build only (no descent). */
int orc_build_graph(const int32_t* K, const double* X, const double* Y,
                    int32_t n, int top_k, int cost_mode, int id_order,
                    int knn_mode, orc_result** out);

/* Run the descent/comb/check pipeline on a graph given by edges
 * (internal ids v1<v2 in edge-id order, normalised costs D, raw Do).
 * node_label may be NULL (labels = ids). */
int orc_solve_graph(int32_t n_nodes, int32_t n_edges, const int32_t* ev1,
                    const int32_t* ev2, const double* D, const double* Do,
                    const int32_t* node_label, int threads, orc_result** out);

void orc_free(orc_result* r);
const char* orc_error(const orc_result* r);
int orc_status(const orc_result* r);
int32_t orc_num_nodes(const orc_result* r);
int32_t orc_num_edges(const orc_result* r);
/* edges in edge-id order: internal ids (v1<v2), labels of the endpoints,
 * raw cost Do and normalised cost D */
void orc_get_edges(const orc_result* r, int32_t* v1, int32_t* v2, int32_t* lab1,
                   int32_t* lab2, double* Do, double* D);
/* internal id -> TSPLIB label, and internal id -> deduplicated input index */
void orc_get_nodes(const orc_result* r, int32_t* label, int32_t* fxy_index);
void orc_get_F(const orc_result* r, double* F);
/* primal x per edge id (0 where the edge is not in the solution) */
void orc_get_x(const orc_result* r, double* x);
double orc_lp_value(const orc_result* r);
int32_t orc_max_rank(const orc_result* r);
void orc_get_stats(const orc_result* r, orc_stats* s);
/* comb structure of the final extraction (roots ascending): per comb node
 * count; node ids concatenated; returns number of combs */
int32_t orc_get_combs(const orc_result* r, int32_t* comb_size, int32_t* comb_nodes);
/* per-node A/B counts of the final extraction (device-side StatAB rule) */
void orc_get_statab(const orc_result* r, int32_t* A, int32_t* B);
/* FXY per-node cutoff radius (the stat pass), deduplicated input order */
int32_t orc_num_points(const orc_result* r);
void orc_get_cutoffs(const orc_result* r, double* cutoff, int32_t* stat);
double orc_size_per_node(const orc_result* r);

/* Batched CPU solve of many independent instances (instance-parallel over
 * `threads` OpenMP threads).  offs has n_inst+1 entries into X/Y.  Writes the
 * LP value and status per instance. Returns ORC_OK. */
int orc_solve_batch(int32_t n_inst, const int64_t* offs, const double* X,
                    const double* Y, int top_k, int cost_mode, int threads,
                    double* lp_out, int32_t* status_out, int64_t* iters_out);

/* Entropically smoothed F2M dual bound (f2m_smooth_oracle.cpp).  Graph of
 * the FP32 points: union of each point's top_k nearest (ties by index), lists
 * ascending in neighbour index.  orc_smooth_graph fills row (n+1) and, when
 * cap >= S, nbr/c (S); returns S. */
int orc_smooth_graph(const float* x, const float* y, int32_t n, int32_t top_k, int64_t* row,
                     int32_t* nbr, float* c, int64_t cap);
/* L = bound after `iters` damped Jacobi steps; dLdx/dLdy (n) and dLdc (S,
 * per slot, the edge's total) when non-null.  Graph from (gx, gy) if given;
 * costs from (x, y) on that graph, or c_override. */
int orc_smooth_bound(const float* x, const float* y, int32_t n, int32_t top_k, double tau,
                     int32_t iters, double omega, int32_t newton_max, const float* gx,
                     const float* gy, const float* c_override, double* L, double* dLdx,
                     double* dLdy, double* dLdc);

#ifdef __cplusplus
}
#endif
#endif
