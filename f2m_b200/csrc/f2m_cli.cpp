// F2M.solver.exe: the reference's command line (RUN.cpp:12-31) over the C ABI.
//   F2M.solver.exe file N
// writes <file>.topN.F2M_report / .F2M_solution / .DM (and <file>_duplicates)
// next to the input, as the reference does.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/f2m.h"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::printf(
            "usage: ./F2M.RUN.exe fileXY topK\nfileXY == file in TSPLIB format\ntopK == the number of top K "
            "closest neighbors for each node\n");
        return 0;
    }
    const std::string file = argv[1];
    const int N = std::atoi(argv[2]);
    f2m_ctx* ctx = nullptr;
    f2m_status s = f2m_create(&ctx, 0);
    if (s != F2M_OK) {
        std::fprintf(stderr, "f2m: no usable CUDA device (status %d)\n", (int)s);
        return 1;
    }
    f2m_params p;
    f2m_default_params(&p);
    f2m_result* r = nullptr;
    s = f2m_solve_file(ctx, file.c_str(), N, &p, 1, &r);
    int rc = 0;
    if (r && (s == F2M_OK || s == F2M_ERR_NOT_CONVERGED)) {
        f2m_stats st;
        f2m_result_stats(r, &st);
        std::printf("Edges:%d\nNodes:%d\n", f2m_result_n_edges(r), f2m_result_n_nodes(r));
        if (s == F2M_OK) {
            std::printf("Optimal Found: Yes\nOptimal Value: %.15g\nRunTime: %g\nMAX edge rank: %d\n",
                        f2m_result_lp(r), f2m_result_seconds(r), f2m_result_max_rank(r));
            std::printf("Solution File: %s.top%d.F2M_solution\n", file.c_str(), N);
        } else {
            std::printf("ERROR: Optimal Solution not Found\n");
        }
    } else {
        std::fprintf(stderr, "f2m: %s (status %d)\n", f2m_last_error(ctx), (int)s);
        rc = 1;
    }
    f2m_result_free(r);
    f2m_destroy(ctx);
    return rc;
}
