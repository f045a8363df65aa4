/*
 * CPU oracle for the F2M hot path -- TEST INFRASTRUCTURE ONLY (see
 * f2m_oracle.h).  A restatement, in plain C++17/FP64, of the reference
 * solver aav-antonov/F2M.  Each block cites the reference file:line whose
 * behaviour it restates.  The product library (f2m_b200) never links this.
 *
 * Parity notes (where the reference's own behaviour is undefined or hangs):
 *  - get_KXY's `int area` overflows for x-span > 46340 and is 0 for a zero
 *    x-span (FXY.hpp:305); the reference then never leaves cuda_D2_stat.  The
 *    oracle widens the area to int64 and falls back to the y-span when the
 *    x-span is 0.  Inputs the reference can run are unaffected.
 *  - nvcc contracts `s*j + s*L` and `dY*dY + dX*dX` into FMAs
 *    (FXY.hpp:382,458,480,493); the oracle uses fma(s,j,s*L) and
 *    fma(dY,dY,dX*dX).  For integer coordinates every product is exact.
 *  - qpart_ptr_B/EF read one element past either end of a node's list
 *    (graph_cuda_partition.hpp:17-18,44-45); the value read never changes
 *    the result, so the oracle tests the bound first.
 *  - a stale comb index in the repair loop (comb_IRREGULAR_B kept from an
 *    earlier check, graph_cuda_comb.hpp:121-147) makes the reference read
 *    past its comb arrays; the oracle skips such indices.
 */
#include "f2m_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <numeric>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* ------------------------------------------------------------------ */
/* parameters: the reference's hard-coded constants                     */
/* ------------------------------------------------------------------ */
struct Params {
    double error_B = 1e-7;       // graph_cuda.cu:56
    double error_B_comb = 1e2;   // graph_cuda.cu:57
    int glob_K = 5;              // graph_cuda.cu:370
    int glob_rounds = 200;       // graph_cuda.cu:375
    int glob_inner = 50;         // graph_cuda.cu:377
    double glob_tol = 0.01;      // graph_cuda.cu:394
    int factor0 = 100;           // graph_cuda.cu:178
    int factor_step = 300;       // graph_cuda.cu:186
    int factor_cap = 5000;       // graph_cuda.cu:186
    int max_rounds = 10000;      // graph_cuda.cu:179
    int fix_rounds = 100;        // graph_cuda.cu:214
    int fix_factor = 500;        // graph_cuda.cu:216
    int check_every = 50;        // graph_cuda.cu:323
    int frozen_iters = 20;       // graph_cuda_comb.hpp:556
    double ef_thr = 1.0;         // graph_cuda.cu:259
    int ef_small_deg = 10;       // graph_cuda_partition.hpp:62
    int ef_min = 3;              // graph_cuda_partition.hpp:50
    double comb_thr = 0.25;      // graph_cuda_comb.hpp:420
    double shift0 = 0.5;         // graph_cuda.cu:72
    double shift_max = 32;       // graph_cuda.cu:125
};

/* ------------------------------------------------------------------ */
/* points: get_size / get_KXY (FXY.hpp:186-309)                          */
/* ------------------------------------------------------------------ */
struct Points {
    std::vector<int> K;
    std::vector<double> X, Y;
    double size_per_node = 0;
    // duplicates[k0][k] (FXY.hpp:37,263); insertion order kept by the map
    std::unordered_map<int, std::unordered_map<int, int>> duplicates;
};

// FXY.hpp:231-309 applied to an in-memory triple stream.
static int finish_points(Points& P, const std::vector<int>& k, const std::vector<double>& x,
                         const std::vector<double>& y, std::string& err) {
    std::unordered_map<double, std::unordered_map<double, int>> filtr;  // FXY.hpp:233
    double min_x = 0, min_y = 0, max_x = 0, max_y = 0;
    int i = 0;
    for (size_t t = 0; t < k.size(); ++t) {
        double xx = std::round(x[t] * 1000);  // FXY.hpp:252-256
        double yy = std::round(y[t] * 1000);
        xx /= 1000;
        yy /= 1000;
        if (k[t] <= -1) continue;  // FXY.hpp:258
        auto fx = filtr.find(xx);
        if (fx != filtr.end()) {
            auto fy = fx->second.find(yy);
            if (fy != fx->second.end()) {  // FXY.hpp:260-265
                P.duplicates[fy->second][k[t]]++;
                continue;
            }
        }
        filtr[xx][yy] = k[t];
        if (i == 0) {
            min_x = xx; min_y = yy; max_x = xx; max_y = yy;
        } else {
            if (min_x > xx) min_x = xx;
            if (min_y > yy) min_y = yy;
            if (max_x < xx) max_x = xx;
            if (max_y < yy) max_y = yy;
        }
        P.K.push_back(k[t]);
        P.X.push_back(xx);
        P.Y.push_back(yy);
        i++;
    }
    if (i < 2) { err = "fewer than 2 distinct points"; return ORC_ERR_INPUT; }
    // FXY.hpp:305-306 with the area widened to int64 (see header note)
    double sx = max_x - min_x, sy = max_y - min_y;
    long long area = (long long)(sx * sx);
    if (area == 0) area = (long long)(sy * sy);
    if (area == 0) { err = "degenerate bounding box"; return ORC_ERR_INPUT; }
    P.size_per_node = std::sqrt((double)area / (double)i);
    return ORC_OK;
}

// FXY.hpp:186-229 (get_size) + the fscanf loop of FXY.hpp:241-291.
static int parse_tsplib(const std::string& path, Points& P, std::string& err) {
    std::ifstream F(path);
    if (!F.is_open()) { err = "cannot open " + path; return ORC_ERR_INPUT; }
    std::string line, body;
    int start = 0, count = 0;
    while (std::getline(F, line)) {
        if (line.compare(0, 3, "EOF") == 0) break;
        if (start == 1) { count++; body += line; body += ' '; continue; }
        if (line.compare(0, 18, "NODE_COORD_SECTION") == 0) start = 1;
    }
    if (count == 0) { err = "file is not in TSPLIB format"; return ORC_ERR_INPUT; }
    std::vector<int> k;
    std::vector<double> x, y;
    const char* p = body.c_str();
    for (;;) {
        int kk = -1, n = 0;
        double xx = 0, yy = 0;
        int r = sscanf(p, "%d%n", &kk, &n);
        if (r == EOF) break;
        if (r != 1) { err = "non-numeric token in NODE_COORD_SECTION"; return ORC_ERR_INPUT; }
        p += n;
        r = sscanf(p, "%lf%n", &xx, &n);
        if (r != 1) { err = "truncated coordinate triple"; return ORC_ERR_INPUT; }
        p += n;
        r = sscanf(p, "%lf%n", &yy, &n);
        if (r != 1) { err = "truncated coordinate triple"; return ORC_ERR_INPUT; }
        p += n;
        k.push_back(kk); x.push_back(xx); y.push_back(yy);
    }
    return finish_points(P, k, x, y, err);
}

/* ------------------------------------------------------------------ */
/* spatial grid used only to enumerate points in a box quickly           */
/* ------------------------------------------------------------------ */
struct Grid {
    double x0 = 0, y0 = 0, h = 1;
    long long nx = 1, ny = 1;
    std::vector<int> start, idx;
    void build(const Points& P, double cell) {
        int n = (int)P.X.size();
        double minx = P.X[0], maxx = P.X[0], miny = P.Y[0], maxy = P.Y[0];
        for (int i = 1; i < n; ++i) {
            minx = std::min(minx, P.X[i]); maxx = std::max(maxx, P.X[i]);
            miny = std::min(miny, P.Y[i]); maxy = std::max(maxy, P.Y[i]);
        }
        x0 = minx; y0 = miny;
        double span = std::max(maxx - minx, maxy - miny);
        h = std::max(cell, span / 2048.0);
        if (!(h > 0)) h = 1;
        nx = (long long)((maxx - minx) / h) + 1;
        ny = (long long)((maxy - miny) / h) + 1;
        start.assign(nx * ny + 1, 0);
        std::vector<long long> c(n);
        for (int i = 0; i < n; ++i) {
            c[i] = cell_of(P.X[i], P.Y[i]);
            start[c[i] + 1]++;
        }
        for (long long t = 0; t < nx * ny; ++t) start[t + 1] += start[t];
        idx.assign(n, 0);
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int i = 0; i < n; ++i) idx[fill[c[i]]++] = i;  // ascending i per cell
    }
    long long cell_of(double x, double y) const {
        long long cx = (long long)((x - x0) / h), cy = (long long)((y - y0) / h);
        cx = std::min(std::max(cx, 0LL), nx - 1);
        cy = std::min(std::max(cy, 0LL), ny - 1);
        return cy * nx + cx;
    }
    template <class Fn>
    void query(double x, double y, double R, Fn fn) const {
        long long cx0 = (long long)std::floor((x - R - x0) / h), cx1 = (long long)std::floor((x + R - x0) / h);
        long long cy0 = (long long)std::floor((y - R - y0) / h), cy1 = (long long)std::floor((y + R - y0) / h);
        cx0 = std::max(cx0, 0LL); cy0 = std::max(cy0, 0LL);
        cx1 = std::min(cx1, nx - 1); cy1 = std::min(cy1, ny - 1);
        if (cx0 > cx1 || cy0 > cy1) return;
        if ((cx1 - cx0 + 1) * (cy1 - cy0 + 1) > (long long)idx.size()) {
            for (int i : idx) fn(i);
            return;
        }
        for (long long cy = cy0; cy <= cy1; ++cy)
            for (long long cx = cx0; cx <= cx1; ++cx) {
                long long c = cy * nx + cx;
                for (int t = start[c]; t < start[c + 1]; ++t) fn(idx[t]);
            }
    }
};

/* ------------------------------------------------------------------ */
/* FXY kNN candidates (FXY.hpp:23-144, 313-534)                          */
/* ------------------------------------------------------------------ */
// Edge cost as the reference computes it: sqrt(dY*dY + dX*dX) (FXY.hpp:382),
// contracted by nvcc into fma(dY,dY,dX*dX).
static inline double dist_ref(double x1, double y1, double x2, double y2) {
    double dX = std::fabs(x1 - x2), dY = std::fabs(y1 - y2);
    return std::sqrt(std::fma(dY, dY, dX * dX));
}
static inline double cost_of(double d, int mode) {
    if (mode == ORC_COST_NINT) return (double)(long long)(d + 0.5);  // TSPLIB nint
    return d;
}

struct Cutoffs {
    std::vector<double> cut;
    std::vector<int> stat;
};

// cuda_D2_stat_SUB (FXY.hpp:441-505) for node t, ring scale s = 2*size_per_node.
static void stat_sub(const Points& P, const Grid& G, int t, int L, int maxE, double s, int& st,
                     double& cut) {
    const int l = 5;  // FXY.hpp:521
    const double sL = s * (double)L;
    const double max_D = std::fma(s, (double)l, sL);  // FXY.hpp:458
    double lim[l];
    for (int j = 0; j < l; ++j) lim[j] = std::fma(s, (double)j, sL);  // FXY.hpp:480
    int stat[l] = {0, 0, 0, 0, 0};
    const double x1 = P.X[t], y1 = P.Y[t];
    G.query(x1, y1, max_D, [&](int i) {
        if (i == t) return;
        double dX = std::fabs(x1 - P.X[i]);
        if (dX > max_D) return;
        double dY = std::fabs(y1 - P.Y[i]);
        if (dY > max_D) return;
        double dD = std::sqrt(std::fma(dY, dY, dX * dX));
        if (dD > max_D) return;
        for (int j = l - 1; j >= 1; --j) {
            if (lim[j] > dD) stat[j]++;
            else break;
        }
    });
    st = stat[0];  // FXY.hpp:486-502
    cut = lim[0];
    for (int j = 1; j < l; ++j) {
        st = stat[j];
        cut = lim[j];
        if (stat[j] > maxE) break;
    }
}

// cuda_D2_stat (FXY.hpp:508-534): rings from L=0, then L=5,10,20,...
static void compute_cutoffs(const Points& P, const Grid& G, int top_k, int threads, Cutoffs& C) {
    int n = (int)P.X.size();
    C.cut.assign(n, 0);
    C.stat.assign(n, 0);
    double s = 2 * P.size_per_node;  // FXY.hpp:78
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) if (threads > 1)
    for (int t = 0; t < n; ++t) {
        int st;
        double cut;
        stat_sub(P, G, t, 0, top_k, s, st, cut);
        int L = 5;
        while (st < top_k) {
            stat_sub(P, G, t, L, top_k, s, st, cut);
            L *= 2;
        }
        C.cut[t] = cut;
        C.stat[t] = st;
    }
}

struct Cand {  // MyEdge (F2M.h:7-16)
    int k1, k2, v1, v2;
    double d;
};

// cuda_D2_fill (FXY.hpp:347-437) + thrust::sort (FXY.hpp:100-101, stable in
// emission order) + cuda_D2_cutN (FXY.hpp:326-344).
static int knn_literal(const Points& P, const Grid& G, const Cutoffs& C, int mode,
                       std::vector<Cand>& out, std::string& err) {
    int n = (int)P.X.size();
    std::vector<std::vector<Cand>> blocks(n);
    int overflow = 0;
    for (int t = 0; t < n; ++t) {
        double x1 = P.X[t], y1 = P.Y[t], max_D = C.cut[t];
        std::vector<int> nb;
        G.query(x1, y1, max_D, [&](int i) { nb.push_back(i); });
        std::sort(nb.begin(), nb.end());  // the reference scans i ascending
        auto& Q = blocks[t];
        for (int i : nb) {
            if (i == t) continue;
            double dX = std::fabs(x1 - P.X[i]);
            if (dX > max_D) continue;
            double dY = std::fabs(y1 - P.Y[i]);
            if (dY > max_D) continue;
            double dD = std::sqrt(std::fma(dY, dY, dX * dX));
            if (dD > max_D) continue;
            Cand c;
            if (dD < C.cut[i]) {
                if (t < i) c = {P.K[t], P.K[i], t, i, cost_of(dD, mode)};
                else c = {P.K[i], P.K[t], i, t, 1e10};
            } else {
                if (t < i) c = {P.K[t], P.K[i], t, i, cost_of(dD, mode)};
                else c = {P.K[i], P.K[t], i, t, cost_of(dD, mode)};
            }
            Q.push_back(c);
        }
        if ((int)Q.size() != C.stat[t]) overflow++;  // dD == cutoff exactly
    }
    if (overflow) {
        err = "a candidate lies exactly on a cutoff radius (reference block overflow)";
        return ORC_ERR_INPUT;
    }
    out.clear();
    for (auto& b : blocks) out.insert(out.end(), b.begin(), b.end());
    std::stable_sort(out.begin(), out.end(), [](const Cand& a, const Cand& b) { return a.d < b.d; });
    size_t cut = out.size();
    for (size_t t = 1; t < out.size(); ++t)
        if (out[t - 1].d < 1e10 && out[t].d == 1e10) { cut = t; break; }
    out.resize(cut);
    return ORC_OK;
}

// An undirected kept edge in global order, endpoints as FXY indices a<b.
struct KEdge {
    int a, b;
    double Do;
};

// graph::graph greedy loop (graph_tour.hpp:28-90): keep (i,j) unless both
// endpoints already hold E_max kept edges.
static int union_literal(const Points& P, const std::vector<Cand>& cands, int E_max,
                         std::vector<KEdge>& kept, std::string& err) {
    int Vn = (int)P.X.size();
    std::vector<int> stat(Vn, 0);
    std::vector<char> seen(Vn, 0);
    std::unordered_map<long long, int> vv2edge;
    int countEMAX = 0, created = 0;
    kept.clear();
    for (const Cand& c : cands) {
        if (countEMAX == Vn) break;  // graph_tour.hpp:30
        if (c.d == 0) { err = "zero-length edge"; return ORC_ERR_INPUT; }  // :44-49
        int i = c.v1, j = c.v2;  // FXY indices of labels k1,k2
        if (created < Vn) {
            if (!seen[i]) { seen[i] = 1; created++; }
            if (!seen[j]) { seen[j] = 1; created++; }
        }
        if (stat[i] > E_max && stat[j] > E_max) continue;  // :62
        stat[i]++; stat[j]++;
        if (stat[i] == E_max) { countEMAX++; stat[i]++; }
        if (stat[j] == E_max) { countEMAX++; stat[j]++; }
        long long key = (long long)std::min(i, j) * (long long)Vn + std::max(i, j);
        if (vv2edge.count(key)) { err = "duplicate edge key"; return ORC_ERR_INPUT; }  // :77-81
        vv2edge[key] = (int)kept.size();
        kept.push_back({c.v1, c.v2, c.d});
    }
    return ORC_OK;
}

// Equivalent, per-node formulation of FXY + the greedy loop: the kept set is
// the union over nodes of each node's first E_max incident candidates in the
// global (cost, emitter, partner) order; the pair (a<b) at distance d is
// emitted by a if d <= cut[a], else by b (FXY.hpp:388-432).
struct TKey {
    double cost;
    int em, other;
    bool operator<(const TKey& o) const {
        if (cost != o.cost) return cost < o.cost;
        if (em != o.em) return em < o.em;
        return other < o.other;
    }
};
static int knn_topn(const Points& P, const Grid& G, const Cutoffs& C, int mode, int top_k, int E_max,
                    int threads, std::vector<KEdge>& kept, std::string& err) {
    int n = (int)P.X.size();
    int N = std::min(E_max, n - 1);
    std::vector<std::vector<std::pair<TKey, std::pair<int, int>>>> lists(n);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) if (threads > 1) reduction(+ : bad)
    for (int i = 0; i < n; ++i) {
        double x1 = P.X[i], y1 = P.Y[i];
        std::vector<std::pair<TKey, std::pair<int, int>>> c;
        auto consider = [&](int j, double R_in) {
            if (j == i) return;
            double d = dist_ref(x1, y1, P.X[j], P.Y[j]);
            bool cand = (d <= C.cut[i]) || (d <= C.cut[j]);
            if (!cand || d > R_in) return;
            int a = std::min(i, j), b = std::max(i, j);
            if (d == C.cut[a] && d <= C.cut[b]) bad++;  // emitted twice by the reference
            int em = (d <= C.cut[a]) ? a : b;
            int other = (em == a) ? b : a;
            c.push_back({{cost_of(d, mode), em, other}, {a, b}});
        };
        G.query(x1, y1, C.cut[i], [&](int j) { consider(j, C.cut[i]); });
        std::sort(c.begin(), c.end(), [](const auto& p, const auto& q) { return p.first < q.first; });
        if (mode == ORC_COST_NINT && (int)c.size() >= N && N > 0) {
            // candidates outside cut[i] can tie in nint cost with the N-th
            double R = c[N - 1].first.cost + 0.5;
            if (R > C.cut[i]) {
                c.clear();
                G.query(x1, y1, R, [&](int j) { consider(j, std::max(R, C.cut[i])); });
                std::sort(c.begin(), c.end(), [](const auto& p, const auto& q) { return p.first < q.first; });
            }
        }
        if ((int)c.size() > N) c.resize(N);
        lists[i] = std::move(c);
    }
    (void)top_k;
    if (bad) { err = "a candidate lies exactly on a cutoff radius (reference duplicate key)"; return ORC_ERR_INPUT; }
    std::vector<std::pair<TKey, std::pair<int, int>>> all;
    for (auto& l : lists) all.insert(all.end(), l.begin(), l.end());
    std::sort(all.begin(), all.end(), [](const auto& p, const auto& q) { return p.first < q.first; });
    kept.clear();
    for (size_t t = 0; t < all.size(); ++t) {
        if (t > 0 && all[t].second == all[t - 1].second) continue;  // same pair from both sides
        if (all[t].first.cost == 0) { err = "zero-length edge"; return ORC_ERR_INPUT; }
        kept.push_back({all[t].second.first, all[t].second.second, all[t].first.cost});
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* graph: graph::graph tail + graph_c::init                             */
/* ------------------------------------------------------------------ */
struct Graph {
    int Vn = 0, En = 0;
    std::vector<int> label, fxy;       // internal id -> label / FXY index
    std::vector<int> ev1, ev2;         // internal ids, ev1 < ev2 (graph_cuda_init.hpp:31-36)
    std::vector<int> el1, el2;         // lower-label / higher-label endpoint (F2M.h:109-113)
    std::vector<double> Do, D;
    std::vector<int> rank1, rank2;     // rankDo1/rankDo2 (node.cpp:18)
    std::vector<int> row, adj;         // CSR in edge-id order (graph_cuda_init.hpp:42-63)
    double d_min = 0;
};

static void assemble_graph(const Points& P, const std::vector<KEdge>& kept, int id_order, Graph& G) {
    int n = (int)P.X.size();
    std::vector<int> id_of(n, -1);
    if (id_order == ORC_ID_REF) {
        // node creation order = first appearance (label k1 then k2) in the
        // candidate order (graph_tour.hpp:53-58); internal ids follow the
        // unordered_map<int,node*> iteration order (graph_tour.hpp:95-97).
        std::unordered_map<int, int> map_node;
        std::vector<int> created;
        for (const KEdge& e : kept) {
            int ks[2] = {e.a, e.b};
            for (int f : ks) {
                int lab = P.K[f];
                if (map_node.count(lab) == 0) {
                    map_node[lab] = f;
                    created.push_back(f);
                }
            }
        }
        int iV = 0;
        for (auto& kv : map_node) id_of[kv.second] = iV++;
        G.Vn = iV;
    } else {
        for (int i = 0; i < n; ++i) id_of[i] = i;
        G.Vn = n;
    }
    G.label.assign(G.Vn, 0);
    G.fxy.assign(G.Vn, 0);
    for (int i = 0; i < n; ++i)
        if (id_of[i] >= 0) { G.label[id_of[i]] = P.K[i]; G.fxy[id_of[i]] = i; }
    G.En = (int)kept.size();
    G.ev1.resize(G.En); G.ev2.resize(G.En); G.el1.resize(G.En); G.el2.resize(G.En);
    G.Do.resize(G.En); G.D.resize(G.En); G.rank1.resize(G.En); G.rank2.resize(G.En);
    double d_min = 1e16;
    for (int e = 0; e < G.En; ++e) {
        int u = id_of[kept[e].a], v = id_of[kept[e].b];
        G.ev1[e] = std::min(u, v); G.ev2[e] = std::max(u, v);
        if (G.label[u] < G.label[v]) { G.el1[e] = u; G.el2[e] = v; }
        else { G.el1[e] = v; G.el2[e] = u; }
        G.Do[e] = kept[e].Do;
        if (kept[e].Do < d_min) d_min = kept[e].Do;  // graph_tour.hpp:70
    }
    G.d_min = d_min;
    for (int e = 0; e < G.En; ++e) G.D[e] = G.Do[e] / d_min;  // F2M.h:101, graph_tour.hpp:94
    // CSR (graph_cuda_init.hpp:26-63): slots in edge-id order per node
    G.row.assign(G.Vn + 1, 0);
    for (int e = 0; e < G.En; ++e) { G.row[G.ev1[e] + 1]++; G.row[G.ev2[e] + 1]++; }
    for (int v = 0; v < G.Vn; ++v) G.row[v + 1] += G.row[v];
    G.adj.assign(2 * (size_t)G.En, 0);
    std::vector<int> fill(G.row.begin(), G.row.end() - 1);
    for (int e = 0; e < G.En; ++e) {
        int r1 = fill[G.ev1[e]]++ - G.row[G.ev1[e]];
        int r2 = fill[G.ev2[e]]++ - G.row[G.ev2[e]];
        G.adj[G.row[G.ev1[e]] + r1] = e;
        G.adj[G.row[G.ev2[e]] + r2] = e;
        // rankDo (node.cpp:18): position in the node's push-ordered list
        int rl = (G.el1[e] == G.ev1[e]) ? r1 : r2;
        int rh = (G.el1[e] == G.ev1[e]) ? r2 : r1;
        G.rank1[e] = rl; G.rank2[e] = rh;
    }
}

/* ------------------------------------------------------------------ */
/* the solver state: graph_c + the host stage of graph                   */
/* ------------------------------------------------------------------ */
struct Solver {
    const Graph& G;
    Params prm;
    int threads;
    std::vector<double> F, grad;
    std::vector<int> perm;              // cuda_Edges_d_by_Nodes as edge ids, permuted in place
    std::vector<int> efcnt;             // cuda_EF_NodesStat
    std::vector<int> efoff, eflist, efn;  // cuda_EF snapshot (update_EF)
    std::vector<int> combcnt, blockid, statA, statB;
    std::vector<int> comb_root, comb_vs, comb_vn, comb_V, comb_es, comb_en, comb_E;
    orc_stats st{};
    bool converged = false;
    // host stage (graph)
    std::vector<double> dcpu;
    std::vector<std::vector<int>> node_edges;  // node::edges, persistent across checks
    std::vector<std::vector<int>> eA, eB;
    std::vector<int> sA, sB;
    std::vector<int> irrB;                     // comb_IRREGULAR_B (persistent, F2M.h:166)
    struct CombH {
        std::unordered_map<int, int> nodes, edgesB;
        std::unordered_map<int, float> XB;
        int STATUS = 1, AxB_status = 1;
    };
    std::vector<CombH> Combs;
    double porog;

    explicit Solver(const Graph& g, int thr) : G(g), threads(thr) {
        F.assign(G.Vn, 0.0);                  // graph_cuda_init.hpp:183
        grad.assign(G.Vn, 0.0);
        perm = G.adj;
        efcnt.assign(G.Vn, 0);
        combcnt.assign(G.Vn, 0);
        blockid.assign(G.Vn, 0);
        statA.assign(G.Vn, 0);
        statB.assign(G.Vn, 0);
        porog = prm.error_B * prm.error_B_comb;  // graph_cuda_comb.hpp:156
        node_edges.resize(G.Vn);
        for (int v = 0; v < G.Vn; ++v) node_edges[v].assign(G.adj.begin() + G.row[v], G.adj.begin() + G.row[v + 1]);
    }
    int deg(int v) const { return G.row[v + 1] - G.row[v]; }
    // cuda_recompute_Edges (graph_cuda_grad.hpp:257-268)
    double dval(int e) const { return G.D[e] + 0.5 * F[G.ev1[e]] + 0.5 * F[G.ev2[e]]; }

    // cuda_get_Nodes_grad_R (graph_cuda_grad.hpp:321-340)
    double grad_of(const int* list, int cnt) const {
        double v0 = dval(list[0]), v1 = 1e6, v2 = 1e6;
        for (int i = 1; i < cnt; ++i) {
            double v = dval(list[i]);
            if (v < v0) { v2 = v1; v1 = v0; v0 = v; continue; }
            if (v < v1) { v2 = v1; v1 = v; continue; }
            if (v < v2) { v2 = v; continue; }
        }
        return -(v1 + v2) / 2;
    }
    // qpart_ptr_B (graph_cuda_partition.hpp:3-25)
    int qpartB(int* list, int size, double avg) const {
        int low = 0, high = size - 1, i = low, j = high;
        while (i < j) {
            while (i <= high && dval(list[i]) <= avg) i++;
            while (j >= low && dval(list[j]) > avg) j--;
            if (i < j) std::swap(list[i], list[j]);
        }
        return j + 1;
    }
    // qpart_ptr_EF (graph_cuda_partition.hpp:27-54)
    int qpartEF(int* list, int size, double avg) const {
        int pivot;
        for (;;) {
            pivot = qpartB(list, size, avg);
            if (pivot < prm.ef_min) { avg += 1; continue; }
            break;
        }
        return pivot;
    }
    double max_abs(const std::vector<double>& g) const {  // max_node_grad (graph_cuda_maxmin.hpp:29-37)
        double m = 0;
        for (double x : g) m = std::max(m, std::fabs(x));
        return m;
    }
    void grad_prefix() {
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
        for (int v = 0; v < G.Vn; ++v) grad[v] = grad_of(&perm[G.row[v]], efcnt[v]);
    }
    void grad_ef() {
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
        for (int v = 0; v < G.Vn; ++v) grad[v] = grad_of(&eflist[efoff[v]], efn[v]);
    }
    void apply_F(bool masked) {  // cuda_update_Nodes_F(_BLOCK) (graph_cuda_grad.hpp:302-317)
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
        for (int v = 0; v < G.Vn; ++v)
            if (!masked || blockid[v] == 0) F[v] += grad[v];
    }
    // block_GLOB + block_GLOB_N (graph_cuda.cu:363-430)
    void block_GLOB() {
        for (int v = 0; v < G.Vn; ++v) efcnt[v] = std::min(deg(v), prm.glob_K);  // setvalue2V (:354-372)
        for (int go = 0; go < prm.glob_rounds; ++go) {
            st.glob_rounds++;
            for (int it = 0; it < prm.glob_inner; ++it) {
                grad_prefix();
                apply_F(false);
                st.iters_glob++;
            }
            // cuda_partition_v4 (graph_cuda_partition.hpp:89-115)
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
            for (int v = 0; v < G.Vn; ++v) {
                int* list = &perm[G.row[v]];
                if (deg(v) < prm.glob_K) { efcnt[v] = deg(v); continue; }
                double avg = dval(list[0]);
                for (int i = 1; i < prm.glob_K; ++i) { double x = dval(list[i]); if (x > avg) avg = x; }
                efcnt[v] = qpartEF(list, deg(v), avg);
            }
            grad_prefix();
            if (max_abs(grad) < prm.glob_tol) break;
        }
    }
    // check_OPT (graph_cuda.cu:254-271) with cuda_partition_v2
    double check_OPT() {
        st.checks++;
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
        for (int v = 0; v < G.Vn; ++v) {
            if (deg(v) < prm.ef_small_deg) efcnt[v] = deg(v);
            else efcnt[v] = qpartEF(&perm[G.row[v]], deg(v), prm.ef_thr);
        }
        grad_prefix();
        double m = max_abs(grad);
        st.max_grad = m;
        return m;
    }
    // update_EF (graph_cuda.cu:229-252)
    void update_EF() {
        efoff.assign(G.Vn, 0);
        efn = efcnt;
        long long s = 0;
        for (int v = 0; v < G.Vn; ++v) { efoff[v] = (int)s; s += efcnt[v]; }
        eflist.resize(s);
        for (int v = 0; v < G.Vn; ++v)
            for (int i = 0; i < efcnt[v]; ++i) eflist[efoff[v] + i] = perm[G.row[v] + i];
        st.ef_slots = s;
    }
    // block_EF (graph_cuda.cu:308-338)
    int64_t block_EF(int N) {
        grad_ef();
        double MA = max_abs(grad);
        int count_M = 0;
        int64_t n = 0;
        for (int go = 0; go < N; ++go) {
            grad_ef();
            apply_F(false);
            n++;
            count_M++;
            if (count_M >= prm.check_every) {
                if (MA < prm.error_B) break;
                count_M = 0;
            }
        }
        return n;
    }
    // run_start_cuda (graph_cuda.cu:163-199)
    void run_start() {
        block_GLOB();
        check_OPT();
        update_EF();
        int factor = prm.factor0;
        for (int go = 1; go <= prm.max_rounds; ++go) {
            st.ef_rounds++;
            st.iters_ef += block_EF(factor);
            double M = check_OPT();
            update_EF();
            if (factor < prm.factor_cap) factor += prm.factor_step;
            if (M < prm.error_B) { converged = true; break; }
        }
    }
    // run_fix_cuda (graph_cuda.cu:204-226)
    void run_fix() {
        check_OPT();
        update_EF();
        for (int go = 1; go <= prm.fix_rounds; ++go) {
            st.iters_repair += block_EF(prm.fix_factor);
            double M = check_OPT();
            update_EF();
            if (M < prm.error_B) break;
        }
    }
    // get_cuda_comb_size / get_cuda_comb_fill BFS (graph_cuda_comb.hpp:258-392)
    int bfs(int tid, bool check, std::vector<int>* nodes, std::vector<int>* edges,
            std::vector<int>& mark_n, std::vector<int>& mark_e, int stamp) const {
        int ind_break = 0;
        std::vector<int> fn{tid}, fe, A{tid}, B;
        mark_n[tid] = stamp;
        while (!A.empty()) {
            B.clear();
            for (int lA : A) {
                const int* ptr = &perm[G.row[lA]];
                for (int i = 0; i < combcnt[lA]; ++i) {
                    int e = ptr[i];
                    double x = dval(e);
                    if (x >= -porog && x <= porog) {
                        ind_break = -1;
                        if (check && (G.ev1[e] < tid || G.ev2[e] < tid)) { ind_break = 1; break; }
                        if (mark_e[e] != stamp) { mark_e[e] = stamp; fe.push_back(e); }
                        int v = G.ev1[e];
                        if (v == lA) v = G.ev2[e];
                        if (mark_n[v] != stamp) { mark_n[v] = stamp; B.push_back(v); fn.push_back(v); }
                    }
                }
                if (ind_break == 1) break;
            }
            if (ind_break == 1) break;
            std::swap(A, B);
        }
        if (ind_break == -1) {
            if (nodes) *nodes = fn;
            if (edges) *edges = fe;
            return 1;
        }
        return 0;
    }
    // get_combs (graph_cuda_comb.hpp:415-475)
    void get_combs() {
#pragma omp parallel for schedule(static) num_threads(threads) if (threads > 1)
        for (int v = 0; v < G.Vn; ++v) combcnt[v] = qpartB(&perm[G.row[v]], efcnt[v], prm.comb_thr);
        std::vector<int> mark_n(G.Vn, -1), mark_e(G.En, -1);
        comb_root.clear(); comb_vs.clear(); comb_vn.clear(); comb_V.clear();
        comb_es.clear(); comb_en.clear(); comb_E.clear();
        int stamp = 0;
        for (int v = 0; v < G.Vn; ++v) {
            std::vector<int> nn, ee;
            if (bfs(v, true, &nn, &ee, mark_n, mark_e, stamp++)) {
                comb_root.push_back(v);
                comb_vs.push_back((int)comb_V.size()); comb_vn.push_back((int)nn.size());
                comb_V.insert(comb_V.end(), nn.begin(), nn.end());
                comb_es.push_back((int)comb_E.size()); comb_en.push_back((int)ee.size());
                comb_E.insert(comb_E.end(), ee.begin(), ee.end());
            }
        }
        // cuda_get_Nodes_StatAB (graph_cuda_grad.hpp:274-295)
        for (int v = 0; v < G.Vn; ++v) {
            int a = 0, b = 0;
            for (int i = 0; i < combcnt[v]; ++i) {
                double x = dval(perm[G.row[v] + i]);
                if (x < -porog) a++;
                else if (x < porog) b++;
            }
            statA[v] = a; statB[v] = b;
        }
        st.n_combs = (int)comb_root.size();
    }
    /* ---- host stage D: host_combs_check (graph_cuda_comb.hpp:121-147) ---- */
    // Ax_b (Ax_b.cpp:19-158, Ax_b.h:9-52)
    struct AxB {
        std::vector<std::vector<int>> Ai, Av;
        std::vector<int> b;
        std::vector<double> d, Aj, x, x_grad, b_grad;
        double d_max_error = 0;
        int go_max = 0, i_count = 0, j_count = 0;
        explicit AxB(const std::vector<int>& A) {
            int j = 0, Aj_norm = 0;
            std::vector<int> Aij, Avj;
            for (size_t k = 0; k + 1 < A.size(); k += 2) {
                int i = A[k], v = A[k + 1];
                if (!(i >= -1)) break;
                if (i > i_count) i_count = i;
                if (i == -1) {
                    b.push_back(v);
                    Aj.push_back(std::sqrt((double)Aj_norm));
                    Aj_norm = 0;
                    j++;
                    Ai.push_back(Aij); Av.push_back(Avj);
                    Aij.clear(); Avj.clear();
                } else {
                    Aij.push_back(i); Avj.push_back(v);
                    Aj_norm += v * v;
                }
            }
            j_count = j;
            x.assign(i_count + 1, 0.0);
            x_grad.assign(i_count + 1, 0.0);
            d.assign(j_count, 0.0);
            b_grad.assign(j_count, 0.0);
        }
        double ax(int j, const std::vector<double>& X) const {
            double v = 0;
            for (size_t i = 0; i < Ai[j].size(); i++) v += Av[j][i] * X[Ai[j][i]];
            return v;
        }
        void solve() {
            go_max = 0;
            for (int go = 1; go < 1000; go++) {
                std::fill(x_grad.begin(), x_grad.end(), 0.0);
                d_max_error = 0;
                for (size_t j = 0; j < Ai.size(); j++) {
                    d[j] = (ax((int)j, x) - b[j]) / Aj[j];
                    if (std::fabs(d[j]) > d_max_error) d_max_error = std::fabs(d[j]);
                    for (size_t i = 0; i < Ai[j].size(); i++) x_grad[Ai[j][i]] += Av[j][i] * d[j] / Aj[j];
                }
                if (d_max_error < 1e-8) { go_max = go; break; }
                std::fill(b_grad.begin(), b_grad.end(), 0.0);
                for (size_t j = 0; j < Ai.size(); j++) b_grad[j] = ax((int)j, x_grad);
                double gg = 0, gd = 0;
                for (size_t j = 0; j < b_grad.size(); j++) gg += b_grad[j] * b_grad[j];
                for (size_t j = 0; j < d.size(); j++) gd += d[j] * b_grad[j];
                double alfa = -gd / gg;
                for (size_t j = 0; j < x.size(); j++) x[j] += x_grad[j] * alfa;
            }
        }
    };
    int host_check() {
        int Vn = G.Vn;
        dcpu.resize(G.En);
        // EF_thread type 1 (E_thread.cpp:39): d = D + F[v1]/2 + F[v2]/2, v1 = lower label
        for (int e = 0; e < G.En; ++e) dcpu[e] = G.D[e] + F[G.el1[e]] / 2 + F[G.el2[e]] / 2;
        // V_thread 1: node::resort (node.cpp:19); V_thread 3: get_statusAB (node.cpp:49-57)
        eA.assign(Vn, {}); eB.assign(Vn, {});
        sA.assign(Vn, 0); sB.assign(Vn, 0);
        double vb = prm.error_B * prm.error_B_comb;
        for (int v = 0; v < Vn; ++v) {
            auto& ed = node_edges[v];
            std::sort(ed.begin(), ed.end(), [&](int a, int b) { return dcpu[a] < dcpu[b]; });
            for (int e : ed) {
                if (dcpu[e] < vb) {
                    if (dcpu[e] > -vb) { sB[v]++; eB[v].push_back(e); }
                    else { sA[v]++; eA[v].push_back(e); }
                } else break;
            }
        }
        // COMB_thread (comb_thread.cpp:33-52, 73-133)
        Combs.clear();
        Combs.resize(comb_root.size());
        for (size_t c = 0; c < comb_root.size(); ++c) {
            for (int i = 0; i < comb_vn[c]; ++i) Combs[c].nodes[comb_V[comb_vs[c] + i]]++;
            for (int i = 0; i < comb_en[c]; ++i) Combs[c].edgesB[comb_E[comb_es[c] + i]]++;
        }
        // COMB_solve_thread: comb::solve_simple (comb_thread.cpp:180-195)
        std::vector<int> irrA;
        for (size_t c = 0; c < Combs.size(); ++c) {
            auto& C = Combs[c];
            for (auto& kv : C.nodes) {
                int sv = 4 - 2 * sA[kv.first] - sB[kv.first];
                if (sv != 0) { C.STATUS = -1; break; }
            }
            if (C.STATUS == 1)
                for (auto& kv : C.nodes)
                    for (int e : eB[kv.first]) C.XB[e] = 0.5f;
            if (C.STATUS == -1) irrA.push_back((int)c);  // get_comb_IRREGULAR_A
        }
        st.irr_a = (int)irrA.size();
        if (!irrA.empty()) {
            // comb::solve_AxB (comb_thread.cpp:272-304)
            for (int c : irrA) {
                auto& C = Combs[c];
                std::vector<int> rows;
                std::unordered_map<int, int> mapX, mapXR;
                int countX = 0;
                for (auto& kv : C.nodes) {
                    for (int e : eB[kv.first]) {
                        int i;
                        if (mapX.count(e)) i = mapX[e];
                        else { i = countX; mapXR[i] = e; mapX[e] = i; countX++; }
                        rows.push_back(i); rows.push_back(1);
                    }
                    rows.push_back(-1);
                    rows.push_back(2 - (int)eA[kv.first].size());
                }
                AxB ab(rows);
                ab.solve();
                C.AxB_status = ab.go_max;
                for (size_t j = 0; j < ab.x.size(); j++) C.XB[mapXR[(int)j]] = (float)ab.x[j];
            }
            irrB.clear();  // get_comb_IRREGULAR_B (comb_thread.cpp:257-270)
            for (size_t c = 0; c < Combs.size(); ++c)
                if (Combs[c].AxB_status == 0) irrB.push_back((int)c);
        }
        st.irr_b = (int)irrB.size();
        return (int)irrB.size();
    }
    // shift_comb_IRREGULAR_B + cuda_IRREGULAR_B_recompute (graph_cuda_comb.hpp:484-574)
    void shift_refit(double shiftV, int type) {
        std::fill(blockid.begin(), blockid.end(), 0);
        for (int c : irrB) {
            if (c < 0 || c >= (int)comb_root.size()) continue;  // stale index (header note)
            for (int i = 0; i < comb_vn[c]; ++i) {
                int nid = comb_V[comb_vs[c] + i];
                int v = 4 - 2 * statA[nid] - statB[nid];
                if (v != 0) {
                    int shift = v > 0 ? 1 : -1;
                    F[nid] += shiftV * shift;
                    blockid[nid] = 1;
                    if (type == 1) break;
                }
            }
        }
        for (int go = 0; go < prm.frozen_iters; ++go) {  // block_EF_iter_BLOCK
            grad_ef();
            apply_F(true);
            st.iters_repair++;
        }
        std::fill(blockid.begin(), blockid.end(), 0);
        run_fix();
    }
    // graph::RUN (graph_cuda.cu:47-155)
    int run() {
        run_start();
        get_combs();
        int IRR_B = host_check();
        if (IRR_B > 0) {
            double s = prm.shift0;
            auto step = [&](double sv, int type) {
                st.repair_steps++;
                shift_refit(sv, type);
                get_combs();
                return host_check();
            };
            for (;;) {
                if ((IRR_B = step(s, 0)) == 0) break;
                if ((IRR_B = step(s, 1)) == 0) break;
                s = -s;
                if ((IRR_B = step(s, 0)) == 0) break;
                s = -s;
                if ((IRR_B = step(s, 1)) == 0) break;
                s = -s;
                s *= 2;
                if (std::fabs(s) > prm.shift_max) break;
            }
        }
        return IRR_B;
    }
};

}  // namespace

/* ------------------------------------------------------------------ */
/* result object and C API                                               */
/* ------------------------------------------------------------------ */
struct orc_result {
    int status = ORC_OK;
    std::string err;
    Points P;
    Cutoffs C;
    Graph G;
    std::vector<double> F, x;
    std::vector<int> comb_size, comb_nodes, statA, statB;
    std::unordered_map<int, double> X;  // graph::X (F2M.h:161)
    double lp = 0;
    int max_rank = 0;
    double run_seconds = 0;
    orc_stats st{};
};

namespace {

int build(orc_result* r, int top_k, int cost_mode, int id_order, int knn_mode, int threads) {
    if (top_k < 3) { r->err = "N must be at least 3"; return ORC_ERR_INPUT; }
    int n = (int)r->P.X.size();
    int tk = top_k;
    if (tk > n - 1) tk = n - 1;  // FXY.hpp:77 (clamped also when tk == n, where the reference hangs)
    Grid grid;
    grid.build(r->P, 2 * r->P.size_per_node);
    compute_cutoffs(r->P, grid, tk, threads, r->C);
    std::vector<KEdge> kept;
    int s;
    if (knn_mode == ORC_KNN_LITERAL) {
        std::vector<Cand> cands;
        s = knn_literal(r->P, grid, r->C, cost_mode, cands, r->err);
        if (s) return s;
        s = union_literal(r->P, cands, top_k, kept, r->err);
    } else {
        s = knn_topn(r->P, grid, r->C, cost_mode, tk, top_k, threads, kept, r->err);
    }
    if (s) return s;
    assemble_graph(r->P, kept, id_order, r->G);
    return ORC_OK;
}

void solve_graph(orc_result* r, int threads) {
    auto t0 = std::chrono::steady_clock::now();
    Solver S(r->G, threads);
    int IRR_B = S.run();
    auto t1 = std::chrono::steady_clock::now();
    r->run_seconds = std::chrono::duration<double>(t1 - t0).count();
    r->F = S.F;
    r->st = S.st;
    r->st.d_min = r->G.d_min;
    r->statA = S.statA;
    r->statB = S.statB;
    r->comb_size.clear(); r->comb_nodes.clear();
    for (size_t c = 0; c < S.comb_root.size(); ++c) {
        r->comb_size.push_back(S.comb_vn[c]);
        for (int i = 0; i < S.comb_vn[c]; ++i) r->comb_nodes.push_back(S.comb_V[S.comb_vs[c] + i]);
    }
    r->x.assign(r->G.En, 0.0);
    r->X.clear();
    if (IRR_B == 0) {
        // graph::RUN primal (graph_cuda.cu:135-147): node::get_eA_X (node.cpp:61-71)
        for (int v = 0; v < r->G.Vn; ++v)
            for (int e : S.eA[v]) {
                int v0 = r->G.label[v];
                int l1 = r->G.label[r->G.el1[e]], l2 = r->G.label[r->G.el2[e]];
                if (v0 < l1) r->X[e] = 1;
                if (v0 < l2) r->X[e] = 1;
            }
        for (auto& C : S.Combs)
            for (auto& kv : C.XB) r->X[kv.first] = kv.second;
        // graph::getOVAL (graph_tour.hpp:165-184)
        double OVAL = 0;
        int mr = 0;
        for (auto& kv : r->X) {
            int e = kv.first;
            int rr = std::min(r->G.rank1[e], r->G.rank2[e]);
            if (rr > mr) mr = rr;
            OVAL += kv.second * r->G.Do[e];
            r->x[e] = kv.second;
        }
        r->lp = OVAL;
        r->max_rank = mr;
        r->status = ORC_OK;
    } else {
        r->status = ORC_ERR_NOT_CONVERGED;
        r->err = "Optimal Solution not Found";
    }
}

void write_files(orc_result* r, const std::string& file, int top_k) {
    std::string base = file + ".top" + std::to_string(top_k);
    {   // graph::print_file_report (graph_tour.hpp:218-241)
        std::ofstream f(base + ".F2M_report");
        if (r->status == ORC_OK) {
            f << "Optimal Found: " << "Yes" << "\n";
            f << "Optimal Value: " << std::setprecision(15) << r->lp << "\n";
            f << "Time: " << r->run_seconds << "\n";
            f << "MAX edge rank: " << r->max_rank << "\n";
        } else {
            f << "ERROR: Optimal Solution not Found\n";
        }
    }
    if (r->status == ORC_OK) {  // graph::print_file_solution (graph_tour.hpp:186-214)
        std::ofstream f(base + ".F2M_solution");
        for (auto& kv : r->X) {
            int e = kv.first;
            f << r->G.label[r->G.el1[e]] << " " << r->G.label[r->G.el2[e]] << " " << std::setprecision(4)
              << kv.second << "\n";
        }
    }
}

}  // namespace

extern "C" {

int orc_solve_file(const char* path, int top_k, int cost_mode, int id_order, int knn_mode,
                   int write, int threads, orc_result** out) {
    orc_result* r = new orc_result();
    *out = r;
    int s = parse_tsplib(path, r->P, r->err);
    if (!s) s = build(r, top_k, cost_mode, id_order, knn_mode, threads);
    if (s) { r->status = s; return s; }
    solve_graph(r, threads);
    if (write) write_files(r, path, top_k);
    return r->status;
}

int orc_solve_points(const int32_t* K, const double* X, const double* Y, int32_t n, int top_k,
                     int cost_mode, int id_order, int knn_mode, int threads, orc_result** out) {
    orc_result* r = new orc_result();
    *out = r;
    std::vector<int> k(K, K + n);
    std::vector<double> x(X, X + n), y(Y, Y + n);
    int s = finish_points(r->P, k, x, y, r->err);
    if (!s) s = build(r, top_k, cost_mode, id_order, knn_mode, threads);
    if (s) { r->status = s; return s; }
    solve_graph(r, threads);
    return r->status;
}

int orc_build_graph(const int32_t* K, const double* X, const double* Y, int32_t n, int top_k,
                    int cost_mode, int id_order, int knn_mode, orc_result** out) {
    orc_result* r = new orc_result();
    *out = r;
    std::vector<int> k(K, K + n);
    std::vector<double> x(X, X + n), y(Y, Y + n);
    int s = finish_points(r->P, k, x, y, r->err);
    if (!s) s = build(r, top_k, cost_mode, id_order, knn_mode, 1);
    r->status = s;
    return s;
}

int orc_solve_graph(int32_t n_nodes, int32_t n_edges, const int32_t* ev1, const int32_t* ev2,
                    const double* D, const double* Do, const int32_t* node_label, int threads,
                    orc_result** out) {
    orc_result* r = new orc_result();
    *out = r;
    Graph& G = r->G;
    G.Vn = n_nodes;
    G.En = n_edges;
    G.label.resize(n_nodes);
    G.fxy.resize(n_nodes);
    for (int v = 0; v < n_nodes; ++v) { G.label[v] = node_label ? node_label[v] : v; G.fxy[v] = v; }
    G.ev1.assign(ev1, ev1 + n_edges);
    G.ev2.assign(ev2, ev2 + n_edges);
    G.el1.resize(n_edges); G.el2.resize(n_edges);
    G.D.assign(D, D + n_edges);
    G.Do.assign(Do, Do + n_edges);
    G.d_min = 0;
    for (int e = 0; e < n_edges; ++e) {
        if (G.label[ev1[e]] < G.label[ev2[e]]) { G.el1[e] = ev1[e]; G.el2[e] = ev2[e]; }
        else { G.el1[e] = ev2[e]; G.el2[e] = ev1[e]; }
    }
    G.row.assign(n_nodes + 1, 0);
    for (int e = 0; e < n_edges; ++e) { G.row[ev1[e] + 1]++; G.row[ev2[e] + 1]++; }
    for (int v = 0; v < n_nodes; ++v) G.row[v + 1] += G.row[v];
    G.adj.assign(2 * (size_t)n_edges, 0);
    G.rank1.assign(n_edges, 0); G.rank2.assign(n_edges, 0);
    std::vector<int> fill(G.row.begin(), G.row.end() - 1);
    for (int e = 0; e < n_edges; ++e) {
        int r1 = fill[ev1[e]]++ - G.row[ev1[e]];
        int r2 = fill[ev2[e]]++ - G.row[ev2[e]];
        G.adj[G.row[ev1[e]] + r1] = e;
        G.adj[G.row[ev2[e]] + r2] = e;
        G.rank1[e] = (G.el1[e] == ev1[e]) ? r1 : r2;
        G.rank2[e] = (G.el1[e] == ev1[e]) ? r2 : r1;
    }
    solve_graph(r, threads);
    return r->status;
}

void orc_free(orc_result* r) { delete r; }
const char* orc_error(const orc_result* r) { return r->err.c_str(); }
int orc_status(const orc_result* r) { return r->status; }
int32_t orc_num_nodes(const orc_result* r) { return r->G.Vn; }
int32_t orc_num_edges(const orc_result* r) { return r->G.En; }
int32_t orc_num_points(const orc_result* r) { return (int32_t)r->P.X.size(); }
double orc_size_per_node(const orc_result* r) { return r->P.size_per_node; }

void orc_get_edges(const orc_result* r, int32_t* v1, int32_t* v2, int32_t* lab1, int32_t* lab2,
                   double* Do, double* D) {
    const Graph& G = r->G;
    for (int e = 0; e < G.En; ++e) {
        if (v1) v1[e] = G.ev1[e];
        if (v2) v2[e] = G.ev2[e];
        if (lab1) lab1[e] = G.label[G.el1[e]];
        if (lab2) lab2[e] = G.label[G.el2[e]];
        if (Do) Do[e] = G.Do[e];
        if (D) D[e] = G.D[e];
    }
}
void orc_get_nodes(const orc_result* r, int32_t* label, int32_t* fxy_index) {
    for (int v = 0; v < r->G.Vn; ++v) {
        if (label) label[v] = r->G.label[v];
        if (fxy_index) fxy_index[v] = r->G.fxy[v];
    }
}
void orc_get_F(const orc_result* r, double* F) { std::copy(r->F.begin(), r->F.end(), F); }
void orc_get_x(const orc_result* r, double* x) { std::copy(r->x.begin(), r->x.end(), x); }
double orc_lp_value(const orc_result* r) { return r->lp; }
int32_t orc_max_rank(const orc_result* r) { return r->max_rank; }
void orc_get_stats(const orc_result* r, orc_stats* s) { *s = r->st; }
int32_t orc_get_combs(const orc_result* r, int32_t* comb_size, int32_t* comb_nodes) {
    if (comb_size) std::copy(r->comb_size.begin(), r->comb_size.end(), comb_size);
    if (comb_nodes) std::copy(r->comb_nodes.begin(), r->comb_nodes.end(), comb_nodes);
    return (int32_t)r->comb_size.size();
}
void orc_get_statab(const orc_result* r, int32_t* A, int32_t* B) {
    std::copy(r->statA.begin(), r->statA.end(), A);
    std::copy(r->statB.begin(), r->statB.end(), B);
}
void orc_get_cutoffs(const orc_result* r, double* cutoff, int32_t* stat) {
    for (size_t i = 0; i < r->C.cut.size(); ++i) {
        if (cutoff) cutoff[i] = r->C.cut[i];
        if (stat) stat[i] = r->C.stat[i];
    }
}

int orc_solve_batch(int32_t n_inst, const int64_t* offs, const double* X, const double* Y, int top_k,
                    int cost_mode, int threads, double* lp_out, int32_t* status_out, int64_t* iters_out) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) if (threads > 1)
    for (int b = 0; b < n_inst; ++b) {
        int64_t o = offs[b], n = offs[b + 1] - offs[b];
        std::vector<int32_t> K(n);
        for (int64_t i = 0; i < n; ++i) K[i] = (int32_t)(i + 1);
        orc_result* r = nullptr;
        orc_solve_points(K.data(), X + o, Y + o, (int32_t)n, top_k, cost_mode, ORC_ID_FXY, ORC_KNN_TOPN, 1, &r);
        lp_out[b] = r->lp;
        status_out[b] = r->status;
        if (iters_out) iters_out[b] = r->st.iters_glob + r->st.iters_ef + r->st.iters_repair;
        orc_free(r);
    }
    return ORC_OK;
}

}  // extern "C"
