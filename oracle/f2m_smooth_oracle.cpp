// CPU oracle of the entropically smoothed F2M dual bound -- TEST
// INFRASTRUCTURE ONLY (the reference solves the LP only; this restates the
// definitions that the CUDA path of f2m_b200 implements, in plain FP64 loops).
//
// Graph: the union over points of each point's N nearest neighbours by FP32
// Euclidean distance c = sqrtf(dx*dx + dy*dy) (no FMA), ties by index.
// Node lists are ascending in neighbour index; mirror[s] is the slot of the
// same edge in the neighbour's list.
//
// Bound: with z_e = (u_a + u_b - c_e)/tau and sigma the logistic function,
//   L(u) = 2 sum_v u_v - tau sum_e softplus(z_e)
// is the dual of min c.x + tau sum_e [x ln x + (1-x) ln(1-x)] over the degree-2
// polytope, so L(u) is a lower bound of that smoothed LP for every u.  The
// forward pass runs T damped Jacobi coordinate-ascent steps from u = 0:
//   s_v = the root of sum_{e=(v,w)} sigma((s + u_w - c_e)/tau) = 2,
//   u_v <- (1 - omega) u_v + omega s_v,
// and returns L(u^T).  The backward pass is the exact adjoint of that
// computation (implicit function theorem for each root), giving dL/dc_e and,
// through c_e = |p_a - p_b|, dL/d(coordinates).  At a stationary u,
// dL/dc_e = sigma(z_e), the smoothed x_e.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "f2m_oracle.h"

namespace {

struct SGraph {
    int V = 0;
    std::vector<int64_t> row;
    std::vector<int> nbr, mirror;
    std::vector<float> c;
};

float sdist(float x0, float y0, float x1, float y1) {
    const float dx = x0 - x1, dy = y0 - y1;
    const float q = dx * dx + dy * dy;  // built with -ffp-contract=off
    return std::sqrt(q);
}

SGraph build_graph(const float* x, const float* y, int V, int N) {
    SGraph G;
    G.V = V;
    N = std::min(N, V - 1);
    std::vector<std::vector<int>> adj(V);
    std::vector<std::pair<float, int>> cand(V);
    for (int i = 0; i < V; ++i) {
        int m = 0;
        for (int j = 0; j < V; ++j)
            if (j != i) cand[m++] = {sdist(x[i], y[i], x[j], y[j]), j};
        std::partial_sort(cand.begin(), cand.begin() + N, cand.begin() + m);
        for (int k = 0; k < N; ++k) {
            adj[i].push_back(cand[k].second);
            adj[cand[k].second].push_back(i);
        }
    }
    G.row.assign(V + 1, 0);
    for (int v = 0; v < V; ++v) {
        std::sort(adj[v].begin(), adj[v].end());
        adj[v].erase(std::unique(adj[v].begin(), adj[v].end()), adj[v].end());
        G.row[v + 1] = G.row[v] + (int64_t)adj[v].size();
    }
    G.nbr.resize(G.row[V]);
    G.c.resize(G.row[V]);
    G.mirror.resize(G.row[V]);
    for (int v = 0; v < V; ++v)
        for (size_t k = 0; k < adj[v].size(); ++k) {
            const int w = adj[v][k];
            G.nbr[G.row[v] + k] = w;
            G.c[G.row[v] + k] = sdist(x[v], y[v], x[w], y[w]);
        }
    for (int v = 0; v < V; ++v)
        for (int64_t s = G.row[v]; s < G.row[v + 1]; ++s) {
            const int w = G.nbr[s];
            const int64_t t = std::lower_bound(G.nbr.begin() + G.row[w], G.nbr.begin() + G.row[w + 1], v) -
                              G.nbr.begin();
            G.mirror[s] = (int)t;
        }
    return G;
}

double sigmoid(double z) {
    if (z >= 0) return 1.0 / (1.0 + std::exp(-z));
    const double e = std::exp(z);
    return e / (1.0 + e);
}
double softplus(double z) { return std::max(z, 0.0) + std::log1p(std::exp(-std::fabs(z))); }

// sum_k sigma(z_k) - 2 without cancellation: each term is split into its
// rounding to 0 or 1 (counted exactly) and the small remainder
// m = min(sigma, 1 - sigma) = e/(1+e), e = exp(-|z|), so the tiny residuals
// that decide a root between two well-separated costs keep full relative
// precision.  Also returns sum m (the scale of g) and sum sigma(1 - sigma).
struct LogitSum {
    double g = 0, scale = 0, slope = 0;
};
LogitSum logit_sum(const double* z, int n) {
    LogitSum r;
    int cnt = 0;
    double tail = 0;
    for (int k = 0; k < n; ++k) {
        const double e = std::exp(-std::fabs(z[k]));
        const double m = e / (1.0 + e), big = 1.0 / (1.0 + e);
        if (z[k] >= 0) { ++cnt; tail -= m; } else { tail += m; }
        r.scale += m;
        r.slope += m * big;
    }
    r.g = (double)(cnt - 2) + tail;
    return r;
}

// Root s of sum_k sigma((s - a_k)/tau) = 2: Newton's method from the LP root
// (the midpoint of the 2nd and 3rd smallest a_k), kept inside a bracket by
// bisection, stopped at a relative residual of 1e-14, a step below the
// resolution of s, or a bracket of a few ulps.
double node_root(const double* a, int n, double tau, int max_it) {
    std::vector<double> z(n);
    double m0 = INFINITY, m1 = INFINITY, m2 = INFINITY;
    for (int k = 0; k < n; ++k) {
        const double v = a[k];
        if (v < m0) { m2 = m1; m1 = m0; m0 = v; }
        else if (v < m1) { m2 = m1; m1 = v; }
        else if (v < m2) { m2 = v; }
    }
    double lo = m0 - 40 * tau, hi = m2 + 40 * tau;
    double s = 0.5 * (m1 + m2);  // the LP root; exact when the costs are far apart
    for (int it = 0; it < max_it; ++it) {
        for (int k = 0; k < n; ++k) z[k] = (s - a[k]) / tau;
        const LogitSum r = logit_sum(z.data(), n);
        const double g = r.g, gp = r.slope / tau;
        if (g > 0) hi = s; else lo = s;
        if (g == 0 || std::fabs(g) <= 1e-14 * r.scale) break;
        double sn = (gp > 0) ? s - g / gp : 0.5 * (lo + hi);
        if (std::fabs(sn - s) <= 4e-16 * (1.0 + std::fabs(s))) break;  // step below resolution
        if (!(sn > lo && sn < hi)) sn = 0.5 * (lo + hi);
        if (sn == s || hi - lo <= 4e-16 * (1.0 + std::fabs(s))) break;
        s = sn;
    }
    return s;
}

struct Fwd {
    std::vector<std::vector<double>> u;  // u^0 .. u^T
    std::vector<std::vector<double>> s;  // s^0 .. s^{T-1}
    double L = 0;
};

void jacobi(const SGraph& G, const std::vector<double>& u, double tau, double omega, int max_it,
            std::vector<double>& s_out, std::vector<double>& un) {
    std::vector<double> a;
    for (int v = 0; v < G.V; ++v) {
        const int64_t r0 = G.row[v], r1 = G.row[v + 1];
        a.resize(r1 - r0);
        for (int64_t k = r0; k < r1; ++k) a[k - r0] = (double)G.c[k] - u[G.nbr[k]];
        const double s = node_root(a.data(), (int)(r1 - r0), tau, max_it);
        s_out[v] = s;
        un[v] = (1.0 - omega) * u[v] + omega * s;
    }
}

double bound(const SGraph& G, const std::vector<double>& u, double tau) {
    double su = 0, sp = 0;
    for (int v = 0; v < G.V; ++v) {
        su += 2.0 * u[v];
        for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k)
            if (G.nbr[k] > v) sp += softplus((u[v] + u[G.nbr[k]] - (double)G.c[k]) / tau);
    }
    return su - tau * sp;
}

Fwd forward(const SGraph& G, double tau, int T, double omega, int max_it) {
    Fwd F;
    F.u.assign(T + 1, std::vector<double>(G.V, 0.0));
    F.s.assign(T, std::vector<double>(G.V, 0.0));
    for (int t = 0; t < T; ++t) jacobi(G, F.u[t], tau, omega, max_it, F.s[t], F.u[t + 1]);
    F.L = bound(G, F.u[T], tau);
    return F;
}

// Adjoint: dL/dc per slot (both slots of an edge carry the edge's total).
std::vector<double> backward_c(const SGraph& G, const Fwd& F, double tau, double omega) {
    const int V = G.V, T = (int)F.s.size();
    const int64_t S = G.row[V];
    std::vector<double> lam(V), lam2(V), gc(S, 0.0), q(S);
    const std::vector<double>& uT = F.u[T];
    std::vector<double> sgT(S);
    std::vector<double> z;
    for (int v = 0; v < V; ++v) {
        z.clear();
        for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k) {
            z.push_back((uT[v] + uT[G.nbr[k]] - (double)G.c[k]) / tau);
            sgT[k] = sigmoid(z.back());
        }
        lam[v] = -logit_sum(z.data(), (int)z.size()).g;  // 2 - sum sigma
    }
    for (int t = T - 1; t >= 0; --t) {
        const std::vector<double>& u = F.u[t];
        const std::vector<double>& s = F.s[t];
        for (int v = 0; v < V; ++v) {
            double D = 0;
            for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k) {
                const double e = std::exp(-std::fabs((s[v] + u[G.nbr[k]] - (double)G.c[k]) / tau));
                q[k] = (e / (1.0 + e)) * (1.0 / (1.0 + e)) / tau;
                D += q[k];
            }
            const double mu = D > 0 ? omega * lam[v] / D : 0.0;  // D == 0: every sigma saturated
            for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k) {
                q[k] *= mu;
                gc[k] += q[k];
            }
        }
        for (int w = 0; w < V; ++w) {
            double l = (1.0 - omega) * lam[w];
            for (int64_t k = G.row[w]; k < G.row[w + 1]; ++k) l -= q[G.mirror[k]];
            lam2[w] = l;
        }
        lam.swap(lam2);
    }
    std::vector<double> dc(S);
    for (int v = 0; v < V; ++v)
        for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k) dc[k] = sgT[k] + gc[k] + gc[G.mirror[k]];
    return dc;
}

}  // namespace

extern "C" {

int orc_smooth_graph(const float* x, const float* y, int32_t n, int32_t top_k, int64_t* row,
                     int32_t* nbr, float* c, int64_t cap) {
    if (n < 4 || top_k < 3) return -1;
    const SGraph G = build_graph(x, y, n, top_k);
    const int64_t S = G.row[n];
    if (row) std::copy(G.row.begin(), G.row.end(), row);
    if (nbr && S <= cap) std::copy(G.nbr.begin(), G.nbr.end(), nbr);
    if (c && S <= cap) std::copy(G.c.begin(), G.c.end(), c);
    return (int)S;
}

// Forward (and, when an output gradient is given, backward) of the bound.
// The graph is built from (gx, gy) when given, else from (x, y); edge costs
// are the distances of (x, y) on that graph, or `c_override` (S entries).
// Fixing the graph this way keeps it constant under finite differences.
int orc_smooth_bound(const float* x, const float* y, int32_t n, int32_t top_k, double tau,
                     int32_t iters, double omega, int32_t newton_max, const float* gx,
                     const float* gy, const float* c_override, double* L, double* dLdx,
                     double* dLdy, double* dLdc) {
    if (n < 4 || top_k < 3 || !(tau > 0) || iters < 0) return ORC_ERR_INPUT;
    SGraph G = build_graph(gx ? gx : x, gy ? gy : y, n, top_k);
    for (int v = 0; v < n; ++v)
        for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k)
            G.c[k] = c_override ? c_override[k] : sdist(x[v], y[v], x[G.nbr[k]], y[G.nbr[k]]);
    const Fwd F = forward(G, tau, iters, omega, newton_max);
    *L = F.L;
    if (!dLdx && !dLdy && !dLdc) return ORC_OK;
    const std::vector<double> dc = backward_c(G, F, tau, omega);
    if (dLdc) std::copy(dc.begin(), dc.end(), dLdc);
    for (int v = 0; v < n; ++v) {
        double gx = 0, gy = 0;
        for (int64_t k = G.row[v]; k < G.row[v + 1]; ++k) {
            const int w = G.nbr[k];
            const double ce = (double)G.c[k];
            if (ce == 0) continue;
            gx += dc[k] * ((double)x[v] - (double)x[w]) / ce;
            gy += dc[k] * ((double)y[v] - (double)y[w]) / ce;
        }
        if (dLdx) dLdx[v] = gx;
        if (dLdy) dLdy[v] = gy;
    }
    return ORC_OK;
}

}  // extern "C"
