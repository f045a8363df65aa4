// f2m_b200 host runtime: the C ABI of include/f2m.h.
//
// Device work (kNN, graph build, descent, partitions, combs, primal) runs in
// the kernels of f2m_kernels.cu.  The host side mirrors the reference's own
// host stages: TSPLIB parsing (FXY.hpp:186-309), the graph assembly in the
// reference's node order (graph_tour.hpp:28-110), the host comb check with
// its Ax=b solver (graph_cuda_comb.hpp:121-147, E_thread.cpp, V_thread.cpp,
// comb_thread.cpp, Ax_b.cpp), the repair-loop driver (graph_cuda.cu:69-126)
// and the output files (graph_tour.hpp:186-241, FXY.hpp:146-183).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <memory>
#include <atomic>
#include <mutex>
#include <thread>
#include <numeric>
#include <string>
#include <unordered_map>
#include <type_traits>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "f2m_internal.h"

using namespace f2m;

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */
namespace {

// NVTX range for the lifetime of a scope (visible in Nsight timelines; a
// no-op without a tool attached)
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

struct Arena {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    template <class T>
    T* take(size_t n) {
        size_t off = (used + 255) & ~(size_t)255;
        used = off + n * sizeof(T);
        return base ? reinterpret_cast<T*>(base + off) : nullptr;
    }
};

}  // namespace

struct f2m_ctx {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int64_t launches = 0;
    char* dev = nullptr;
    size_t dev_cap = 0;
    char* pinned = nullptr;
    size_t pinned_cap = 0;
    // CUDA events around the phases of the last batched call
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool timed = false;
    Batch last{};  // pointers of the last batched call (for the work counters)
    cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[4] = {nullptr, nullptr, nullptr, nullptr};
    // CUDA graph of the smoothed bound's per-step launches, replayed while the
    // call's shape (sizes, parameters, arena) repeats
    cudaGraphExec_t sgraph = nullptr;
    std::vector<int64_t> skey;
    int64_t sgraph_launches = 0;
    // work and kernel time of the last smoothed-bound call (persistent path)
    int64_t smooth_terms = -1;
    float smooth_ms = 0.f;
};

namespace {

f2m_status fail(f2m_ctx* c, f2m_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}
f2m_status cuda_fail(f2m_ctx* c, cudaError_t e, const char* where) {
    return fail(c, F2M_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define F2M_CUDA(call)                                                  \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);        \
    } while (0)

cudaError_t ensure_device(f2m_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->dev_cap) return cudaSuccess;
    if (ctx->dev) cudaFree(ctx->dev);
    ctx->dev = nullptr;
    ctx->dev_cap = 0;
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&ctx->dev, want);
    if (e != cudaSuccess) return e;
    ctx->dev_cap = want;
    return cudaSuccess;
}
cudaError_t ensure_pinned(f2m_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->pinned_cap) return cudaSuccess;
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_cap = 0;
    size_t want = bytes + bytes / 8 + 4096;
    cudaError_t e = cudaHostAlloc(&ctx->pinned, want, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    ctx->pinned_cap = want;
    return cudaSuccess;
}

DevParams to_dev(const f2m_params& p) {
    DevParams d;
    d.error_B = p.error_B;
    d.porog = p.error_B * p.error_B_comb;  // graph_cuda_comb.hpp:156
    d.glob_tol = p.glob_tol;
    d.ef_thr = p.ef_thr;
    d.comb_thr = p.comb_thr;
    d.glob_K = p.glob_K;
    d.glob_rounds = p.glob_rounds;
    d.glob_inner = p.glob_inner;
    d.factor0 = p.factor0;
    d.factor_step = p.factor_step;
    d.factor_cap = p.factor_cap;
    d.max_rounds = p.max_rounds;
    d.fix_rounds = p.fix_rounds;
    d.fix_factor = p.fix_factor;
    d.check_every = p.check_every;
    d.frozen_iters = p.frozen_iters;
    d.ef_small_deg = p.ef_small_deg;
    d.ef_min = p.ef_min;
    d.max_iters = p.max_iters;
    d.spin_limit = p.grid_spin_limit > 0 ? p.grid_spin_limit : 1;
    return d;
}

/* ------------------------------------------------------------------ */
/* batch plan + device layout                                           */
/* ------------------------------------------------------------------ */
constexpr int kChunk = 256;
constexpr int32_t kHostDedupPoints = 16384;

struct Plan {
    int32_t n_inst = 0;
    int64_t n_total = 0;
    int32_t max_n = 0;
    int32_t N = 0;
    std::vector<int32_t> chunk_inst, chunk_start, order;
    // order[seg[c] .. seg[c] + cnt[c]) are the instances of solver class c
    std::vector<int32_t> seg, cnt;
    std::vector<int32_t> class_vcap;
    int64_t S_cap = 0;
};

void make_plan(Plan& pl, int32_t n_inst, const int64_t* offs, int32_t N) {
    pl.n_inst = n_inst;
    pl.N = N;
    pl.n_total = offs[n_inst] - offs[0];
    pl.max_n = 0;
    pl.chunk_inst.clear();
    pl.chunk_start.clear();
    for (int32_t b = 0; b < n_inst; ++b) {
        const int32_t n = (int32_t)(offs[b + 1] - offs[b]);
        pl.max_n = std::max(pl.max_n, n);
        for (int32_t s = 0; s < n; s += kChunk) {
            pl.chunk_inst.push_back(b);
            pl.chunk_start.push_back(s);
        }
    }
    pl.order.resize(n_inst);
    std::iota(pl.order.begin(), pl.order.end(), 0);
    std::stable_sort(pl.order.begin(), pl.order.end(), [&](int a, int b) {
        return offs[a + 1] - offs[a] > offs[b + 1] - offs[b];
    });
    // largest first, so the classes are contiguous from the largest down
    const int nc = solve_num_classes();
    pl.seg.assign(nc, 0);
    pl.cnt.assign(nc, 0);
    pl.class_vcap.assign(nc, 4);
    for (int32_t b = 0; b < n_inst; ++b) {
        const int32_t n = (int32_t)(offs[b + 1] - offs[b]);
        const int c = solve_class_of(n);
        pl.cnt[c]++;
        pl.class_vcap[c] = std::max(pl.class_vcap[c], n);
    }
    // order holds class nc-1 first (largest instances), then nc-2, ...
    int32_t acc = 0;
    for (int c = nc - 1; c >= 0; --c) { pl.seg[c] = acc; acc += pl.cnt[c]; }
    const int64_t Neff = std::min<int64_t>(N, std::max<int32_t>(pl.max_n - 1, 1));
    pl.S_cap = 2 * Neff * std::max<int64_t>(pl.n_total, 1);
}

// Carves every buffer of a batched call out of one arena.  With A.base ==
// nullptr it only measures.
void carve_grid(Arena& A, GridState& G, int64_t n, int64_t S) {
    G.Ha = A.take<double>(n);
    G.Hb = A.take<double>(n);
    G.efc = A.take<int32_t>(n);
    G.gD = A.take<double>(S);
    G.gW = A.take<uint32_t>(S);
    G.scratch = A.take<int32_t>(2 * n);
    G.irr = A.take<int32_t>(n);
    G.bar = A.take<unsigned>(4);
    G.err = A.take<int32_t>(4);
    G.axb_used = A.take<unsigned long long>(2);
    G.part = A.take<double>(2 * kGridMaxCtas);
    G.partl = A.take<long long>(2 * kGridMaxCtas);
    G.own = A.take<int32_t>(n);
    G.owner = A.take<int32_t>(n);
    G.rd = A.take<int32_t>(n);
    G.prog = A.take<unsigned>(kGridMaxCtas);
    G.nbm = A.take<unsigned>((int64_t)kGridMaxCtas * kGridNbWords);
    G.okey = A.take<unsigned long long>(n);
    G.okey2 = A.take<unsigned long long>(n);
    G.otmp_bytes = grid_order_temp_bytes(n);
    G.otmp = A.take<unsigned char>(G.otmp_bytes);
}

void carve(Arena& A, Batch& B, const Plan& pl, bool own_inputs, int64_t** deg, int64_t** scan_scratch,
           int32_t** d_chunk_inst, int32_t** d_chunk_start, int32_t** d_order, int64_t n_chunks = -1) {
    if (n_chunks < 0) n_chunks = (int64_t)pl.chunk_inst.size();
    const int64_t n = std::max<int64_t>(pl.n_total, 1);
    const int32_t ni = pl.n_inst;
    const int64_t S = std::max<int64_t>(pl.S_cap, 1);
    const int64_t nN = n * pl.N;
    B.n_inst = ni;
    B.N = pl.N;
    B.N_cut = pl.N;
    B.n_total = (int32_t)pl.n_total;
    if (own_inputs) {
        B.offs = A.take<int64_t>(ni + 1);
        B.X_in = A.take<double>(n);
        B.Y_in = A.take<double>(n);
    }
    B.K_in = nullptr;
    B.Pr = A.take<double2>(n);
    B.P = A.take<double2>(n);
    B.K = A.take<int32_t>(n);
    B.dup_of = A.take<int32_t>(n);
    B.Vn = A.take<int32_t>(ni);
    B.spn = A.take<double>(ni);
    B.dmin_bits = A.take<unsigned long long>(ni);
    B.status = A.take<int32_t>(ni);
    B.gx0 = A.take<double>(ni);
    B.gy0 = A.take<double>(ni);
    B.gh = A.take<double>(ni);
    B.gnx = A.take<int32_t>(ni);
    B.gny = A.take<int32_t>(ni);
    B.pcell = A.take<int32_t>(n);
    B.cellcnt = A.take<int64_t>(n + 1);
    B.cellstart = A.take<int64_t>(n + 1);
    B.cellcur = A.take<int32_t>(n);
    B.sidx = A.take<int32_t>(n);
    B.spt = A.take<double2>(n);
    B.cut = A.take<double>(n);
    B.stat = A.take<int32_t>(n);
    B.ntop = A.take<int32_t>(n);
    B.top_nbr = A.take<int32_t>(nN);
    B.top_cost = A.take<double>(nN);
    B.top_em = A.take<int32_t>(nN);
    B.top_oth = A.take<int32_t>(nN);
    B.rev = A.take<int32_t>(n);
    B.cursor = A.take<int32_t>(n);
    B.tdup = A.take<uint8_t>(nN);
    B.row = A.take<int64_t>(n + 1);
    B.s_nbr = A.take<int32_t>(S);
    B.s_cost = A.take<double>(S);
    B.s_em = A.take<int32_t>(S);
    B.s_oth = A.take<int32_t>(S);
    B.slot = A.take<Slot>(S);
    B.perm = A.take<uint16_t>(S);
    B.pslot = A.take<Slot>(S);
    B.mirror = A.take<int32_t>(S);
    B.efD = A.take<double>(S);
    B.efN = A.take<uint16_t>(S);
    B.xcode = A.take<uint8_t>(S);
    B.xval = A.take<float>(S);
    B.clab = A.take<int32_t>(n);
    B.cirr = A.take<int32_t>(n);
    B.selD = A.take<double>(S);
    B.selW = A.take<uint16_t>(S);
    B.sel_stride = S / n;
    B.S_cap = S;
    B.F = A.take<double>(n);
    B.efcnt = A.take<int32_t>(n);
    B.ccnt = A.take<int32_t>(n);
    B.shift = A.take<double>(n);
    B.lp = A.take<double>(ni);
    B.n_edges = A.take<int32_t>(ni);
    B.n_combs = A.take<int32_t>(ni);
    B.n_irr = A.take<int32_t>(ni);
    B.max_rank = A.take<int32_t>(ni);
    B.deg_viol = A.take<int32_t>(ni);
    B.iters = A.take<int64_t>(ni);
    B.work_nodes = A.take<int64_t>(ni);
    B.work_slots = A.take<int64_t>(ni);
    B.work_pad = A.take<int64_t>(ni);
    B.checks = A.take<int32_t>(ni);
    B.max_grad = A.take<double>(ni);
    B.dual = A.take<double>(ni);
    *d_chunk_inst = A.take<int32_t>(n_chunks + 1);
    *d_chunk_start = A.take<int32_t>(n_chunks + 1);
    *d_order = A.take<int32_t>(ni + 1);
    B.chunk_inst = *d_chunk_inst;
    B.chunk_start = *d_chunk_start;
    B.n_chunks = (int32_t)n_chunks;
    B.order = *d_order;
    B.n_items = ni;
    B.queue = A.take<int32_t>(8);
    *deg = A.take<int64_t>(n + 1);
    *scan_scratch = A.take<int64_t>(scan_scratch_elems(n) + 1);
}


/* ------------------------------------------------------------------ */
/* host comb check and repair loop (the reference's host stage)          */
/* ------------------------------------------------------------------ */
// One instance pulled back to the host, in the reference's data model.
// std::allocator whose value-less construct leaves trivially constructible
// elements uninitialised: resize() of the large per-edge arrays then skips a
// serial zero fill of memory that the parallel fills overwrite anyway (every
// resize of these arrays is followed by a write of every element).
template <class T>
struct NoFillAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoFillAlloc<U>;
    };
    NoFillAlloc() = default;
    template <class U>
    NoFillAlloc(const NoFillAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new ((void*)p) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using hvec = std::vector<T, NoFillAlloc<T>>;

struct HostInst {
    int V = 0, E = 0;
    std::vector<int> label;            // internal id -> TSPLIB label
    std::vector<int64_t> row;          // V+1 local slot offsets
    std::vector<int> nbr;              // per slot
    std::vector<double> Dn, cost;      // per slot
    std::vector<uint16_t> perm;        // per slot (current list order)
    std::vector<int> mirror;           // per slot
    std::vector<int> slot_edge;        // per slot -> edge id
    hvec<int> ev1, ev2, el1, el2;      // per edge
    std::vector<int> rank1, rank2;     // per edge
    hvec<double> eD, eDo;              // per edge
    std::vector<double> F;
    std::vector<int> efcnt, ccnt;
    double dmin = 0;
};

// Edge ids in the reference's global order: slots with nbr>v, sorted by the
// candidate key (cost, emitter, partner) (FXY.hpp:100-101, graph_tour.hpp:28-90).
// fn(begin, end) over [0, n) in contiguous ranges on up to 32 host threads
// (inline below 20,000 items)
template <class Fn>
void parallel_for(int64_t n, Fn fn, int64_t serial_below = 20000) {
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t T = (n < serial_below) ? 1 : std::min<int64_t>(std::min<int64_t>(hw, 32), n);
    if (T <= 1) { fn((int64_t)0, n); return; }
    std::vector<std::thread> pool;
    for (int64_t t = 1; t < T; ++t) pool.emplace_back(fn, n * t / T, n * (t + 1) / T);
    fn((int64_t)0, n / T);
    for (auto& th : pool) th.join();
}

// std::sort of a large array as sorted chunks merged pairwise, each level's
// merges side by side (the keys here are unique, so the order is the same)
template <class T, class Less>
void parallel_sort(std::vector<T>& a, Less less, int64_t serial_below = 200000) {
    const int64_t n = (int64_t)a.size();
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    int64_t parts = 1;
    while (parts * 2 <= std::min<int64_t>(hw, 32)) parts *= 2;
    if (n < serial_below || parts < 2) { std::sort(a.begin(), a.end(), less); return; }
    std::vector<int64_t> b(parts + 1);
    for (int64_t p = 0; p <= parts; ++p) b[p] = n * p / parts;
    {
        std::vector<std::thread> pool;
        for (int64_t p = 1; p < parts; ++p)
            pool.emplace_back([&, p] { std::sort(a.begin() + b[p], a.begin() + b[p + 1], less); });
        std::sort(a.begin() + b[0], a.begin() + b[1], less);
        for (auto& th : pool) th.join();
    }
    std::vector<T> tmp(n);
    for (int64_t w = 1; w < parts; w *= 2) {
        const int64_t pairs = parts / (2 * w);
        std::vector<std::thread> pool;
        for (int64_t q = 0; q < pairs; ++q)
            pool.emplace_back([&, q] {
                const int64_t l = b[2 * w * q], m = b[2 * w * q + w], r = b[2 * w * (q + 1)];
                std::merge(a.begin() + l, a.begin() + m, a.begin() + m, a.begin() + r, tmp.begin() + l, less);
            });
        for (auto& th : pool) th.join();
        a.swap(tmp);
    }
}

// get_KXY's rounding and de-duplication (FXY.hpp:252-267): coordinates
// rounded to 1e-3 and the first occurrence of each rounded point kept, in
// input order.  A sort of the rounded points (ties by input index) finds the
// repeats instead of the reference's nested hash maps; +0 and -0 compare
// equal and a point with a NaN coordinate is never a repeat, as there.
void host_dedup_points(const double* x, const double* y, const int32_t* labels, int32_t n,
                       std::vector<double>& hx, std::vector<double>& hy, std::vector<int32_t>& hl) {
    std::vector<double> rx(n), ry(n);
    parallel_for(n, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
            double xx = std::round(x[i] * 1000), yy = std::round(y[i] * 1000);
            rx[i] = xx / 1000;
            ry[i] = yy / 1000;
        }
    });
    auto nanp = [&](int32_t i) { return rx[i] != rx[i] || ry[i] != ry[i]; };
    std::vector<int32_t> idx(n);
    for (int32_t i = 0; i < n; ++i) idx[i] = i;
    parallel_sort(idx, [&](int32_t a, int32_t b) {
        const bool na = nanp(a), nb = nanp(b);
        if (na != nb) return nb;
        if (!na) {
            if (rx[a] != rx[b]) return rx[a] < rx[b];
            if (ry[a] != ry[b]) return ry[a] < ry[b];
        }
        return a < b;
    }, 50000);
    std::vector<char> dup(n, 0);
    for (int32_t k = 1; k < n; ++k) {
        const int32_t a = idx[k - 1], b = idx[k];
        if (!nanp(a) && !nanp(b) && rx[a] == rx[b] && ry[a] == ry[b]) dup[b] = 1;
    }
    hx.clear();
    hy.clear();
    hl.clear();
    for (int32_t i = 0; i < n; ++i) {
        if (dup[i]) continue;
        hx.push_back(rx[i]);
        hy.push_back(ry[i]);
        hl.push_back(labels ? labels[i] : i + 1);
    }
}

// Host stage times of one call, printed to stderr when F2M_HOST_TIMING is
// set (the device phases have their own CUDA-event timers).
struct StageClock {
    bool on = std::getenv("F2M_HOST_TIMING") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    std::string line;
    void mark(const char* name) {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        char buf[64];
        std::snprintf(buf, sizeof(buf), " %s=%.2f", name, std::chrono::duration<double, std::milli>(now - t).count());
        line += buf;
        t = now;
    }
    ~StageClock() {
        if (on && !line.empty()) std::fprintf(stderr, "f2m host stages (ms):%s\n", line.c_str());
    }
};

template <class SlotOf>
void fill_edges(HostInst& H, int64_t E, SlotOf slot_of);

void number_edges(HostInst& H, const std::vector<int>& em, const std::vector<int>& oth) {
    Range rg("f2m number edges");
    struct K { double c; int e, o; int v; int64_t s; };
    // slots with nbr > v, numbered per node, filled side by side
    std::vector<int64_t> first(H.V + 1, 0);
    parallel_for(H.V, [&](int64_t v0, int64_t v1) {
        for (int64_t v = v0; v < v1; ++v) {
            int64_t c = 0;
            for (int64_t a = H.row[v]; a < H.row[v + 1]; ++a) c += H.nbr[a] > v;
            first[v + 1] = c;
        }
    });
    for (int v = 0; v < H.V; ++v) first[v + 1] += first[v];
    std::vector<K> ks(first[H.V]);
    parallel_for(H.V, [&](int64_t v0, int64_t v1) {
        for (int64_t v = v0; v < v1; ++v) {
            int64_t q = first[v];
            for (int64_t a = H.row[v]; a < H.row[v + 1]; ++a)
                if (H.nbr[a] > v) ks[q++] = K{H.cost[a], em[a], oth[a], (int)v, a};
        }
    });
    parallel_sort(ks, [](const K& x, const K& y) {
        if (x.c != y.c) return x.c < y.c;
        if (x.e != y.e) return x.e < y.e;
        return x.o < y.o;
    });
    fill_edges(H, (int64_t)ks.size(), [&](int64_t e) { return ks[e].s; });
}

// The same numbering from the edge order computed on the device
// (launch_edge_order): ord[e] is the slot of edge e in its lower-id
// endpoint's list.
void number_edges_ordered(HostInst& H, const uint32_t* ord, int64_t E) {
    Range rg("f2m number edges");
    fill_edges(H, E, [&](int64_t e) { return (int64_t)ord[e]; });
}

// Edge arrays of H from the edges in order, each given by its slot in the
// lower-id endpoint's list (the endpoint is found through the mirror slot).
template <class SlotOf>
void fill_edges(HostInst& H, int64_t E, SlotOf slot_of) {
    H.E = (int)E;
    H.slot_edge.assign(H.nbr.size(), -1);
    H.ev1.resize(H.E); H.ev2.resize(H.E); H.el1.resize(H.E); H.el2.resize(H.E);
    H.rank1.resize(H.E); H.rank2.resize(H.E); H.eD.resize(H.E); H.eDo.resize(H.E);
    parallel_for(H.E, [&](int64_t e0, int64_t e1) {
    for (int64_t e = e0; e < e1; ++e) {
        const int64_t a = slot_of(e);
        const int u = H.nbr[a];
        const int v = H.nbr[H.row[u] + H.mirror[a]];
        H.slot_edge[a] = e;
        H.slot_edge[H.row[u] + H.mirror[a]] = e;
        H.ev1[e] = v; H.ev2[e] = u;
        H.eD[e] = H.Dn[a]; H.eDo[e] = H.cost[a];
        const int rv = (int)(a - H.row[v]), ru = H.mirror[a];
        if (H.label[v] < H.label[u]) { H.el1[e] = v; H.el2[e] = u; H.rank1[e] = rv; H.rank2[e] = ru; }
        else { H.el1[e] = u; H.el2[e] = v; H.rank1[e] = ru; H.rank2[e] = rv; }
    }
    });
}

struct HostCheck {
    HostInst& H;
    double vb;
    std::vector<std::vector<int>> node_edges, eA, eB;
    std::vector<int> sA, sB;
    std::vector<int> irrB;  // comb_IRREGULAR_B, kept across checks (F2M.h:166)
    struct CombH {
        std::unordered_map<int, int> nodes;
        std::unordered_map<int, float> XB;
        int STATUS = 1, AxB_status = 1;
    };
    std::vector<CombH> Combs;
    std::vector<std::vector<int>> comb_V;  // BFS order
    int irr_a = 0;

    HostCheck(HostInst& h, double band) : H(h), vb(band) {
        node_edges.resize(H.V);
        parallel_for(H.V, [&](int64_t v0, int64_t v1) {
            for (int64_t v = v0; v < v1; ++v)
                node_edges[v].assign(H.slot_edge.begin() + H.row[v], H.slot_edge.begin() + H.row[v + 1]);
        });
    }
    double dgpu(int64_t a, int v) const {  // cuda_recompute_Edges
        const int u = H.nbr[a];
        return (v < u) ? (H.Dn[a] + 0.5 * H.F[v]) + 0.5 * H.F[u] : (H.Dn[a] + 0.5 * H.F[u]) + 0.5 * H.F[v];
    }
    // get_cuda_comb_size/fill BFS order from each component's smallest id
    // over the comb prefix (graph_cuda_comb.hpp:258-392)
    void extract_combs() {
        comb_V.clear();
        std::vector<int> seen(H.V, 0);
        std::vector<int> eseen(H.E, 0);
        for (int r = 0; r < H.V; ++r) {
            if (seen[r]) continue;
            std::vector<int> fn{r}, A{r}, Bn;
            bool any = false, lower = false;
            std::vector<int> touched{r};
            seen[r] = 1;
            while (!A.empty() && !lower) {
                Bn.clear();
                for (int lA : A) {
                    const int64_t r0 = H.row[lA];
                    for (int k = 0; k < H.ccnt[lA]; ++k) {
                        const int64_t a = r0 + H.perm[r0 + k];
                        const double d = dgpu(a, lA);
                        if (d >= -vb && d <= vb) {
                            any = true;
                            const int v = H.nbr[a];
                            if (v < r) { lower = true; break; }
                            if (!seen[v]) { seen[v] = 1; touched.push_back(v); Bn.push_back(v); fn.push_back(v); }
                        }
                    }
                    if (lower) break;
                }
                std::swap(A, Bn);
            }
            if (lower) {
                for (int t : touched) if (t != r) seen[t] = 0;  // revisit from its own root later
                seen[r] = 1;
                continue;
            }
            if (any) comb_V.push_back(fn);
        }
    }
    // Ax_b (Ax_b.cpp:19-158)
    struct AxB {
        std::vector<std::vector<int>> Ai, Av;
        std::vector<int> b;
        std::vector<double> d, Aj, x, x_grad, b_grad;
        double d_max_error = 0;
        int go_max = 0, i_count = 0, j_count = 0;
        explicit AxB(const std::vector<int>& A) {
            int j = 0, norm = 0;
            std::vector<int> Aij, Avj;
            for (size_t k = 0; k + 1 < A.size(); k += 2) {
                const int i = A[k], v = A[k + 1];
                if (!(i >= -1)) break;
                if (i > i_count) i_count = i;
                if (i == -1) {
                    b.push_back(v);
                    Aj.push_back(std::sqrt((double)norm));
                    norm = 0;
                    j++;
                    Ai.push_back(Aij); Av.push_back(Avj);
                    Aij.clear(); Avj.clear();
                } else {
                    Aij.push_back(i); Avj.push_back(v);
                    norm += v * v;
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
                for (size_t j = 0; j < Ai.size(); j++) b_grad[j] = ax((int)j, x_grad);
                double gg = 0, gd = 0;
                for (size_t j = 0; j < b_grad.size(); j++) gg += b_grad[j] * b_grad[j];
                for (size_t j = 0; j < d.size(); j++) gd += d[j] * b_grad[j];
                const double alfa = -gd / gg;
                for (size_t j = 0; j < x.size(); j++) x[j] += x_grad[j] * alfa;
            }
        }
    };
    // host_combs_check (graph_cuda_comb.hpp:121-147)
    int check() {
        const int E = H.E;
        std::vector<double> dcpu(E);
        parallel_for(E, [&](int64_t e0, int64_t e1) {
            for (int64_t e = e0; e < e1; ++e)  // E_thread.cpp:39
                dcpu[e] = H.eD[e] + H.F[H.el1[e]] / 2 + H.F[H.el2[e]] / 2;
        });
        eA.assign(H.V, {});
        eB.assign(H.V, {});
        sA.assign(H.V, 0);
        sB.assign(H.V, 0);
        parallel_for(H.V, [&](int64_t v0, int64_t v1) {
            for (int64_t v = v0; v < v1; ++v) {  // node::resort + node::get_statusAB
                auto& ed = node_edges[v];
                std::sort(ed.begin(), ed.end(), [&](int a, int b) { return dcpu[a] < dcpu[b]; });
                for (int e : ed) {
                    if (dcpu[e] < vb) {
                        if (dcpu[e] > -vb) { sB[v]++; eB[v].push_back(e); }
                        else { sA[v]++; eA[v].push_back(e); }
                    } else break;
                }
            }
        });
        extract_combs();
        Combs.clear();
        Combs.resize(comb_V.size());
        // combs are independent: each is built and solved by one thread, in
        // the reference's order inside the comb (its maps' insertion order,
        // which the Ax=b rows follow)
        parallel_for((int64_t)comb_V.size(), [&](int64_t c0, int64_t c1) {
            for (int64_t c = c0; c < c1; ++c) {  // COMB_thread + solve_simple
                auto& C = Combs[c];
                for (int v : comb_V[c]) C.nodes[v]++;
                for (auto& kv : C.nodes)
                    if (4 - 2 * sA[kv.first] - sB[kv.first] != 0) { C.STATUS = -1; break; }
                if (C.STATUS == 1)
                    for (auto& kv : C.nodes)
                        for (int e : eB[kv.first]) C.XB[e] = 0.5f;
            }
        }, 256);
        std::vector<int> irrA;
        for (size_t c = 0; c < comb_V.size(); ++c)
            if (Combs[c].STATUS != 1) irrA.push_back((int)c);
        irr_a = (int)irrA.size();
        if (!irrA.empty()) {
            parallel_for((int64_t)irrA.size(), [&](int64_t j0, int64_t j1) {
            for (int64_t jj = j0; jj < j1; ++jj) {  // comb::solve_AxB (comb_thread.cpp:272-304)
                const int c = irrA[jj];
                auto& C = Combs[c];
                std::vector<int> rows;
                std::unordered_map<int, int> mapX, mapXR;
                int countX = 0;
                for (auto& kv : C.nodes) {
                    for (int e : eB[kv.first]) {
                        int i;
                        auto it = mapX.find(e);
                        if (it != mapX.end()) i = it->second;
                        else { i = countX; mapXR[i] = e; mapX[e] = i; countX++; }
                        rows.push_back(i);
                        rows.push_back(1);
                    }
                    rows.push_back(-1);
                    rows.push_back(2 - (int)eA[kv.first].size());
                }
                AxB ab(rows);
                ab.solve();
                C.AxB_status = ab.go_max;
                for (size_t j = 0; j < ab.x.size(); j++) C.XB[mapXR[(int)j]] = (float)ab.x[j];
            }
            }, 2);
            irrB.clear();  // get_comb_IRREGULAR_B
            for (size_t c = 0; c < Combs.size(); ++c)
                if (Combs[c].AxB_status == 0) irrB.push_back((int)c);
        }
        return (int)irrB.size();
    }
    // shift_comb_IRREGULAR_B (graph_cuda_comb.hpp:484-522) with the device A/B
    // rule (cuda_get_Nodes_StatAB, graph_cuda_grad.hpp:274-295)
    void shifts(double shiftV, int type, std::vector<double>& sh) const {
        sh.assign(H.V, 0.0);
        for (int c : irrB) {
            if (c < 0 || c >= (int)comb_V.size()) continue;  // stale index
            for (int nid : comb_V[c]) {
                const int64_t r0 = H.row[nid];
                int A = 0, B = 0;
                for (int k = 0; k < H.ccnt[nid]; ++k) {
                    const double d = dgpu(r0 + H.perm[r0 + k], nid);
                    if (d < -vb) A++;
                    else if (d < vb) B++;
                }
                const int v = 4 - 2 * A - B;
                if (v != 0) {
                    sh[nid] += shiftV * (v > 0 ? 1 : -1);
                    if (type == 1) break;
                }
            }
        }
    }
};

}  // namespace

/* ------------------------------------------------------------------ */
/* result object                                                        */
/* ------------------------------------------------------------------ */
struct f2m_result {
    int32_t status = F2M_OK;
    std::string err;
    HostInst H;
    hvec<double> x;                      // per edge
    std::unordered_map<int, double> X;   // graph::X in insertion order
    double lp = NAN;
    int32_t max_rank = 0;
    double seconds = 0;
    f2m_stats st{};
    // inputs kept for the output files
    std::vector<int> dup_label_of;       // per input point: label of the kept copy or -1
    std::vector<int> in_label;
};

namespace {

/* ------------------------------------------------------------------ */
/* one batched device pass                                              */
/* ------------------------------------------------------------------ */
struct DevCall {
    Plan pl;
    Batch B{};
    GridState G{};
    bool grid = false;      // the single large instance runs on the grid-wide solver
    bool spatial = true;    // the grid solver's nodes can be ordered by their points (node = point)
    int64_t* deg = nullptr;
    int64_t* scan = nullptr;
    int32_t *ci = nullptr, *cs = nullptr, *ord = nullptr;
    EdgeSort es{};          // device edge order buffers (single-instance calls)
    bool has_es = false;
};

void carve_edge_sort(Arena& A, EdgeSort& E, int64_t S) {
    E.k1 = A.take<unsigned long long>(S);
    E.k2 = A.take<unsigned long long>(S);
    E.v1 = A.take<uint32_t>(S);
    E.v2 = A.take<uint32_t>(S);
    E.tmp_bytes = edge_order_temp_bytes(S);
    E.tmp = A.take<unsigned char>(E.tmp_bytes);
    E.xout = A.take<double>((S * 20 + 7) / 8);  // E = S/2 edges x 40 bytes
}

f2m_status setup_call(f2m_ctx* ctx, DevCall& C, int32_t n_inst, const int64_t* h_offs, int32_t top_k,
                      const f2m_params& prm, bool own_inputs) {
    make_plan(C.pl, n_inst, h_offs, top_k);
    C.grid = C.pl.max_n > solve_max_nodes() || (prm.solver == 2 && n_inst == 1);
    if (C.grid && n_inst > 1)
        return fail(ctx, F2M_ERR_CAPACITY, "batched instances are limited to " +
                                               std::to_string(solve_max_nodes()) +
                                               " points each; solve larger ones one at a time");
    Arena A;
    C.has_es = n_inst == 1;
    carve(A, C.B, C.pl, own_inputs, &C.deg, &C.scan, &C.ci, &C.cs, &C.ord);
    if (C.grid) carve_grid(A, C.G, std::max<int64_t>(C.pl.n_total, 1), C.B.S_cap);
    if (C.has_es) carve_edge_sort(A, C.es, std::max<int64_t>(C.B.S_cap, 1));
    F2M_CUDA(ensure_device(ctx, A.used));
    A.base = ctx->dev;
    A.used = 0;
    carve(A, C.B, C.pl, own_inputs, &C.deg, &C.scan, &C.ci, &C.cs, &C.ord);
    if (C.grid) carve_grid(A, C.G, std::max<int64_t>(C.pl.n_total, 1), C.B.S_cap);
    if (C.has_es) carve_edge_sort(A, C.es, std::max<int64_t>(C.B.S_cap, 1));
    C.B.skip_dedup = 0;
    C.B.cost_mode = prm.cost_mode;
    // work lists through pinned staging
    const size_t nc = C.pl.chunk_inst.size();
    const size_t bytes = (2 * nc + n_inst) * sizeof(int32_t);
    F2M_CUDA(ensure_pinned(ctx, bytes));
    int32_t* hp = reinterpret_cast<int32_t*>(ctx->pinned);
    std::memcpy(hp, C.pl.chunk_inst.data(), nc * sizeof(int32_t));
    std::memcpy(hp + nc, C.pl.chunk_start.data(), nc * sizeof(int32_t));
    std::memcpy(hp + 2 * nc, C.pl.order.data(), n_inst * sizeof(int32_t));
    F2M_CUDA(cudaMemcpyAsync(C.ci, hp, nc * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(C.cs, hp + nc, nc * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(C.ord, hp + 2 * nc, n_inst * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    return F2M_OK;
}

// One persistent launch per solver class, each on its own stream forked from
// the context stream (largest class first), joined back before returning.
f2m_status launch_classes(f2m_ctx* ctx, DevCall& C, const f2m_params& prm) {
    const DevParams P = to_dev(prm);
    if (C.grid) {
        F2M_CUDA(launch_grid_order(C.B, C.G, 0, C.pl.max_n, nullptr, C.spatial, ctx->stream, &ctx->launches));
        F2M_CUDA(launch_solve_grid(C.B, P, C.G, 0, C.pl.max_n, false, ctx->stream, &ctx->launches));
        return F2M_OK;
    }
    const int nc = solve_num_classes();
    F2M_CUDA(cudaEventRecord(ctx->fork, ctx->stream));
    for (int c = nc - 1; c >= 0; --c) {
        const int n = C.pl.cnt[c];
        if (n <= 0) continue;
        F2M_CUDA(cudaStreamWaitEvent(ctx->aux[c], ctx->fork, 0));
        F2M_CUDA(launch_solve_class(c, C.B, P, C.ord + C.pl.seg[c], n, C.B.queue + c,
                                    C.pl.class_vcap[c], ctx->aux[c], &ctx->launches));
        F2M_CUDA(cudaEventRecord(ctx->join[c], ctx->aux[c]));
        F2M_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join[c], 0));
    }
    // irregular combs of the first solve: Ax=b and the primal on the device
    F2M_CUDA(launch_axb(C.B, P, ctx->stream, &ctx->launches));
    return F2M_OK;
}

f2m_status run_device(f2m_ctx* ctx, DevCall& C, const f2m_params& prm, bool build_graph, bool solve) {
    Range rg("f2m enqueue device stages");
    F2M_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    F2M_CUDA(launch_prep(C.B, ctx->stream, &ctx->launches));
    F2M_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
    F2M_CUDA(launch_knn(C.B, C.scan, ctx->stream, &ctx->launches));
    F2M_CUDA(cudaEventRecord(ctx->ev[2], ctx->stream));
    if (build_graph) F2M_CUDA(launch_graph(C.B, C.deg, C.scan, ctx->stream, &ctx->launches));
    F2M_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
    if (solve) {
        f2m_status s = launch_classes(ctx, C, prm);
        if (s) return s;
    }
    F2M_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
    ctx->timed = true;
    ctx->last = C.B;
    return F2M_OK;
}

template <class T>
f2m_status d2h(f2m_ctx* ctx, std::vector<T>& v, const T* src, size_t n) {
    v.resize(n);
    if (n) F2M_CUDA(cudaMemcpyAsync(v.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    return F2M_OK;
}
template <class T>
f2m_status h2d(f2m_ctx* ctx, T* dst, const std::vector<T>& v) {
    if (!v.empty()) F2M_CUDA(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return F2M_OK;
}

// Pull instance b (device-built graph, node ids = de-duplicated input order).
// Copies instance b to the host (through pinned staging, one synchronisation
// for the bulk arrays).  `mu` (optional) serialises the stream work.
f2m_status pull_instance(f2m_ctx* ctx, const DevCall& C, int b, HostInst& H, bool with_keys,
                         std::mutex* mu = nullptr) {
    std::unique_lock<std::mutex> lk;
    if (mu) lk = std::unique_lock<std::mutex>(*mu);
    const Batch& B = C.B;
    int32_t V = 0;
    int64_t base = 0;
    F2M_CUDA(cudaMemcpyAsync(&V, B.Vn + b, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(&base, B.offs + b, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    unsigned long long db = 0;
    F2M_CUDA(cudaMemcpyAsync(&db, B.dmin_bits + b, sizeof(db), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    H.V = V;
    std::memcpy(&H.dmin, &db, sizeof(double));
    std::vector<int64_t> row;
    if (d2h(ctx, row, B.row + base, V + 1)) return F2M_ERR_CUDA;
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    const int64_t s0 = row[0], S = row[V] - row[0];
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t bytes = al(S * sizeof(Slot)) + al(S * 8) + 3 * al(S * 4) + al(S * 2) + al(V * 8) + 3 * al(V * 4);
    F2M_CUDA(ensure_pinned(ctx, bytes));
    char* q = ctx->pinned;
    auto take = [&](size_t n) { char* r = q; q += al(n); return r; };
    Slot* sl = reinterpret_cast<Slot*>(take(S * sizeof(Slot)));
    double* cost = reinterpret_cast<double*>(take(S * 8));
    int32_t* em = reinterpret_cast<int32_t*>(take(S * 4));
    int32_t* oth = reinterpret_cast<int32_t*>(take(S * 4));
    int32_t* mirror = reinterpret_cast<int32_t*>(take(S * 4));
    uint16_t* perm = reinterpret_cast<uint16_t*>(take(S * 2));
    double* F = reinterpret_cast<double*>(take(V * 8));
    int32_t* efcnt = reinterpret_cast<int32_t*>(take(V * 4));
    int32_t* ccnt = reinterpret_cast<int32_t*>(take(V * 4));
    int32_t* K = reinterpret_cast<int32_t*>(take(V * 4));
    auto cp = [&](void* dst, const void* src, size_t n) {
        return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, ctx->stream);
    };
    F2M_CUDA(cp(sl, B.slot + s0, S * sizeof(Slot)));
    F2M_CUDA(cp(cost, B.s_cost + s0, S * 8));
    F2M_CUDA(cp(mirror, B.mirror + s0, S * 4));
    F2M_CUDA(cp(perm, B.perm + s0, S * 2));
    const bool dev_order = with_keys && C.has_es;
    if (dev_order) {  // the edge order sorted on the device: one array back
        const uint32_t* ord = nullptr;
        F2M_CUDA(launch_edge_order(B, b, V, S, C.es, &ord, ctx->stream, &ctx->launches));
        F2M_CUDA(cp(em, ord, (S / 2) * 4));
    } else if (with_keys) {
        F2M_CUDA(cp(em, B.s_em + s0, S * 4));
        F2M_CUDA(cp(oth, B.s_oth + s0, S * 4));
    }
    F2M_CUDA(cp(F, B.F + base, V * 8));
    F2M_CUDA(cp(efcnt, B.efcnt + base, V * 4));
    F2M_CUDA(cp(ccnt, B.ccnt + base, V * 4));
    F2M_CUDA(cp(K, B.K + base, V * 4));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    StageClock clk;
    H.row.resize(V + 1);
    for (int v = 0; v <= V; ++v) H.row[v] = row[v] - s0;
    H.nbr.resize(S);
    H.Dn.resize(S);
    parallel_for(S, [&](int64_t a0, int64_t a1) {
        for (int64_t a = a0; a < a1; ++a) { H.nbr[a] = sl[a].nbr; H.Dn[a] = sl[a].D; }
    });
    H.cost.resize(S);
    H.perm.resize(S);
    H.mirror.resize(S);
    parallel_for(S, [&](int64_t a0, int64_t a1) {
        std::memcpy(H.cost.data() + a0, cost + a0, (a1 - a0) * sizeof(double));
        std::memcpy(H.perm.data() + a0, perm + a0, (a1 - a0) * sizeof(uint16_t));
        std::memcpy(H.mirror.data() + a0, mirror + a0, (a1 - a0) * sizeof(int32_t));
    });
    H.F.assign(F, F + V);
    H.efcnt.assign(efcnt, efcnt + V);
    H.ccnt.assign(ccnt, ccnt + V);
    H.label.assign(K, K + V);
    clk.mark("pull.unpack");
    if (dev_order) {
        std::vector<uint32_t> ord(reinterpret_cast<uint32_t*>(em), reinterpret_cast<uint32_t*>(em) + S / 2);
        if (lk.owns_lock()) lk.unlock();  // the staging is no longer needed
        number_edges_ordered(H, ord.data(), S / 2);
        clk.mark("pull.number_edges");
    } else if (with_keys) {
        std::vector<int> ev(em, em + S), ov(oth, oth + S);
        if (lk.owns_lock()) lk.unlock();  // the staging is no longer needed
        // keys hold FXY indices; node ids here are the same indices
        number_edges(H, ev, ov);
        clk.mark("pull.number_edges");
    }
    return F2M_OK;
}

f2m_status complete_instance(f2m_ctx* ctx, DevCall& C, int b, const f2m_params& prm, f2m_result& R,
                             std::mutex* mu = nullptr) {
    Range rg("f2m complete instance");
    HostInst& H = R.H;
    const double vb = prm.error_B * prm.error_B_comb;
    StageClock clk;
    HostCheck HC(H, vb);
    clk.mark("hostcheck.build");
    int IRR_B = HC.check();
    clk.mark("hostcheck.check");
    int steps = 0;
    if (IRR_B > 0) {
        // the repair steps use the call's stream and work lists: one host
        // thread at a time
        std::unique_lock<std::mutex> lk;
        if (mu) lk = std::unique_lock<std::mutex>(*mu);
        int64_t ibase = 0, s0 = 0;
        F2M_CUDA(cudaMemcpyAsync(&ibase, C.B.offs + b, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
        F2M_CUDA(cudaMemcpyAsync(&s0, C.B.row + ibase, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
        double sv = prm.shift0;
        std::vector<double> sh;
        const int32_t one = b;
        // cuda_IRREGULAR_B_recompute + get_combs_cuda + host_combs_check
        auto step = [&](double shiftV, int type) -> int {
            steps++;
            HC.shifts(shiftV, type, sh);
            Batch B = C.B;
            const int32_t st = kNeedsHost;
            cudaError_t e;
            if ((e = cudaMemcpyAsync(const_cast<double*>(B.shift) + ibase, sh.data(), sh.size() * sizeof(double),
                                     cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(C.ord, &one, sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(B.status + b, &st, sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
                (e = (C.grid ? launch_solve_grid(B, to_dev(prm), C.G, b, H.V, true, ctx->stream, &ctx->launches)
                             : launch_refit_class(solve_class_of(H.V), B, to_dev(prm), C.ord, 1, B.queue + 7,
                                                  std::max<int32_t>(H.V, 4), ctx->stream, &ctx->launches))) != cudaSuccess ||
                (e = cudaMemcpyAsync(H.F.data(), B.F + ibase, H.V * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(H.efcnt.data(), B.efcnt + ibase, H.V * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(H.ccnt.data(), B.ccnt + ibase, H.V * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(H.perm.data(), B.perm + s0, H.perm.size() * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess) {
                ctx->err = cudaGetErrorString(e);
                return -1;
            }
            int32_t st2 = 0;
            cudaMemcpyAsync(&st2, B.status + b, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
            if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) { ctx->err = cudaGetErrorString(e); return -1; }
            if (st2 == F2M_ERR_NOT_CONVERGED || st2 == F2M_ERR_CAPACITY) return -2;
            return HC.check();
        };
        for (;;) {  // graph_cuda.cu:74-126
            if ((IRR_B = step(sv, 0)) <= 0) break;
            if ((IRR_B = step(sv, 1)) <= 0) break;
            sv = -sv;
            if ((IRR_B = step(sv, 0)) <= 0) break;
            sv = -sv;
            if ((IRR_B = step(sv, 1)) <= 0) break;
            sv = -sv;
            sv *= 2;
            if (std::fabs(sv) > prm.shift_max) break;
        }
        if (IRR_B == -1) return fail(ctx, F2M_ERR_CUDA, "repair step failed: " + ctx->err);
        if (IRR_B == -2) IRR_B = 1;
    }
    R.st.repair_steps = steps;
    R.st.irr_a = HC.irr_a;
    R.st.irr_b = IRR_B > 0 ? IRR_B : 0;
    R.st.n_combs = (int32_t)HC.comb_V.size();
    clk.mark("repair");
    R.x.assign(H.E, 0.0);
    R.X.clear();
    if (IRR_B == 0) {
        for (int v = 0; v < H.V; ++v)  // node::get_eA_X (node.cpp:61-71)
            for (int e : HC.eA[v]) {
                const int v0 = H.label[v];
                if (v0 < H.label[H.el1[e]]) R.X[e] = 1;
                if (v0 < H.label[H.el2[e]]) R.X[e] = 1;
            }
        for (auto& Cb : HC.Combs)
            for (auto& kv : Cb.XB) R.X[kv.first] = kv.second;
        double OVAL = 0;  // graph::getOVAL (graph_tour.hpp:165-184)
        int mr = 0;
        for (auto& kv : R.X) {
            const int e = kv.first;
            mr = std::max(mr, std::min(H.rank1[e], H.rank2[e]));
            OVAL += kv.second * H.eDo[e];
            R.x[e] = kv.second;
        }
        R.lp = OVAL;
        R.max_rank = mr;
        R.status = F2M_OK;
        // graph::check_solution (graph_tour.hpp:142-163)
        std::vector<float> deg(H.V, 0.0f);
        std::vector<char> has(H.V, 0);
        for (auto& kv : R.X) {
            deg[H.el1[kv.first]] += (float)kv.second; has[H.el1[kv.first]] = 1;
            deg[H.el2[kv.first]] += (float)kv.second; has[H.el2[kv.first]] = 1;
        }
        int viol = 0;
        for (int v = 0; v < H.V; ++v)
            if (has[v] && !(deg[v] > 2.0f - 1e-2f && deg[v] < 2.0f + 1e-2f)) viol++;
        R.st.degree_violations = viol;
    } else {
        R.status = F2M_ERR_NOT_CONVERGED;
        R.err = "Optimal Solution not Found";
        R.lp = NAN;
    }
    clk.mark("primal");
    // FP64 dual bound with u = -F/2 in d_min units
    double fsum = 0, neg = 0;
    for (int v = 0; v < H.V; ++v) fsum += H.F[v];
    for (int e = 0; e < H.E; ++e) {
        const double d = (H.eD[e] + 0.5 * H.F[H.ev1[e]]) + 0.5 * H.F[H.ev2[e]];
        neg += std::min(0.0, d);
    }
    R.st.dual_value = H.dmin * (-fsum + neg);
    R.st.d_min = H.dmin;
    clk.mark("dual");
    return F2M_OK;
}

// The result of an instance the device completed (every comb regular, or
// the irregular ones solved by Ax=b, status F2M_OK): the edge arrays in the
// reference's edge order (graph_tour.hpp:28-98) are written on the device
// (launch_edge_order, then k_export_edges) and come back in one copy, with
// the node labels and potentials; OVAL, MAX edge rank, the degree check and
// the FP64 dual bound are the device's (graph_tour.hpp:142-184; OVAL summed
// in the solver's order, which agrees with the host stage's hash order to
// rounding).  The host builds none of the comb stage's structures.  Used by
// the points path; the file path keeps the host stage, which also writes the
// reference's files.
f2m_status export_from_device(f2m_ctx* ctx, const DevCall& C, int b, f2m_result& R) {
    Range rg("f2m export instance (device)");
    const Batch& B = C.B;
    HostInst& H = R.H;
    int32_t V = 0, nc = 0, ni = 0, mr = 0, viol = 0;
    int64_t base = 0;
    unsigned long long db = 0;
    double lp = 0, dual = 0;
    auto small = [&](void* dst, const void* src, size_t n) {
        return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, ctx->stream);
    };
    F2M_CUDA(small(&V, B.Vn + b, 4));
    F2M_CUDA(small(&base, B.offs + b, 8));
    F2M_CUDA(small(&db, B.dmin_bits + b, 8));
    F2M_CUDA(small(&nc, B.n_combs + b, 4));
    F2M_CUDA(small(&ni, B.n_irr + b, 4));
    F2M_CUDA(small(&mr, B.max_rank + b, 4));
    F2M_CUDA(small(&viol, B.deg_viol + b, 4));
    F2M_CUDA(small(&lp, B.lp + b, 8));
    F2M_CUDA(small(&dual, B.dual + b, 8));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    int64_t r0 = 0, r1 = 0;
    F2M_CUDA(small(&r0, B.row + base, 8));
    F2M_CUDA(small(&r1, B.row + base + V, 8));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    const int64_t S = r1 - r0, E = S / 2;
    const uint32_t* ord = nullptr;
    F2M_CUDA(launch_edge_order(B, b, V, S, C.es, &ord, ctx->stream, &ctx->launches));
    const EdgeExport X = edge_export_view(C.es.xout, E);
    F2M_CUDA(launch_export_edges(B, b, V, ord, E, X, ctx->stream, &ctx->launches));
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    F2M_CUDA(ensure_pinned(ctx, al(E * 40) + al(V * 12)));
    char* q = ctx->pinned;
    F2M_CUDA(small(q, C.es.xout, E * 40));  // Do, D, x, ev1, ev2, el1, el2 back to back
    double* F = reinterpret_cast<double*>(q + al(E * 40));
    int32_t* K = reinterpret_cast<int32_t*>(q + al(E * 40) + V * 8);
    F2M_CUDA(small(F, B.F + base, V * 8));
    F2M_CUDA(small(K, B.K + base, V * 4));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    const EdgeExport P = edge_export_view(q, E);
    H.V = V;
    H.E = (int)E;
    std::memcpy(&H.dmin, &db, sizeof(double));
    H.label.assign(K, K + V);
    H.F.assign(F, F + V);
    H.ev1.resize(E); H.ev2.resize(E); H.el1.resize(E); H.el2.resize(E);
    H.eDo.resize(E); H.eD.resize(E); R.x.resize(E);
    parallel_for(E, [&](int64_t e0, int64_t e1) {
        const size_t n4 = (e1 - e0) * 4, n8 = (e1 - e0) * 8;
        std::memcpy(H.ev1.data() + e0, P.ev1 + e0, n4);
        std::memcpy(H.ev2.data() + e0, P.ev2 + e0, n4);
        std::memcpy(H.el1.data() + e0, P.el1 + e0, n4);
        std::memcpy(H.el2.data() + e0, P.el2 + e0, n4);
        std::memcpy(H.eDo.data() + e0, P.Do + e0, n8);
        std::memcpy(H.eD.data() + e0, P.D + e0, n8);
        std::memcpy(R.x.data() + e0, P.x + e0, n8);
    });
    R.X.clear();
    R.lp = lp;
    R.max_rank = mr;
    R.status = F2M_OK;
    R.st.repair_steps = 0;
    R.st.irr_a = ni;  // irregular combs, solved by Ax=b on the device
    R.st.irr_b = 0;
    R.st.n_combs = nc;
    R.st.degree_violations = viol;
    R.st.dual_value = dual;
    R.st.d_min = H.dmin;
    return F2M_OK;
}

f2m_status pull_stats(f2m_ctx* ctx, const DevCall& C, int b, f2m_result& R) {
    int64_t it = 0;
    int32_t ch = 0;
    double mg = 0;
    F2M_CUDA(cudaMemcpyAsync(&it, C.B.iters + b, sizeof(it), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(&ch, C.B.checks + b, sizeof(ch), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(&mg, C.B.max_grad + b, sizeof(mg), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    R.st.iterations = it;
    R.st.checks = ch;
    R.st.max_grad = mg;
    return F2M_OK;
}

}  // namespace

/* ------------------------------------------------------------------ */
/* C ABI                                                                */
/* ------------------------------------------------------------------ */
extern "C" {

void f2m_default_params(f2m_params* p) {
    p->error_B = 1e-7;
    p->error_B_comb = 1e2;
    p->glob_K = 5;
    p->glob_rounds = 200;
    p->glob_inner = 50;
    p->glob_tol = 0.01;
    p->factor0 = 100;
    p->factor_step = 300;
    p->factor_cap = 5000;
    p->max_rounds = 10000;
    p->fix_rounds = 100;
    p->fix_factor = 500;
    p->check_every = 50;
    p->frozen_iters = 20;
    p->ef_thr = 1.0;
    p->ef_small_deg = 10;
    p->ef_min = 3;
    p->comb_thr = 0.25;
    p->shift0 = 0.5;
    p->shift_max = 32;
    p->max_iters = 20000000;
    p->cost_mode = F2M_COST_REF_EUCLID;
    p->solver = 0;
    p->grid_spin_limit = (int64_t)1 << 26;
}

f2m_status f2m_create(f2m_ctx** out, int device) {
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return F2M_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return F2M_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return F2M_ERR_NO_DEVICE;
    f2m_ctx* c = new f2m_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return F2M_ERR_CUDA;
    }
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            delete c;
            return F2M_ERR_CUDA;
        }
    for (int k = 0; k < 4; ++k)
        if (cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->join[k], cudaEventDisableTiming) != cudaSuccess) {
            delete c;
            return F2M_ERR_CUDA;
        }
    if (cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) != cudaSuccess) {
        delete c;
        return F2M_ERR_CUDA;
    }
    *out = c;
    return F2M_OK;
}

void f2m_destroy(f2m_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->dev) cudaFree(c->dev);
    if (c->pinned) cudaFreeHost(c->pinned);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) {
        if (c->aux[k]) cudaStreamDestroy(c->aux[k]);
        if (c->join[k]) cudaEventDestroy(c->join[k]);
    }
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->sgraph) cudaGraphExecDestroy(c->sgraph);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

f2m_status f2m_phase_times(f2m_ctx* ctx, float* ms, f2m_work* work) {
    if (!ctx || !ctx->timed) return F2M_ERR_INPUT;
    F2M_CUDA(cudaEventSynchronize(ctx->ev[4]));
    for (int k = 0; k < 4; ++k) F2M_CUDA(cudaEventElapsedTime(ms + k, ctx->ev[k], ctx->ev[k + 1]));
    if (work) {
        const Batch& B = ctx->last;
        const int n = B.n_inst;
        std::vector<int64_t> wn(n), ws(n), wp(n), it(n);
        std::vector<int32_t> vn(n), st(n);
        int64_t slots = 0;
        F2M_CUDA(cudaMemcpy(wn.data(), B.work_nodes, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(ws.data(), B.work_slots, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(wp.data(), B.work_pad, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(it.data(), B.iters, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(vn.data(), B.Vn, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(st.data(), B.status, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(&slots, B.row + B.n_total, sizeof(int64_t), cudaMemcpyDeviceToHost));
        *work = f2m_work{0, 0, slots, 0, 0, 0};
        for (int b = 0; b < n; ++b) {
            if (st[b] == F2M_ERR_INPUT || st[b] == F2M_ERR_CAPACITY) continue;  // never solved
            work->node_iters += wn[b];
            work->slot_iters += ws[b];
            work->pad_iters += wp[b];
            work->lane_iters += it[b] * 32 * (int64_t)((vn[b] + 31) / 32);
            work->points += vn[b];
        }
    }
    return F2M_OK;
}

const char* f2m_last_error(const f2m_ctx* c) { return c ? c->err.c_str() : "no context"; }
int64_t f2m_kernel_launches(const f2m_ctx* c) { return c ? c->launches : 0; }

f2m_status f2m_sync(f2m_ctx* ctx) {
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    return F2M_OK;
}

f2m_status f2m_fp64_rate(f2m_ctx* ctx, int32_t kind, int32_t repeats, double* lane_ops_per_s) {
    if (!ctx || !lane_ops_per_s || kind < 0 || kind > 2 || repeats < 1)
        return fail(ctx, F2M_ERR_INPUT, "f2m_fp64_rate: kind 0, 1 or 2, repeats >= 1");
    F2M_CUDA(cudaSetDevice(ctx->device));
    int per_sm = 0;
    F2M_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, ctx->device));
    const int blocks = ctx->sms * (per_sm / 256);  // full occupancy of 256-thread CTAs
    constexpr int kIters = 40000;
    F2M_CUDA(ensure_device(ctx, 4096));
    double* out = reinterpret_cast<double*>(ctx->dev);
    double best = 0.0;
    for (int r = 0; r <= repeats; ++r) {  // the first launch warms up
        F2M_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
        if (kind == 2) F2M_CUDA(launch_logit_probe(blocks, kIters / 16, out, ctx->stream));
        else F2M_CUDA(launch_fp64_probe(kind, blocks, kIters, out, ctx->stream));
        F2M_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
        F2M_CUDA(cudaEventSynchronize(ctx->ev[1]));
        ctx->launches++;
        float ms = 0.f;
        F2M_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        const double ops = kind == 2 ? logit_probe_terms(blocks, kIters / 16) : fp64_probe_ops(kind, blocks, kIters);
        if (r > 0 && ms > 0.f) best = std::max(best, ops / (ms * 1e-3));
    }
    ctx->timed = false;  // the phase events now hold the probe's times
    *lane_ops_per_s = best;
    return F2M_OK;
}

f2m_status f2m_smooth_work(const f2m_ctx* ctx, int64_t* terms, float* kernel_ms) {
    if (!ctx) return F2M_ERR_INPUT;
    if (terms) *terms = ctx->smooth_terms;
    if (kernel_ms) *kernel_ms = ctx->smooth_ms;
    return F2M_OK;
}

f2m_status f2m_partition_selfcheck(f2m_ctx* ctx, int32_t n_cases, uint64_t seed, int64_t* mismatches) {
    if (!ctx || !mismatches || n_cases < 0)
        return fail(ctx, F2M_ERR_INPUT, "f2m_partition_selfcheck: n_cases >= 0 and an output pointer");
    F2M_CUDA(cudaSetDevice(ctx->device));
    F2M_CUDA(ensure_device(ctx, 4096));
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(ctx->dev);
    F2M_CUDA(cudaMemsetAsync(bad, 0, sizeof(*bad), ctx->stream));
    F2M_CUDA(launch_partition_check(n_cases, seed, bad, ctx->stream));
    ctx->launches++;
    unsigned long long h = 0;
    F2M_CUDA(cudaMemcpyAsync(&h, bad, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    *mismatches = (int64_t)h;
    return F2M_OK;
}

static f2m_status check_args(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs, int32_t top_k,
                             const f2m_params* params) {
    if (!ctx) return F2M_ERR_INPUT;
    if (n_inst < 1 || !offs) return fail(ctx, F2M_ERR_INPUT, "need at least one instance");
    if (top_k < 3) return fail(ctx, F2M_ERR_INPUT, "N must be at least 3");
    if (top_k > 256) return fail(ctx, F2M_ERR_CAPACITY, "N above 256 is not supported");
    if (params && params->cost_mode != F2M_COST_REF_EUCLID && params->cost_mode != F2M_COST_NINT)
        return fail(ctx, F2M_ERR_INPUT, "unknown cost mode");
    for (int32_t b = 0; b < n_inst; ++b)
        if (offs[b + 1] < offs[b]) return fail(ctx, F2M_ERR_INPUT, "offsets must be non-decreasing");
    if (offs[0] != 0) return fail(ctx, F2M_ERR_INPUT, "offs[0] must be 0");
    if (offs[n_inst] > INT32_MAX) return fail(ctx, F2M_ERR_CAPACITY, "too many points in one call");
    return F2M_OK;
}

// Host completion of the batch instances whose combs need the Ax=b stage.
// Instances whose combs need the host stage (comb_thread.cpp, Ax_b.cpp) are
// completed by a pool of host threads.  Their device state is first copied
// in one go into pinned staging (one synchronisation for all of them); the
// threads then rebuild the host instances and run the comb checks side by
// side, and any repair refits share the call's stream under a mutex.
static f2m_status complete_batch(f2m_ctx* ctx, DevCall& C, const f2m_params& prm,
                                 std::vector<int32_t>& status, std::vector<double>& lp,
                                 std::vector<int32_t>* max_rank) {
    std::vector<int> todo;
    for (int b = 0; b < C.pl.n_inst; ++b)
        if (status[b] == kNeedsHost) todo.push_back(b);
    if (todo.empty()) return F2M_OK;
    Range rg("f2m host comb stage");
    const Batch& B = C.B;
    const int ni = C.pl.n_inst;
    std::vector<int32_t> Vn(ni);
    std::vector<int64_t> offs(ni + 1);
    std::vector<unsigned long long> db(ni);
    F2M_CUDA(cudaMemcpyAsync(Vn.data(), B.Vn, ni * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(offs.data(), B.offs, (ni + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(db.data(), B.dmin_bits, ni * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    const size_t nt = todo.size();
    std::vector<std::vector<int64_t>> rows(nt);
    for (size_t k = 0; k < nt; ++k) {
        const int b = todo[k];
        rows[k].resize(Vn[b] + 1);
        F2M_CUDA(cudaMemcpyAsync(rows[k].data(), B.row + offs[b], (Vn[b] + 1) * sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    }
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    // staging layout per instance: slots, cost, em, oth, mirror, perm | F, efcnt, ccnt, K
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    std::vector<size_t> off(nt + 1, 0);
    for (size_t k = 0; k < nt; ++k) {
        const int64_t V = Vn[todo[k]], S = rows[k][V] - rows[k][0];
        off[k + 1] = off[k] + al(S * sizeof(Slot)) + al(S * 8) + 3 * al(S * 4) + al(S * 2) + al(V * 8) +
                     3 * al(V * 4);
    }
    F2M_CUDA(ensure_pinned(ctx, off[nt]));
    char* stage = ctx->pinned;
    struct View {
        Slot* slot; double* cost; int32_t* em; int32_t* oth; int32_t* mirror; uint16_t* perm;
        double* F; int32_t* efcnt; int32_t* ccnt; int32_t* K;
    };
    std::vector<View> views(nt);
    for (size_t k = 0; k < nt; ++k) {
        const int b = todo[k];
        const int64_t V = Vn[b], s0 = rows[k][0], S = rows[k][V] - s0, base = offs[b];
        char* q = stage + off[k];
        View& w = views[k];
        auto take = [&](size_t bytes) { char* r = q; q += al(bytes); return r; };
        w.slot = reinterpret_cast<Slot*>(take(S * sizeof(Slot)));
        w.cost = reinterpret_cast<double*>(take(S * 8));
        w.em = reinterpret_cast<int32_t*>(take(S * 4));
        w.oth = reinterpret_cast<int32_t*>(take(S * 4));
        w.mirror = reinterpret_cast<int32_t*>(take(S * 4));
        w.perm = reinterpret_cast<uint16_t*>(take(S * 2));
        w.F = reinterpret_cast<double*>(take(V * 8));
        w.efcnt = reinterpret_cast<int32_t*>(take(V * 4));
        w.ccnt = reinterpret_cast<int32_t*>(take(V * 4));
        w.K = reinterpret_cast<int32_t*>(take(V * 4));
        auto cp = [&](void* dst, const void* src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        };
        F2M_CUDA(cp(w.slot, B.slot + s0, S * sizeof(Slot)));
        F2M_CUDA(cp(w.cost, B.s_cost + s0, S * 8));
        F2M_CUDA(cp(w.em, B.s_em + s0, S * 4));
        F2M_CUDA(cp(w.oth, B.s_oth + s0, S * 4));
        F2M_CUDA(cp(w.mirror, B.mirror + s0, S * 4));
        F2M_CUDA(cp(w.perm, B.perm + s0, S * 2));
        F2M_CUDA(cp(w.F, B.F + base, V * 8));
        F2M_CUDA(cp(w.efcnt, B.efcnt + base, V * 4));
        F2M_CUDA(cp(w.ccnt, B.ccnt + base, V * 4));
        F2M_CUDA(cp(w.K, B.K + base, V * 4));
    }
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    std::mutex mu;
    std::atomic<size_t> next{0};
    std::vector<f2m_status> err(nt, F2M_OK);
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < nt;) {
            const int b = todo[k];
            const View& w = views[k];
            f2m_result R;
            HostInst& H = R.H;
            const int V = Vn[b];
            const int64_t s0 = rows[k][0], S = rows[k][V] - s0;
            H.V = V;
            std::memcpy(&H.dmin, &db[b], sizeof(double));
            H.row.resize(V + 1);
            for (int v = 0; v <= V; ++v) H.row[v] = rows[k][v] - s0;
            H.nbr.resize(S);
            H.Dn.resize(S);
            for (int64_t a = 0; a < S; ++a) { H.nbr[a] = w.slot[a].nbr; H.Dn[a] = w.slot[a].D; }
            H.cost.assign(w.cost, w.cost + S);
            H.perm.assign(w.perm, w.perm + S);
            H.mirror.assign(w.mirror, w.mirror + S);
            H.F.assign(w.F, w.F + V);
            H.efcnt.assign(w.efcnt, w.efcnt + V);
            H.ccnt.assign(w.ccnt, w.ccnt + V);
            H.label.assign(w.K, w.K + V);
            number_edges(H, std::vector<int>(w.em, w.em + S), std::vector<int>(w.oth, w.oth + S));
            const f2m_status s = complete_instance(ctx, C, b, prm, R, &mu);
            err[k] = s;
            if (s) continue;
            status[b] = R.status;
            lp[b] = R.lp;
            if (max_rank) (*max_rank)[b] = R.max_rank;
        }
    };
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nthr = std::min(nt, std::min<size_t>(hw, 32));
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nthr; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (f2m_status s : err)
        if (s) return s;
    return F2M_OK;
}

f2m_status f2m_solve_batch(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs, const double* x,
                           const double* y, int32_t top_k, const f2m_params* params,
                           f2m_batch_out* out) {
    f2m_status s = check_args(ctx, n_inst, offs, top_k, params);
    if (s) return s;
    if (!out || !out->lp || !out->status) return fail(ctx, F2M_ERR_INPUT, "lp and status outputs are required");
    f2m_params prm;
    f2m_default_params(&prm);
    if (params) prm = *params;
    cudaSetDevice(ctx->device);
    DevCall C;
    if ((s = setup_call(ctx, C, n_inst, offs, top_k, prm, true))) return s;
    const int64_t n = C.pl.n_total;
    F2M_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(C.B.offs), offs, (n_inst + 1) * sizeof(int64_t),
                             cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.X_in), x, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.Y_in), y, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if ((s = run_device(ctx, C, prm, true, true))) return s;
    std::vector<int32_t> status(n_inst), mr;
    std::vector<double> lp(n_inst);
    F2M_CUDA(cudaMemcpyAsync(status.data(), C.B.status, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(lp.data(), C.B.lp, n_inst * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (out->max_rank) {
        mr.resize(n_inst);
        F2M_CUDA(cudaMemcpyAsync(mr.data(), C.B.max_rank, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (out->n_nodes) F2M_CUDA(cudaMemcpyAsync(out->n_nodes, C.B.Vn, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (out->n_edges) F2M_CUDA(cudaMemcpyAsync(out->n_edges, C.B.n_edges, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (out->n_combs) F2M_CUDA(cudaMemcpyAsync(out->n_combs, C.B.n_combs, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (out->iterations) F2M_CUDA(cudaMemcpyAsync(out->iterations, C.B.iters, n_inst * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (out->n_irregular) F2M_CUDA(cudaMemcpyAsync(out->n_irregular, C.B.n_irr, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if ((s = complete_batch(ctx, C, prm, status, lp, out->max_rank ? &mr : nullptr))) return s;
    std::memcpy(out->status, status.data(), n_inst * sizeof(int32_t));
    std::memcpy(out->lp, lp.data(), n_inst * sizeof(double));
    if (out->max_rank) std::memcpy(out->max_rank, mr.data(), n_inst * sizeof(int32_t));
    return F2M_OK;
}

f2m_status f2m_solve_batch_device(f2m_ctx* ctx, int32_t n_inst, const int64_t* h_offs,
                                  const int64_t* d_offs, const double* d_x, const double* d_y,
                                  int32_t top_k, const f2m_params* params, f2m_batch_out* d_out) {
    f2m_status s = check_args(ctx, n_inst, h_offs, top_k, params);
    if (s) return s;
    if (!d_out || !d_out->lp || !d_out->status) return fail(ctx, F2M_ERR_INPUT, "lp and status outputs are required");
    f2m_params prm;
    f2m_default_params(&prm);
    if (params) prm = *params;
    cudaSetDevice(ctx->device);
    DevCall C;
    if ((s = setup_call(ctx, C, n_inst, h_offs, top_k, prm, false))) return s;
    C.B.offs = d_offs;
    C.B.X_in = d_x;
    C.B.Y_in = d_y;
    if ((s = run_device(ctx, C, prm, true, true))) return s;
    // instances whose combs need the host Ax=b stage are completed here
    std::vector<int32_t> status(n_inst);
    F2M_CUDA(cudaMemcpyAsync(status.data(), C.B.status, n_inst * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    bool any = false;
    for (int32_t v : status) any |= (v == kNeedsHost);
    if (any) {
        std::vector<double> lp;
        if ((s = d2h(ctx, lp, C.B.lp, n_inst))) return s;
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
        if ((s = complete_batch(ctx, C, prm, status, lp, nullptr))) return s;
        F2M_CUDA(cudaMemcpyAsync(C.B.lp, lp.data(), n_inst * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        F2M_CUDA(cudaMemcpyAsync(C.B.status, status.data(), n_inst * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    auto cp = [&](void* dst, const void* src, size_t bytes) {
        return dst ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream) : cudaSuccess;
    };
    F2M_CUDA(cp(d_out->lp, C.B.lp, n_inst * sizeof(double)));
    F2M_CUDA(cp(d_out->status, C.B.status, n_inst * sizeof(int32_t)));
    F2M_CUDA(cp(d_out->n_nodes, C.B.Vn, n_inst * sizeof(int32_t)));
    F2M_CUDA(cp(d_out->n_edges, C.B.n_edges, n_inst * sizeof(int32_t)));
    F2M_CUDA(cp(d_out->n_combs, C.B.n_combs, n_inst * sizeof(int32_t)));
    F2M_CUDA(cp(d_out->max_rank, C.B.max_rank, n_inst * sizeof(int32_t)));
    F2M_CUDA(cp(d_out->iterations, C.B.iters, n_inst * sizeof(int64_t)));
    F2M_CUDA(cp(d_out->n_irregular, C.B.n_irr, n_inst * sizeof(int32_t)));
    return F2M_OK;
}

}  // extern "C"

namespace {

// The single-instance path: rounding/de-duplication, kNN graph and, when
// `solve`, the dual descent, comb stage and primal.
f2m_status points_call(f2m_ctx* ctx, const double* x, const double* y, const int32_t* labels, int32_t n,
                       int32_t top_k, const f2m_params* params, bool solve, f2m_result** out,
                       const double* F0 = nullptr, int32_t nF0 = 0) {
    *out = nullptr;
    const int64_t offs[2] = {0, n};
    f2m_status s = check_args(ctx, 1, offs, top_k, params);
    if (s) return s;
    f2m_params prm;
    f2m_default_params(&prm);
    if (params) prm = *params;
    cudaSetDevice(ctx->device);
    std::unique_ptr<f2m_result> R(new f2m_result());
    // Large inputs are rounded and de-duplicated on the host, as get_KXY does
    // (FXY.hpp:252-267); the device's per-instance pass is quadratic.
    std::vector<double> hx, hy;
    std::vector<int32_t> hl;
    bool host_dedup = n > kHostDedupPoints;
    StageClock clk;
    if (host_dedup) {
        host_dedup_points(x, y, labels, n, hx, hy, hl);
        x = hx.data();
        y = hy.data();
        labels = hl.data();
        n = (int32_t)hx.size();
    }
    clk.mark("dedup");
    const int64_t offs2[2] = {0, n};
    DevCall C;
    if ((s = setup_call(ctx, C, 1, offs2, top_k, prm, true))) return s;
    C.B.skip_dedup = host_dedup ? 1 : 0;
    int32_t* dK = nullptr;
    if (labels) {
        // labels ride in the (unused) cursor buffer until k_prep compacts them
        dK = C.B.cursor;
        C.B.K_in = dK;
        F2M_CUDA(cudaMemcpyAsync(dK, labels, n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    }
    F2M_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(C.B.offs), offs2, 2 * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.X_in), x, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.Y_in), y, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    auto t0 = std::chrono::steady_clock::now();
    F2M_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    F2M_CUDA(launch_prep(C.B, ctx->stream, &ctx->launches));
    F2M_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
    F2M_CUDA(launch_knn(C.B, C.scan, ctx->stream, &ctx->launches));
    F2M_CUDA(cudaEventRecord(ctx->ev[2], ctx->stream));
    C.B.K_in = nullptr;
    F2M_CUDA(launch_graph(C.B, C.deg, C.scan, ctx->stream, &ctx->launches));
    F2M_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
    if (F0) {  // warm start: the potentials of the same nodes (node order of a result)
        int32_t V = 0;
        F2M_CUDA(cudaMemcpyAsync(&V, C.B.Vn, sizeof(V), cudaMemcpyDeviceToHost, ctx->stream));
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
        if (V != nF0)
            return fail(ctx, F2M_ERR_INPUT, "the starting potentials have " + std::to_string(nF0) +
                                                " values for " + std::to_string(V) + " nodes");
        // the per-point "shift" buffer is free until a repair step: use it for F0
        F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.shift), F0, V * sizeof(double),
                                 cudaMemcpyHostToDevice, ctx->stream));
        C.B.F0 = C.B.shift;
    }
    if (!solve) {  // the graph only: edges in the reference's edge order
        F2M_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
        if ((s = pull_instance(ctx, C, 0, R->H, true))) return s;
        std::fill(R->H.F.begin(), R->H.F.end(), 0.0);
        R->status = F2M_OK;
        R->lp = NAN;
        R->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        *out = R.release();
        return F2M_OK;
    }
    clk.mark("setup");
    if ((s = launch_classes(ctx, C, prm))) return s;
    F2M_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
    ctx->timed = true;
    ctx->last = C.B;
    int32_t st = 0;
    F2M_CUDA(cudaMemcpyAsync(&st, C.B.status, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    clk.mark("device");
    if (st != F2M_OK && st != kNeedsHost) {
        R->status = st;
        R->err = st == F2M_ERR_INPUT ? "invalid instance (fewer than 4 distinct points or degenerate box)"
                 : st == F2M_ERR_CUDA ? "a grid barrier wait of the whole-GPU solver ran out "
                                        "(grid_spin_limit polls); the solve was abandoned"
                                      : "instance exceeds a solver limit or did not converge";
        ctx->err = R->err;
        *out = R.release();
        return (f2m_status)st;
    }
    // every comb regular, or the irregular ones solved by Ax=b on the device:
    // the device's primal stands and its arrays come back in edge order;
    // otherwise (an Ax=b system that did not converge, so the repair loop
    // runs) the host comb stage as the reference runs it
    if (st == F2M_OK) {
        if ((s = export_from_device(ctx, C, 0, *R))) return s;
        clk.mark("export");
    } else {
        if ((s = pull_instance(ctx, C, 0, R->H, true))) return s;
        clk.mark("pull");
        if ((s = complete_instance(ctx, C, 0, prm, *R))) return s;
    }
    clk.mark("complete");
    if ((s = pull_stats(ctx, C, 0, *R))) return s;
    R->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = R.release();
    return (f2m_status)(*out)->status;
}

}  // namespace

extern "C" {

f2m_status f2m_solve_points(f2m_ctx* ctx, const double* x, const double* y, const int32_t* labels,
                            int32_t n, int32_t top_k, const f2m_params* params, f2m_result** out) {
    return points_call(ctx, x, y, labels, n, top_k, params, true, out);
}

f2m_status f2m_solve_points_from(f2m_ctx* ctx, const double* x, const double* y, const int32_t* labels,
                                 int32_t n, int32_t top_k, const double* F0, int32_t n_F0,
                                 const f2m_params* params, f2m_result** out) {
    if (!F0) return ctx ? fail(ctx, F2M_ERR_INPUT, "F0 is required") : F2M_ERR_INPUT;
    return points_call(ctx, x, y, labels, n, top_k, params, true, out, F0, n_F0);
}

f2m_status f2m_knn(f2m_ctx* ctx, const double* x, const double* y, const int32_t* labels, int32_t n,
                   int32_t top_k, f2m_result** out) {
    return points_call(ctx, x, y, labels, n, top_k, nullptr, false, out);
}

// graph_c(graph*) + graph::RUN() (F2M.h:175,320) on a graph the caller built:
// edges in edge-id order, per-node lists in that order (graph_cuda_init.hpp:
// 42-63), D as given, d_min = the smallest Do (graph_tour.hpp:70).
f2m_status f2m_solve_graph(f2m_ctx* ctx, int32_t n_nodes, int32_t n_edges, const int32_t* v1,
                           const int32_t* v2, const double* D, const double* Do, const int32_t* labels,
                           const f2m_params* params, f2m_result** out) {
    *out = nullptr;
    if (!ctx) return F2M_ERR_INPUT;
    if (n_nodes < 4 || n_edges < 1 || !v1 || !v2 || !D || !Do)
        return fail(ctx, F2M_ERR_INPUT, "need at least 4 nodes and 1 edge");
    f2m_params prm;
    f2m_default_params(&prm);
    if (params) prm = *params;
    std::vector<int64_t> row(n_nodes + 1, 0);
    double dmin = INFINITY;
    for (int32_t e = 0; e < n_edges; ++e) {
        const int a = v1[e], b = v2[e];
        if (a < 0 || b < 0 || a >= n_nodes || b >= n_nodes || a == b || !(Do[e] > 0) || !(D[e] > 0))
            return fail(ctx, F2M_ERR_INPUT, "edge " + std::to_string(e) + " is invalid");
        row[a + 1]++;
        row[b + 1]++;
        dmin = std::min(dmin, Do[e]);
    }
    int64_t maxdeg = 0;
    for (int32_t v = 0; v < n_nodes; ++v) {
        maxdeg = std::max(maxdeg, row[v + 1]);
        row[v + 1] += row[v];
    }
    if (maxdeg > 65535) return fail(ctx, F2M_ERR_CAPACITY, "a node has more than 65535 edges");
    const int64_t S = row[n_nodes];
    cudaSetDevice(ctx->device);
    std::unique_ptr<f2m_result> R(new f2m_result());
    HostInst& H = R->H;
    H.V = n_nodes;
    H.E = n_edges;
    H.dmin = dmin;
    H.row = row;
    H.nbr.resize(S);
    H.Dn.resize(S);
    H.cost.resize(S);
    H.mirror.resize(S);
    H.slot_edge.resize(S);
    H.ev1.resize(n_edges); H.ev2.resize(n_edges); H.el1.resize(n_edges); H.el2.resize(n_edges);
    H.rank1.resize(n_edges); H.rank2.resize(n_edges);
    H.eD.assign(D, D + n_edges);
    H.eDo.assign(Do, Do + n_edges);
    H.label.resize(n_nodes);
    for (int32_t v = 0; v < n_nodes; ++v) H.label[v] = labels ? labels[v] : v + 1;
    std::vector<int64_t> fill(row.begin(), row.end() - 1);
    std::vector<Slot> slots(S);
    for (int32_t e = 0; e < n_edges; ++e) {
        const int a = std::min(v1[e], v2[e]), b = std::max(v1[e], v2[e]);
        const int64_t sa = fill[a]++, sb = fill[b]++;
        const int ra = (int)(sa - row[a]), rb = (int)(sb - row[b]);
        H.nbr[sa] = b; H.nbr[sb] = a;
        H.Dn[sa] = H.Dn[sb] = D[e];
        H.cost[sa] = H.cost[sb] = Do[e];
        H.mirror[sa] = rb; H.mirror[sb] = ra;
        H.slot_edge[sa] = H.slot_edge[sb] = e;
        H.ev1[e] = a; H.ev2[e] = b;
        if (H.label[a] < H.label[b]) { H.el1[e] = a; H.el2[e] = b; H.rank1[e] = ra; H.rank2[e] = rb; }
        else { H.el1[e] = b; H.el2[e] = a; H.rank1[e] = rb; H.rank2[e] = ra; }
        slots[sa] = Slot{D[e], b, ra};
        slots[sb] = Slot{D[e], a, rb};
    }
    std::vector<uint16_t> perm(S);
    for (int32_t v = 0; v < n_nodes; ++v)
        for (int64_t q = row[v]; q < row[v + 1]; ++q) perm[q] = (uint16_t)(q - row[v]);
    // device buffers of one instance; the list capacity follows the degrees
    const int64_t offs[2] = {0, n_nodes};
    const int32_t cap_n = (int32_t)std::min<int64_t>(256, std::max<int64_t>(3, (S + n_nodes - 1) / n_nodes + 1));
    DevCall C;
    f2m_status st = setup_call(ctx, C, 1, offs, cap_n, prm, true);
    if (st) return st;
    if (C.B.S_cap < S) return fail(ctx, F2M_ERR_CAPACITY, "graph too dense for the solver's list arrays");
    C.spatial = false;  // no coordinates: the grid solver keeps the caller's node order
    Batch& B = C.B;
    std::vector<int32_t> mirror32(H.mirror.begin(), H.mirror.end());
    const int32_t one_v = n_nodes, ok = F2M_OK;
    unsigned long long db;
    std::memcpy(&db, &dmin, sizeof(db));
    std::vector<double> zeros(n_nodes, 0.0);
    auto h2 = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
    };
    F2M_CUDA(h2(const_cast<int64_t*>(B.offs), offs, sizeof(offs)));
    F2M_CUDA(h2(B.Vn, &one_v, sizeof(one_v)));
    F2M_CUDA(h2(B.status, &ok, sizeof(ok)));
    F2M_CUDA(h2(B.dmin_bits, &db, sizeof(db)));
    F2M_CUDA(h2(B.row, row.data(), row.size() * sizeof(int64_t)));
    F2M_CUDA(h2(B.slot, slots.data(), S * sizeof(Slot)));
    F2M_CUDA(h2(B.perm, perm.data(), S * sizeof(uint16_t)));
    F2M_CUDA(h2(B.mirror, mirror32.data(), S * sizeof(int32_t)));
    F2M_CUDA(h2(B.s_cost, H.cost.data(), S * sizeof(double)));
    F2M_CUDA(h2(B.K, H.label.data(), n_nodes * sizeof(int32_t)));
    F2M_CUDA(h2(const_cast<double*>(B.shift), zeros.data(), n_nodes * sizeof(double)));
    auto t0 = std::chrono::steady_clock::now();
    F2M_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    F2M_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
    F2M_CUDA(cudaEventRecord(ctx->ev[2], ctx->stream));
    F2M_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
    f2m_status s = launch_classes(ctx, C, prm);
    if (s) return s;
    F2M_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
    ctx->timed = true;
    ctx->last = C.B;
    int32_t stt = 0;
    F2M_CUDA(cudaMemcpyAsync(&stt, B.status, sizeof(stt), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if (stt != F2M_OK && stt != kNeedsHost) {
        R->status = stt;
        R->err = "instance exceeds a solver limit or did not converge";
        *out = R.release();
        return (f2m_status)stt;
    }
    H.perm.resize(S);
    H.F.resize(n_nodes);
    H.efcnt.resize(n_nodes);
    H.ccnt.resize(n_nodes);
    F2M_CUDA(cudaMemcpyAsync(H.perm.data(), B.perm, S * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(H.F.data(), B.F, n_nodes * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(H.efcnt.data(), B.efcnt, n_nodes * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(H.ccnt.data(), B.ccnt, n_nodes * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if ((s = pull_stats(ctx, C, 0, *R))) return s;
    if ((s = complete_instance(ctx, C, 0, prm, *R))) return s;
    if ((s = pull_stats(ctx, C, 0, *R))) return s;
    R->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = R.release();
    return (f2m_status)(*out)->status;
}

/* ------------------------------------------------------------------ */
/* smoothed bound (f2m_smooth.cu)                                       */
/* ------------------------------------------------------------------ */
void f2m_default_smooth_params(f2m_smooth_params* p) {
    p->tau = 1e-3;
    p->iters = 100;
    p->damping = 0.5;
    p->newton_max = 60;
    p->checkpoint = 16;
    p->solver = 0;
}

int32_t f2m_smooth_max_nodes(void) { return smooth_max_nodes(); }

f2m_status f2m_set_class_bounds(const int32_t* max_nodes) {
    if (!max_nodes) return F2M_ERR_INPUT;
    return solve_set_bounds(max_nodes) == 0 ? F2M_OK : F2M_ERR_INPUT;
}
void f2m_get_class_bounds(int32_t* max_nodes) { solve_get_bounds(max_nodes); }
f2m_status f2m_set_solver_smem_kb(int32_t kb) {
    return solve_set_smem_kb(kb) == 0 ? F2M_OK : F2M_ERR_INPUT;
}
int32_t f2m_get_solver_smem_kb(void) { return solve_get_smem_kb(); }

}  // extern "C"

namespace {

// The per-step launches (4 x iters + a few) as one CUDA graph: captured on
// the first call of a shape and replayed while the shape repeats (all kernel
// arguments are sizes, parameters and arena pointers, which the key covers;
// the data they point to is written before each replay).
cudaError_t smooth_steps_graph(f2m_ctx* ctx, SmoothBatch& B, bool grad) {
    int64_t tb, ob;
    std::memcpy(&tb, &B.tau, 8);
    std::memcpy(&ob, &B.omega, 8);
    const std::vector<int64_t> key{B.n_total, B.n_inst, B.N, B.iters, B.ckpt, B.newton_max, grad ? 1 : 0,
                                   tb, ob, (int64_t)(intptr_t)ctx->dev, (int64_t)ctx->dev_cap};
    if (ctx->sgraph && key == ctx->skey) {
        ctx->launches += ctx->sgraph_launches;
        return cudaGraphLaunch(ctx->sgraph, ctx->stream);
    }
    if (ctx->sgraph) {
        cudaGraphExecDestroy(ctx->sgraph);
        ctx->sgraph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    int64_t n = 0;
    const cudaError_t el = launch_smooth_steps(B, grad, ctx->stream, &n);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &g);
    if (el != cudaSuccess) e = el;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->sgraph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        ctx->sgraph = nullptr;
        return e;
    }
    ctx->skey = key;
    ctx->sgraph_launches = n;
    ctx->launches += n;
    return cudaGraphLaunch(ctx->sgraph, ctx->stream);
}

// Edge outputs of f2m_smoothed_bound_bwd_edges (all null for the other entries).
struct SmoothEdgesOut {
    int64_t cap = 0;
    int64_t* n_edges = nullptr;
    int32_t* a = nullptr;
    int32_t* b = nullptr;
    float* c = nullptr;
    double* dc = nullptr;
};

// Shared body of the smoothed-bound entry points: buffers from the context's
// arena, host inputs copied in, graph + bound (+ adjoint) on the device.
f2m_status smooth_call(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs, const float* x,
                       const float* y, int32_t top_k, const f2m_smooth_params* p,
                       const double* dL, double* L, float* gx, float* gy,
                       const SmoothEdgesOut* eo = nullptr) {
    if (!ctx) return F2M_ERR_INPUT;
    if (n_inst < 1 || !offs || !x || !y || !L) return fail(ctx, F2M_ERR_INPUT, "missing inputs");
    if (top_k < 3 || top_k > 64) return fail(ctx, F2M_ERR_INPUT, "top_k must be in [3, 64]");
    f2m_smooth_params sp;
    f2m_default_smooth_params(&sp);
    if (p) sp = *p;
    if (!(sp.tau > 0) || sp.iters < 0 || !(sp.damping > 0 && sp.damping <= 1) || sp.newton_max < 1 ||
        sp.checkpoint < 1 || sp.solver < 0 || sp.solver > 2)
        return fail(ctx, F2M_ERR_INPUT, "invalid smoothing parameters");
    if (offs[0] != 0) return fail(ctx, F2M_ERR_INPUT, "offs[0] must be 0");
    cudaSetDevice(ctx->device);
    const int32_t vmax = smooth_max_nodes();
    int32_t max_v = 0;
    for (int32_t b = 0; b < n_inst; ++b) {
        const int64_t v = offs[b + 1] - offs[b];
        if (v < 4) return fail(ctx, F2M_ERR_INPUT, "every instance needs at least 4 points");
        if (v > vmax)
            return fail(ctx, F2M_ERR_CAPACITY, "instances are limited to " + std::to_string(vmax) + " points");
        max_v = std::max<int32_t>(max_v, (int32_t)v);
    }
    const int64_t n = offs[n_inst];
    const bool grad = gx || gy;
    const int32_t N = top_k;
    const int32_t K = sp.checkpoint;
    const int32_t nck = std::max(1, (sp.iters + K - 1) / K);
    const int64_t S = 2 * n * N + 8 * n;  // union lists: own N + reverse (+ slack)
    const bool steps = sp.solver == 2 || (sp.solver == 0 && n_inst < ctx->sms);
    SmoothBatch B;
    int64_t* scan = nullptr;
    double* dLd = nullptr;
    auto carve_s = [&](Arena& A) {
        B.offs = A.take<int64_t>(n_inst + 1);
        B.x = A.take<float>(n);
        B.y = A.take<float>(n);
        B.top = A.take<unsigned long long>(n * N);
        B.rdeg = A.take<int32_t>(n);
        B.tcur = A.take<int32_t>(n);
        B.tcap = A.take<int64_t>(n + 1);
        B.tnbr = A.take<int32_t>(S);
        B.deg = A.take<int64_t>(n);
        B.row = A.take<int64_t>(n + 1);
        scan = A.take<int64_t>(scan_scratch_elems(n) + 1);
        B.nbr = A.take<int32_t>(S);
        B.mirror = A.take<int64_t>(S);
        B.c = A.take<float>(S);
        B.L = A.take<double>(n_inst);
        dLd = A.take<double>(n_inst);
        B.queue = A.take<int32_t>(1);
        B.work = A.take<unsigned long long>(1);
        if (steps) {
            B.ua = A.take<double>(n);
            B.ub = A.take<double>(n);
            B.Lp = A.take<double>(n);
        }
        if (grad) {
            B.ck = A.take<double>(n * nck);
            B.segu = A.take<double>(n * K);
            B.segs = A.take<double>(n * K);
            B.lam = A.take<double>(n);
            B.lam2 = A.take<double>(n);
            B.q = A.take<double>(S);
            B.gc = A.take<double>(S);
            B.gx = A.take<float>(n);
            B.gy = A.take<float>(n);
        }
    };
    Arena A;
    carve_s(A);
    F2M_CUDA(ensure_device(ctx, A.used));
    A.base = ctx->dev;
    A.used = 0;
    carve_s(A);
    ctx->timed = false;  // the arena no longer holds a solve batch
    B.n_inst = n_inst;
    B.N = N;
    B.n_total = n;
    B.tau = sp.tau;
    B.omega = sp.damping;
    B.iters = sp.iters;
    B.newton_max = sp.newton_max;
    B.ckpt = K;
    B.n_ck = nck;
    B.dL = dLd;
    std::vector<double> up(n_inst, 1.0);
    if (dL) std::copy(dL, dL + n_inst, up.begin());
    F2M_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(B.offs), offs, (n_inst + 1) * sizeof(int64_t),
                             cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<float*>(B.x), x, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<float*>(B.y), y, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(dLd, up.data(), n_inst * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(launch_smooth_graph(B, scan, ctx->stream, &ctx->launches));
    B.solver = steps ? 2 : 1;
    ctx->smooth_terms = -1;
    ctx->smooth_ms = 0.f;
    if (steps) {
        F2M_CUDA(smooth_steps_graph(ctx, B, grad));
    } else {
        F2M_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
        F2M_CUDA(launch_smooth_bound(B, max_v, grad, ctx->stream, &ctx->launches));
        F2M_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
    }
    F2M_CUDA(cudaMemcpyAsync(L, B.L, n_inst * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (gx) F2M_CUDA(cudaMemcpyAsync(gx, B.gx, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (gy) F2M_CUDA(cudaMemcpyAsync(gy, B.gy, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    unsigned long long terms = 0;
    if (!steps) F2M_CUDA(cudaMemcpyAsync(&terms, B.work, sizeof(terms), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!steps) {
        ctx->smooth_terms = (int64_t)terms;
        F2M_CUDA(cudaEventElapsedTime(&ctx->smooth_ms, ctx->ev[0], ctx->ev[1]));
    }
    if (eo && grad) {
        // edges once each (lower point first, in the lower endpoint's list
        // order) with dL/dc_e = the sum of the edge's two slot shares
        int64_t S_used = 0;
        F2M_CUDA(cudaMemcpy(&S_used, B.row + n, sizeof(int64_t), cudaMemcpyDeviceToHost));
        std::vector<int64_t> row(n + 1), mir(S_used);
        std::vector<int32_t> nb(S_used);
        std::vector<float> cc(S_used);
        std::vector<double> gc(S_used);
        F2M_CUDA(cudaMemcpy(row.data(), B.row, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(nb.data(), B.nbr, S_used * sizeof(int32_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(mir.data(), B.mirror, S_used * sizeof(int64_t), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(cc.data(), B.c, S_used * sizeof(float), cudaMemcpyDeviceToHost));
        F2M_CUDA(cudaMemcpy(gc.data(), B.gc, S_used * sizeof(double), cudaMemcpyDeviceToHost));
        int64_t m = 0;
        for (int32_t b = 0; b < n_inst; ++b)
            for (int64_t g = offs[b]; g < offs[b + 1]; ++g)
                for (int64_t k = row[g]; k < row[g + 1]; ++k) {
                    const int64_t j = offs[b] + nb[k];
                    if (j <= g) continue;
                    if (m < eo->cap) {
                        if (eo->a) eo->a[m] = (int32_t)g;
                        if (eo->b) eo->b[m] = (int32_t)j;
                        if (eo->c) eo->c[m] = cc[k];
                        if (eo->dc) eo->dc[m] = gc[k] + gc[mir[k]];
                    }
                    ++m;
                }
        *eo->n_edges = m;
        if (m > eo->cap) return fail(ctx, F2M_ERR_CAPACITY, "edge arrays hold fewer than the graph's edges");
    }
    return F2M_OK;
}

}  // namespace

extern "C" {

f2m_status f2m_smoothed_bound_fwd(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs, const float* x,
                                  const float* y, int32_t top_k, const f2m_smooth_params* p, double* L) {
    return smooth_call(ctx, n_inst, offs, x, y, top_k, p, nullptr, L, nullptr, nullptr);
}

f2m_status f2m_smoothed_bound_bwd(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs, const float* x,
                                  const float* y, int32_t top_k, const f2m_smooth_params* p,
                                  const double* dL, double* L, float* dL_dx, float* dL_dy) {
    if (!dL_dx || !dL_dy) return ctx ? fail(ctx, F2M_ERR_INPUT, "dL_dx and dL_dy are required") : F2M_ERR_INPUT;
    return smooth_call(ctx, n_inst, offs, x, y, top_k, p, dL, L, dL_dx, dL_dy);
}

f2m_status f2m_smoothed_bound_bwd_edges(f2m_ctx* ctx, int32_t n_inst, const int64_t* offs, const float* x,
                                        const float* y, int32_t top_k, const f2m_smooth_params* p,
                                        const double* dL, double* L, float* dL_dx, float* dL_dy,
                                        int64_t edge_cap, int64_t* n_edges, int32_t* edge_a,
                                        int32_t* edge_b, float* cost, double* dL_dc) {
    if (!dL_dx || !dL_dy || !n_edges || edge_cap < 0)
        return ctx ? fail(ctx, F2M_ERR_INPUT, "dL_dx, dL_dy and n_edges are required") : F2M_ERR_INPUT;
    SmoothEdgesOut eo;
    eo.cap = edge_cap;
    eo.n_edges = n_edges;
    eo.a = edge_a;
    eo.b = edge_b;
    eo.c = cost;
    eo.dc = dL_dc;
    return smooth_call(ctx, n_inst, offs, x, y, top_k, p, dL, L, dL_dx, dL_dy, &eo);
}

}  // extern "C"

namespace {

/* ------------------------------------------------------------------ */
/* TSPLIB input (FXY.hpp:186-309) on the host                           */
/* ------------------------------------------------------------------ */
struct FilePoints {
    std::vector<int> K;
    std::vector<double> X, Y;
    // duplicates[k0][k] (FXY.hpp:37,263)
    std::unordered_map<int, std::unordered_map<int, int>> duplicates;
};

f2m_status parse_tsplib(const std::string& path, FilePoints& P, std::string& err) {
    std::ifstream F(path);
    if (!F.is_open()) { err = "cannot open " + path; return F2M_ERR_INPUT; }
    std::string line, body;
    int start = 0, count = 0;
    while (std::getline(F, line)) {  // get_size (FXY.hpp:186-229)
        if (line.compare(0, 3, "EOF") == 0) break;
        if (start == 1) { count++; body += line; body += ' '; continue; }
        if (line.compare(0, 18, "NODE_COORD_SECTION") == 0) start = 1;
    }
    if (count == 0) { err = "file " + path + " is not in TSPLIB format"; return F2M_ERR_INPUT; }
    std::unordered_map<double, std::unordered_map<double, int>> filtr;  // FXY.hpp:233
    const char* p = body.c_str();
    for (;;) {  // get_KXY (FXY.hpp:241-291)
        int k = -1, n = 0;
        double x = 0, y = 0;
        int r = sscanf(p, "%d%n", &k, &n);
        if (r == EOF) break;
        if (r != 1) { err = "non-numeric token in NODE_COORD_SECTION"; return F2M_ERR_INPUT; }
        p += n;
        if (sscanf(p, "%lf%n", &x, &n) != 1) { err = "truncated coordinate triple"; return F2M_ERR_INPUT; }
        p += n;
        if (sscanf(p, "%lf%n", &y, &n) != 1) { err = "truncated coordinate triple"; return F2M_ERR_INPUT; }
        p += n;
        x = std::round(x * 1000);
        y = std::round(y * 1000);
        x /= 1000;
        y /= 1000;
        if (k <= -1) continue;
        auto fx = filtr.find(x);
        if (fx != filtr.end()) {
            auto fy = fx->second.find(y);
            if (fy != fx->second.end()) { P.duplicates[fy->second][k]++; continue; }
        }
        filtr[x][y] = k;
        P.K.push_back(k);
        P.X.push_back(x);
        P.Y.push_back(y);
    }
    return F2M_OK;
}

// One kNN list entry as the device produced it (FXY index space).
struct TopE {
    double cost;
    int em, oth, a, b;  // key (cost, em, oth); endpoints a<b
};
bool top_less(const TopE& x, const TopE& y) {
    if (x.cost != y.cost) return x.cost < y.cost;
    if (x.em != y.em) return x.em < y.em;
    return x.oth < y.oth;
}

// graph::graph (graph_tour.hpp:28-110) + graph_c::init (graph_cuda_init.hpp:3-70):
// kept edges in global order, nodes created in order of first appearance,
// internal ids in unordered_map<int,node*> iteration order.
void assemble_ref(const FilePoints& P, const std::vector<TopE>& kept, HostInst& H,
                  std::vector<int>& fxy_of) {
    const int n = (int)P.X.size();
    std::unordered_map<int, int> map_node;
    for (const TopE& e : kept) {
        const int ks[2] = {e.a, e.b};
        for (int f : ks)
            if (map_node.count(P.K[f]) == 0) map_node[P.K[f]] = f;
    }
    std::vector<int> id_of(n, -1);
    int iV = 0;
    fxy_of.clear();
    for (auto& kv : map_node) { id_of[kv.second] = iV++; fxy_of.push_back(kv.second); }
    H.V = iV;
    H.label.resize(iV);
    for (int v = 0; v < iV; ++v) H.label[v] = P.K[fxy_of[v]];
    H.E = (int)kept.size();
    H.ev1.resize(H.E); H.ev2.resize(H.E); H.el1.resize(H.E); H.el2.resize(H.E);
    H.rank1.resize(H.E); H.rank2.resize(H.E); H.eD.resize(H.E); H.eDo.resize(H.E);
    double dmin = 1e16;
    for (int e = 0; e < H.E; ++e) {
        const int u = id_of[kept[e].a], v = id_of[kept[e].b];
        H.ev1[e] = std::min(u, v); H.ev2[e] = std::max(u, v);
        if (H.label[u] < H.label[v]) { H.el1[e] = u; H.el2[e] = v; }
        else { H.el1[e] = v; H.el2[e] = u; }
        H.eDo[e] = kept[e].cost;
        dmin = std::min(dmin, kept[e].cost);
    }
    H.dmin = dmin;
    for (int e = 0; e < H.E; ++e) H.eD[e] = H.eDo[e] / dmin;
    H.row.assign(H.V + 1, 0);
    for (int e = 0; e < H.E; ++e) { H.row[H.ev1[e] + 1]++; H.row[H.ev2[e] + 1]++; }
    for (int v = 0; v < H.V; ++v) H.row[v + 1] += H.row[v];
    const int64_t S = H.row[H.V];
    H.nbr.assign(S, 0); H.Dn.assign(S, 0); H.cost.assign(S, 0); H.perm.assign(S, 0);
    H.mirror.assign(S, 0); H.slot_edge.assign(S, 0);
    std::vector<int64_t> fill(H.row.begin(), H.row.end() - 1);
    for (int e = 0; e < H.E; ++e) {
        const int u = H.ev1[e], v = H.ev2[e];
        const int64_t su = fill[u]++, sv = fill[v]++;
        H.nbr[su] = v; H.nbr[sv] = u;
        H.Dn[su] = H.Dn[sv] = H.eD[e];
        H.cost[su] = H.cost[sv] = H.eDo[e];
        H.slot_edge[su] = H.slot_edge[sv] = e;
        const int ru = (int)(su - H.row[u]), rv = (int)(sv - H.row[v]);
        H.perm[su] = (uint16_t)ru; H.perm[sv] = (uint16_t)rv;
        H.mirror[su] = rv; H.mirror[sv] = ru;
        if (H.el1[e] == u) { H.rank1[e] = ru; H.rank2[e] = rv; }
        else { H.rank1[e] = rv; H.rank2[e] = ru; }
    }
}

void write_outputs(const std::string& file, int top_k, const FilePoints& P, const std::vector<TopE>& dm,
                   const f2m_result& R) {
    const std::string base = file + ".top" + std::to_string(top_k);
    {   // FXY::save_to_file (FXY.hpp:146-165)
        std::ofstream f(base + ".DM");
        std::unordered_map<int, int> stat;
        for (const TopE& e : dm) {
            if (stat[e.a] > top_k && stat[e.b] > top_k) continue;
            stat[e.a]++;
            stat[e.b]++;
            f << e.a << " " << e.b << " " << e.cost << "\n";
        }
    }
    if (!P.duplicates.empty()) {  // FXY::save_to_file_duplicates (FXY.hpp:168-183)
        std::ofstream f(file + "_duplicates");
        for (auto& kv : P.duplicates) {
            f << "node used: " << kv.first << " duplicates: ";
            for (auto& kk : kv.second) f << kk.first << " ";
            f << "\n";
        }
    }
    {   // graph::print_file_report (graph_tour.hpp:218-241)
        std::ofstream f(base + ".F2M_report");
        if (R.status == F2M_OK) {
            f << "Optimal Found: " << "Yes" << "\n";
            f << "Optimal Value: " << std::setprecision(15) << R.lp << "\n";
            f << "Time: " << R.seconds << "\n";
            f << "MAX edge rank: " << R.max_rank << "\n";
        } else {
            f << "ERROR: Optimal Solution not Found\n";
        }
    }
    if (R.status == F2M_OK) {  // graph::print_file_solution (graph_tour.hpp:186-214)
        std::ofstream f(base + ".F2M_solution");
        for (auto& kv : R.X) {
            const int e = kv.first;
            f << R.H.label[R.H.el1[e]] << " " << R.H.label[R.H.el2[e]] << " " << std::setprecision(4)
              << kv.second << "\n";
        }
    }
}

}  // namespace

extern "C" {

f2m_status f2m_solve_file(f2m_ctx* ctx, const char* path, int32_t top_k, const f2m_params* params,
                          int32_t write_files, f2m_result** out) {
    *out = nullptr;
    if (!ctx) return F2M_ERR_INPUT;
    if (!path) return fail(ctx, F2M_ERR_INPUT, "no file");
    f2m_params prm;
    f2m_default_params(&prm);
    if (params) prm = *params;
    FilePoints FP;
    std::string err;
    f2m_status s = parse_tsplib(path, FP, err);
    if (s) return fail(ctx, s, err);
    const int32_t n = (int32_t)FP.X.size();
    const int64_t offs[2] = {0, n};
    if ((s = check_args(ctx, 1, offs, top_k, params))) return s;
    if (n < 4) return fail(ctx, F2M_ERR_INPUT, "fewer than 4 distinct points");
    cudaSetDevice(ctx->device);
    std::unique_ptr<f2m_result> R(new f2m_result());
    // kNN on the device with N+1 per node: the first N build the graph, all
    // N+1 give the .DM file (its cap is N+1 per node, FXY.hpp:156)
    const int32_t N1 = std::min(top_k + 1, 256);
    DevCall C;
    if ((s = setup_call(ctx, C, 1, offs, N1, prm, true))) return s;
    C.B.N_cut = top_k;
    int32_t* dK = C.B.cursor;
    C.B.K_in = dK;
    F2M_CUDA(cudaMemcpyAsync(dK, FP.K.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(C.B.offs), offs, 2 * sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.X_in), FP.X.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    F2M_CUDA(cudaMemcpyAsync(const_cast<double*>(C.B.Y_in), FP.Y.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    C.B.skip_dedup = 1;  // parse_tsplib removed the duplicates (FXY.hpp:260-267)
    F2M_CUDA(launch_prep(C.B, ctx->stream, &ctx->launches));
    F2M_CUDA(launch_knn(C.B, C.scan, ctx->stream, &ctx->launches));
    C.B.K_in = nullptr;
    int32_t st = 0;
    F2M_CUDA(cudaMemcpyAsync(&st, C.B.status, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<int32_t> ntop, tn, tem, toth;
    std::vector<double> tc;
    if ((s = d2h(ctx, ntop, C.B.ntop, n)) || (s = d2h(ctx, tn, C.B.top_nbr, (size_t)n * N1)) ||
        (s = d2h(ctx, tc, C.B.top_cost, (size_t)n * N1)) || (s = d2h(ctx, tem, C.B.top_em, (size_t)n * N1)) ||
        (s = d2h(ctx, toth, C.B.top_oth, (size_t)n * N1)))
        return s;
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if (st != F2M_OK) return fail(ctx, (f2m_status)st, "invalid instance (degenerate bounding box)");
    // union of the first N (graph) and first N+1 (.DM) of every node's list
    std::vector<TopE> kept, dm;
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < ntop[i]; ++k) {
            const int64_t o = (int64_t)i * N1 + k;
            const int j = tn[o];
            TopE e{tc[o], tem[o], toth[o], std::min(i, j), std::max(i, j)};
            dm.push_back(e);
            if (k < top_k) kept.push_back(e);
        }
    auto dedup = [](std::vector<TopE>& v) {
        std::sort(v.begin(), v.end(), top_less);
        size_t w = 0;
        for (size_t r = 0; r < v.size(); ++r)
            if (w == 0 || v[r].a != v[w - 1].a || v[r].b != v[w - 1].b || v[r].cost != v[w - 1].cost) v[w++] = v[r];
        v.resize(w);
    };
    dedup(kept);
    dedup(dm);
    HostInst& H = R->H;
    std::vector<int> fxy_of;
    assemble_ref(FP, kept, H, fxy_of);
    // upload the graph in the reference's node order as instance 0
    {
        std::vector<int64_t> row(H.row.begin(), H.row.end());
        std::vector<Slot> sl(H.nbr.size());
        for (size_t a = 0; a < sl.size(); ++a) {
            sl[a].D = H.Dn[a];
            sl[a].nbr = H.nbr[a];
            sl[a].aux = H.perm[a];
        }
        const int32_t Vn = H.V, ok = F2M_OK;
        unsigned long long db;
        std::memcpy(&db, &H.dmin, sizeof(db));
        if ((s = h2d(ctx, C.B.row, row)) || (s = h2d(ctx, C.B.slot, sl)) || (s = h2d(ctx, C.B.s_cost, H.cost)) ||
            (s = h2d(ctx, C.B.perm, H.perm)) || (s = h2d(ctx, C.B.mirror, H.mirror)))
            return s;
        F2M_CUDA(cudaMemcpyAsync(C.B.Vn, &Vn, sizeof(Vn), cudaMemcpyHostToDevice, ctx->stream));
        F2M_CUDA(cudaMemcpyAsync(C.B.status, &ok, sizeof(ok), cudaMemcpyHostToDevice, ctx->stream));
        F2M_CUDA(cudaMemcpyAsync(C.B.dmin_bits, &db, sizeof(db), cudaMemcpyHostToDevice, ctx->stream));
        F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    // graph::RUN (graph_cuda.cu:47-155), timed like dtimeRUN
    auto t0 = std::chrono::steady_clock::now();
    if (C.grid) {
        // nodes in the reference's order, points in file order: order the
        // nodes by their points (fxy_of, staged in the ownership buffer)
        std::vector<int32_t> pof(fxy_of.begin(), fxy_of.end());
        if ((s = h2d(ctx, C.G.own, pof))) return s;
        F2M_CUDA(launch_grid_order(C.B, C.G, 0, H.V, C.G.own, true, ctx->stream, &ctx->launches));
        F2M_CUDA(launch_solve_grid(C.B, to_dev(prm), C.G, 0, H.V, false, ctx->stream, &ctx->launches));
    } else {
        // the host-assembled graph may have fewer nodes than points: re-plan
        // the class from the node count
        std::vector<int32_t> one{0};
        const int c = solve_class_of(H.V);
        F2M_CUDA(cudaMemcpyAsync(C.ord, one.data(), sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
        F2M_CUDA(launch_solve_class(c, C.B, to_dev(prm), C.ord, 1, C.B.queue + 6,
                                    std::max<int32_t>(H.V, 4), ctx->stream, &ctx->launches));
    }
    F2M_CUDA(cudaMemcpyAsync(&st, C.B.status, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if (st != F2M_OK && st != kNeedsHost) return fail(ctx, (f2m_status)st, "the device solve stopped early");
    if ((s = d2h(ctx, H.F, C.B.F, H.V)) || (s = d2h(ctx, H.efcnt, C.B.efcnt, H.V)) ||
        (s = d2h(ctx, H.ccnt, C.B.ccnt, H.V)) || (s = d2h(ctx, H.perm, C.B.perm, H.nbr.size())))
        return s;
    F2M_CUDA(cudaStreamSynchronize(ctx->stream));
    if ((s = pull_stats(ctx, C, 0, *R))) return s;
    if ((s = complete_instance(ctx, C, 0, prm, *R))) return s;
    R->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if ((s = pull_stats(ctx, C, 0, *R))) return s;
    if (write_files) write_outputs(path, top_k, FP, dm, *R);
    *out = R.release();
    return (f2m_status)(*out)->status;
}

void f2m_result_free(f2m_result* r) { delete r; }
int32_t f2m_result_status(const f2m_result* r) { return r->status; }
int32_t f2m_result_n_nodes(const f2m_result* r) { return r->H.V; }
int32_t f2m_result_n_edges(const f2m_result* r) { return r->H.E; }
double f2m_result_lp(const f2m_result* r) { return r->lp; }
int32_t f2m_result_max_rank(const f2m_result* r) { return r->max_rank; }
double f2m_result_seconds(const f2m_result* r) { return r->seconds; }

void f2m_result_edges(const f2m_result* r, int32_t* v1, int32_t* v2, int32_t* lab1, int32_t* lab2,
                      double* Do, double* D, double* x) {
    const HostInst& H = r->H;
    parallel_for(H.E, [&](int64_t e0, int64_t e1) {
        for (int64_t e = e0; e < e1; ++e) {
            if (v1) v1[e] = H.ev1[e];
            if (v2) v2[e] = H.ev2[e];
            if (lab1) lab1[e] = H.label[H.el1[e]];
            if (lab2) lab2[e] = H.label[H.el2[e]];
            if (Do) Do[e] = H.eDo[e];
            if (D) D[e] = H.eD[e];
            if (x) x[e] = e < (int64_t)r->x.size() ? r->x[e] : 0.0;
        }
    });
}
void f2m_result_nodes(const f2m_result* r, int32_t* label, double* F) {
    for (int v = 0; v < r->H.V; ++v) {
        if (label) label[v] = r->H.label[v];
        if (F) F[v] = r->H.F[v];
    }
}
void f2m_result_stats(const f2m_result* r, f2m_stats* s) { *s = r->st; }

}  // extern "C"

/* ------------------------------------------------------------------ */
/* Allocation-free single-instance solve                                */
/* ------------------------------------------------------------------ */
// Some callers cannot allocate device memory while they run: a host
// application that owns the whole GPU through its own memory pool and
// forbids foreign cudaMalloc/cudaFree, or a latency-critical loop where a
// cudaMalloc (which may synchronize the device and has no latency bound) is
// not acceptable.  For them this entry point takes its scratch from one
// fixed array in device memory and allocates nothing itself: no
// cudaMalloc/cudaFree, no pinned or pageable host buffers, no library call
// that allocates.  With CUDA's lazy module loading (the default) the array and
// the solver's kernels are put on a device by the first call there, so
// callers make one warm-up call during their own set-up, before their pool
// takes the GPU and before any stream capture (CUDA_MODULE_LOADING=EAGER
// moves this to library load).  It is limited to one instance of at most
// kNoAllocMaxPoints points and kNoAllocMaxN neighbours, always runs the
// per-instance team solver, and runs only the device stages (instances whose
// combs need the host Ax=b stage are reported, not completed).
namespace {

constexpr int32_t kNoAllocMaxPoints = 2048;
constexpr int32_t kNoAllocMaxN = 24;
constexpr size_t kNoAllocBytes = (size_t)12 << 20;  // 12 MiB of device memory per GPU

// The scratch of f2m_solve_points_noalloc.  In host code this name is only a
// stand-in for the device symbol: its device address comes from
// cudaGetSymbolAddress (one per device, see noalloc_scratch()).
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 256;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device, looked up the
// first time this device is used.  A device reset (cudaDeviceReset, or
// anything else that re-creates the primary context) unmaps the array and
// leaves the saved address stale: callers of this entry point do not reset
// the device between calls.
cudaError_t noalloc_scratch(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

// Work lists of one instance written on the device (no host staging).
__global__ void k_noalloc_setup(int64_t* offs, int32_t* chunk_inst, int32_t* chunk_start, int32_t* order,
                                int32_t n, int32_t n_chunks) {
    const int t = threadIdx.x;
    if (t == 0) { offs[0] = 0; offs[1] = n; order[0] = 0; }
    for (int c = t; c < n_chunks; c += blockDim.x) { chunk_inst[c] = 0; chunk_start[c] = c * kChunk; }
}

// Copies the result out; an instance that needs the host comb stage is
// reported as F2M_ERR_CAPACITY.
__global__ void k_noalloc_finish(const int32_t* st_in, const double* lp_in, int32_t* st_out, double* lp_out) {
    if (threadIdx.x == 0) {
        const int32_t st = st_in[0];
        *st_out = (st == kNeedsHost) ? (int32_t)F2M_ERR_CAPACITY : st;
        *lp_out = (st == F2M_OK) ? lp_in[0] : NAN;
    }
}

}  // namespace

extern "C" f2m_status f2m_solve_points_noalloc(const double* d_x, const double* d_y, int32_t n, int32_t top_k,
                                                const f2m_params* params, double* d_lp, int32_t* d_status,
                                                void* stream) {
    if (!d_x || !d_y || !d_lp || !d_status) return F2M_ERR_INPUT;
    if (n < 4 || top_k < 3) return F2M_ERR_INPUT;
    if (n > kNoAllocMaxPoints || top_k > kNoAllocMaxN) return F2M_ERR_CAPACITY;
    if (params && params->cost_mode != F2M_COST_REF_EUCLID) return F2M_ERR_INPUT;
    if (params && params->solver == 2) return F2M_ERR_INPUT;  // the whole-GPU solver needs its own buffers
    f2m_params prm;
    f2m_default_params(&prm);
    if (params) prm = *params;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    // buffers of one instance carved from the fixed array (vectors stay empty)
    Plan pl;
    pl.n_inst = 1;
    pl.n_total = n;
    pl.max_n = n;
    pl.N = top_k;
    pl.S_cap = 2 * (int64_t)std::min(top_k, n - 1) * n;
    const int32_t n_chunks = (n + kChunk - 1) / kChunk;
    Batch B{};
    int64_t *deg = nullptr, *scan = nullptr;
    int32_t *ci = nullptr, *cs = nullptr, *ord = nullptr;
    Arena A;
    carve(A, B, pl, true, &deg, &scan, &ci, &cs, &ord, n_chunks);
    if (A.used > kNoAllocBytes) return F2M_ERR_CAPACITY;
    void* base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess) return F2M_ERR_CUDA;
    A.base = static_cast<char*>(base);
    A.used = 0;
    carve(A, B, pl, true, &deg, &scan, &ci, &cs, &ord, n_chunks);
    B.X_in = d_x;
    B.Y_in = d_y;
    B.skip_dedup = 0;
    int64_t launches = 0;
    k_noalloc_setup<<<1, 256, 0, s>>>(const_cast<int64_t*>(B.offs), ci, cs, ord, n, n_chunks);
    if (cudaGetLastError() != cudaSuccess) return F2M_ERR_CUDA;
    if (launch_prep(B, s, &launches) != cudaSuccess || launch_knn(B, scan, s, &launches) != cudaSuccess ||
        launch_graph(B, deg, scan, s, &launches) != cudaSuccess ||
        launch_solve_class(solve_class_of(n), B, to_dev(prm), ord, 1, B.queue, std::max<int32_t>(n, 4), s,
                           &launches) != cudaSuccess ||
        launch_axb(B, to_dev(prm), s, &launches) != cudaSuccess)
        return F2M_ERR_CUDA;
    k_noalloc_finish<<<1, 32, 0, s>>>(B.status, B.lp, d_status, d_lp);
    if (cudaGetLastError() != cudaSuccess) return F2M_ERR_CUDA;
    return F2M_OK;
}
