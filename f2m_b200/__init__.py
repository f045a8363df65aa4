"""f2m_b200: B200-native F2M (fractional 2-matching) solver.

Python binding of the C ABI in include/f2m.h (libf2m_b200.so, built in-tree
for sm_100a by f2m_b200/build.py).  The surface mirrors the reference's
F2M.h graph API:

    g = graph("file.tsp", 20)   # graph(std::string file, int E_max), F2M.h:181
    graph_c(g)                  # graph_c(graph*), F2M.h:320
    g.RUN()                     # graph::RUN(), F2M.h:175 -- writes the report files
    g.X                         # graph::X, F2M.h:161: {edge id: x}

plus batched and in-memory entry points (solve_batch, solve_points).  There is
no CPU fallback: without the CUDA library or a device every call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libf2m_b200.so")

OK, ERR_INPUT, ERR_CAPACITY, ERR_NOT_CONVERGED, ERR_CUDA, ERR_NO_DEVICE = range(6)
COST_REF_EUCLID, COST_NINT = 0, 1
STATUS_NAMES = {0: "OK", 1: "ERR_INPUT", 2: "ERR_CAPACITY", 3: "ERR_NOT_CONVERGED",
                4: "ERR_CUDA", 5: "ERR_NO_DEVICE"}


class F2MError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"f2m status {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Params(ctypes.Structure):
    """f2m_params: the reference's constants (defaults from f2m_default_params)."""
    _fields_ = [
        ("error_B", ctypes.c_double), ("error_B_comb", ctypes.c_double),
        ("glob_K", ctypes.c_int32), ("glob_rounds", ctypes.c_int32),
        ("glob_inner", ctypes.c_int32), ("glob_tol", ctypes.c_double),
        ("factor0", ctypes.c_int32), ("factor_step", ctypes.c_int32),
        ("factor_cap", ctypes.c_int32), ("max_rounds", ctypes.c_int32),
        ("fix_rounds", ctypes.c_int32), ("fix_factor", ctypes.c_int32),
        ("check_every", ctypes.c_int32), ("frozen_iters", ctypes.c_int32),
        ("ef_thr", ctypes.c_double), ("ef_small_deg", ctypes.c_int32),
        ("ef_min", ctypes.c_int32), ("comb_thr", ctypes.c_double),
        ("shift0", ctypes.c_double), ("shift_max", ctypes.c_double),
        ("max_iters", ctypes.c_int64), ("cost_mode", ctypes.c_int32),
        ("solver", ctypes.c_int32), ("grid_spin_limit", ctypes.c_int64),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int64), ("checks", ctypes.c_int32),
        ("n_combs", ctypes.c_int32), ("irr_a", ctypes.c_int32), ("irr_b", ctypes.c_int32),
        ("repair_steps", ctypes.c_int32), ("degree_violations", ctypes.c_int32),
        ("max_grad", ctypes.c_double), ("d_min", ctypes.c_double),
        ("dual_value", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Work(ctypes.Structure):
    _fields_ = [("node_iters", ctypes.c_int64), ("slot_iters", ctypes.c_int64),
                ("slots", ctypes.c_int64), ("points", ctypes.c_int64),
                ("pad_iters", ctypes.c_int64), ("lane_iters", ctypes.c_int64)]


class BatchOut(ctypes.Structure):
    _fields_ = [("lp", ctypes.c_void_p), ("status", ctypes.c_void_p),
                ("n_nodes", ctypes.c_void_p), ("n_edges", ctypes.c_void_p),
                ("n_combs", ctypes.c_void_p), ("max_rank", ctypes.c_void_p),
                ("iterations", ctypes.c_void_p), ("n_irregular", ctypes.c_void_p)]


class SmoothParams(ctypes.Structure):
    _fields_ = [("tau", ctypes.c_double), ("iters", ctypes.c_int32), ("damping", ctypes.c_double),
                ("newton_max", ctypes.c_int32), ("checkpoint", ctypes.c_int32),
                ("solver", ctypes.c_int32)]


# Every symbol include/f2m.h declares.
EXPORTS = [
    "f2m_default_params", "f2m_create", "f2m_destroy", "f2m_last_error", "f2m_kernel_launches",
    "f2m_solve_batch", "f2m_solve_batch_device", "f2m_sync", "f2m_solve_points",
    "f2m_solve_file", "f2m_result_free", "f2m_result_status", "f2m_result_n_nodes",
    "f2m_result_n_edges", "f2m_result_lp", "f2m_result_max_rank", "f2m_result_seconds",
    "f2m_result_edges", "f2m_result_nodes", "f2m_result_stats", "f2m_phase_times",
    "f2m_solve_points_noalloc", "f2m_default_smooth_params", "f2m_smoothed_bound_fwd",
    "f2m_smoothed_bound_bwd", "f2m_smooth_max_nodes", "f2m_knn", "f2m_set_class_bounds",
    "f2m_get_class_bounds", "f2m_solve_graph", "f2m_solve_points_from", "f2m_fp64_rate",
    "f2m_partition_selfcheck", "f2m_smooth_work",
    "f2m_smoothed_bound_bwd_edges", "f2m_set_solver_smem_kb", "f2m_get_solver_smem_kb",
]

_lib = None


def lib():
    """Load libf2m_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise F2MError(ERR_NO_DEVICE, f"{LIB_PATH} is missing: run f2m_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        P = ctypes.POINTER
        L.f2m_default_params.argtypes = [P(Params)]
        L.f2m_create.argtypes = [P(vp), ctypes.c_int]
        L.f2m_destroy.argtypes = [vp]
        L.f2m_last_error.argtypes = [vp]
        L.f2m_last_error.restype = ctypes.c_char_p
        L.f2m_kernel_launches.argtypes = [vp]
        L.f2m_kernel_launches.restype = i64
        L.f2m_sync.argtypes = [vp]
        L.f2m_solve_batch.argtypes = [vp, i32, vp, vp, vp, i32, P(Params), P(BatchOut)]
        L.f2m_solve_batch_device.argtypes = [vp, i32, vp, vp, vp, vp, i32, P(Params), P(BatchOut)]
        L.f2m_solve_points.argtypes = [vp, vp, vp, vp, i32, i32, P(Params), P(vp)]
        L.f2m_knn.argtypes = [vp, vp, vp, vp, i32, i32, P(vp)]
        L.f2m_solve_points_from.argtypes = [vp, vp, vp, vp, i32, i32, vp, i32, P(Params), P(vp)]
        L.f2m_solve_graph.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp, P(Params), P(vp)]
        L.f2m_solve_file.argtypes = [vp, ctypes.c_char_p, i32, P(Params), i32, P(vp)]
        L.f2m_result_free.argtypes = [vp]
        for name in ("f2m_result_status", "f2m_result_n_nodes", "f2m_result_n_edges",
                     "f2m_result_max_rank"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = i32
        for name in ("f2m_result_lp", "f2m_result_seconds"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = dbl
        L.f2m_result_edges.argtypes = [vp] * 8
        L.f2m_result_nodes.argtypes = [vp] * 3
        L.f2m_result_stats.argtypes = [vp, P(Stats)]
        L.f2m_phase_times.argtypes = [vp, vp, P(Work)]
        L.f2m_fp64_rate.argtypes = [vp, i32, i32, P(dbl)]
        L.f2m_partition_selfcheck.argtypes = [vp, i32, ctypes.c_uint64, P(ctypes.c_int64)]
        L.f2m_smooth_work.argtypes = [vp, P(ctypes.c_int64), P(ctypes.c_float)]
        L.f2m_solve_points_noalloc.argtypes = [vp, vp, i32, i32, P(Params), vp, vp, vp]
        L.f2m_default_smooth_params.argtypes = [P(SmoothParams)]
        L.f2m_smoothed_bound_fwd.argtypes = [vp, i32, vp, vp, vp, i32, P(SmoothParams), vp]
        L.f2m_smoothed_bound_bwd.argtypes = [vp, i32, vp, vp, vp, i32, P(SmoothParams), vp, vp,
                                             vp, vp]
        L.f2m_smoothed_bound_bwd_edges.argtypes = [vp, i32, vp, vp, vp, i32, P(SmoothParams), vp,
                                                   vp, vp, vp, i64, P(i64), vp, vp, vp, vp]
        L.f2m_smooth_max_nodes.restype = i32
        L.f2m_set_class_bounds.argtypes = [vp]
        L.f2m_get_class_bounds.argtypes = [vp]
        L.f2m_set_solver_smem_kb.argtypes = [i32]
        L.f2m_get_solver_smem_kb.restype = i32
        _lib = L
    return _lib


def default_params(**overrides):
    p = Params()
    lib().f2m_default_params(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def set_class_bounds(bounds):
    """Size-class bounds of the batched solver (3 increasing point counts)."""
    b = np.ascontiguousarray(bounds, np.int32)
    s = lib().f2m_set_class_bounds(b.ctypes.data_as(ctypes.c_void_p))
    if s != OK:
        raise F2MError(s, f"class bounds {list(bounds)} rejected")


def get_class_bounds():
    b = np.zeros(3, np.int32)
    lib().f2m_get_class_bounds(b.ctypes.data_as(ctypes.c_void_p))
    return [int(v) for v in b]


def set_solver_smem_kb(kb):
    """Shared memory (KB) a CTA of the batched solver takes; 0 = all of it."""
    s = lib().f2m_set_solver_smem_kb(int(kb))
    if s != OK:
        raise F2MError(s, f"solver shared memory {kb} KB rejected")


def get_solver_smem_kb():
    return int(lib().f2m_get_solver_smem_kb())


def load_tuning(path=None):
    """Apply the class bounds (and the solver's shared-memory target, when
    recorded) of f2m_b200.autotune (default: the committed
    f2m_b200/tuned_classes.json); returns the bounds, or None."""
    import json
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_classes.json")
    if not os.path.exists(path):
        return None
    rec = json.load(open(path))
    set_class_bounds(rec["bounds"])
    if "smem_kb" in rec:
        set_solver_smem_kb(rec["smem_kb"])
    return rec["bounds"]


def default_smooth_params(**overrides):
    p = SmoothParams()
    lib().f2m_default_smooth_params(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Context:
    """One f2m context (one CUDA stream on one device)."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        s = lib().f2m_create(ctypes.byref(self._h), device)
        if s != OK:
            raise F2MError(s, "no usable CUDA device")

    def close(self):
        if self._h:
            lib().f2m_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def last_error(self):
        return lib().f2m_last_error(self._h).decode()

    def kernel_launches(self):
        return lib().f2m_kernel_launches(self._h)

    def _check(self, s):
        if s not in (OK, ERR_NOT_CONVERGED):
            raise F2MError(s, self.last_error())
        return s

    # -- batched ----------------------------------------------------------
    def solve_batch(self, offs, x, y, top_k, params=None, details=False):
        """Solve independent instances; offs[b]..offs[b+1] index x/y (host arrays).

        Returns (lp, status) or, with details=True, a dict of all per-instance
        outputs."""
        offs = np.ascontiguousarray(offs, np.int64)
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        n = len(offs) - 1
        lp = np.zeros(n, np.float64)
        st = np.zeros(n, np.int32)
        o = BatchOut(lp=lp.ctypes.data, status=st.ctypes.data)
        extra = {}
        if details:
            for k, dt in (("n_nodes", np.int32), ("n_edges", np.int32), ("n_combs", np.int32),
                          ("max_rank", np.int32), ("iterations", np.int64),
                          ("n_irregular", np.int32)):
                extra[k] = np.zeros(n, dt)
                setattr(o, k, extra[k].ctypes.data)
        p = params if params is not None else default_params()
        self._check(lib().f2m_solve_batch(self._h, n, _ptr(offs), _ptr(x), _ptr(y), top_k,
                                          ctypes.byref(p), ctypes.byref(o)))
        if details:
            extra.update(lp=lp, status=st)
            return extra
        return lp, st

    def solve_batch_device(self, h_offs, d_offs, d_x, d_y, top_k, d_lp, d_status, params=None,
                           d_iterations=None):
        """Device-resident batch: d_* are device addresses (ints); outputs too."""
        h_offs = np.ascontiguousarray(h_offs, np.int64)
        n = len(h_offs) - 1
        o = BatchOut(lp=d_lp, status=d_status, iterations=d_iterations)
        p = params if params is not None else default_params()
        self._check(lib().f2m_solve_batch_device(self._h, n, _ptr(h_offs), ctypes.c_void_p(d_offs),
                                                 ctypes.c_void_p(d_x), ctypes.c_void_p(d_y), top_k,
                                                 ctypes.byref(p), ctypes.byref(o)))

    def sync(self):
        self._check(lib().f2m_sync(self._h))

    def phase_times(self):
        """(ms per phase [prep, knn, graph, solve], work counters) of the last batch."""
        ms = np.zeros(4, np.float32)
        w = Work()
        self._check(lib().f2m_phase_times(self._h, _ptr(ms), ctypes.byref(w)))
        return ms, {k: getattr(w, k) for k, _ in Work._fields_}

    def fp64_rate(self, kind=0, repeats=3):
        """Measured FP64 pipe rate of this GPU, FP64 lane operations per second
        (kind 0: DADD, kind 1: DSETP; the roofline of the dual descent), or
        kind 2: logistic terms per second (the smoothed bound's roofline)."""
        r = ctypes.c_double()
        self._check(lib().f2m_fp64_rate(self._h, kind, repeats, ctypes.byref(r)))
        return r.value

    def smooth_work(self):
        """(logistic terms, kernel ms) of the last smoothed-bound call's
        persistent kernel; terms is -1 after the one-launch-per-step path."""
        t = ctypes.c_int64()
        ms = ctypes.c_float()
        self._check(lib().f2m_smooth_work(self._h, ctypes.byref(t), ctypes.byref(ms)))
        return t.value, ms.value

    def partition_selfcheck(self, n_cases=100000, seed=1):
        """Lists on which the warp-cooperative partition and the serial one
        disagree (order or count) over n_cases seeded lists; 0 when exact."""
        r = ctypes.c_int64()
        self._check(lib().f2m_partition_selfcheck(self._h, n_cases, seed, ctypes.byref(r)))
        return r.value

    # -- single instance ----------------------------------------------------
    # -- smoothed bound (no counterpart in the reference) ------------------
    def smoothed_bound(self, offs, x, y, top_k, params=None, grad=False, dL=None):
        """Smoothed F2M dual bound per instance (FP32 points); with grad=True
        also d(sum_b dL[b] L[b]) / d(x, y).  Returns L or (L, dL_dx, dL_dy)."""
        offs = np.ascontiguousarray(offs, np.int64)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        n = len(offs) - 1
        p = params if params is not None else default_smooth_params()
        L = np.zeros(n, np.float64)
        if not grad:
            self._check(lib().f2m_smoothed_bound_fwd(self._h, n, _ptr(offs), _ptr(x), _ptr(y), top_k,
                                                     ctypes.byref(p), _ptr(L)))
            return L
        gx = np.zeros(len(x), np.float32)
        gy = np.zeros(len(y), np.float32)
        up = None if dL is None else np.ascontiguousarray(dL, np.float64)
        self._check(lib().f2m_smoothed_bound_bwd(self._h, n, _ptr(offs), _ptr(x), _ptr(y), top_k,
                                                 ctypes.byref(p), _ptr(up), _ptr(L), _ptr(gx),
                                                 _ptr(gy)))
        return L, gx, gy

    def smoothed_bound_edges(self, offs, x, y, top_k, params=None, dL=None):
        """Backward with the edge-cost gradient: returns (L, dL_dx, dL_dy, edges)
        where edges = (a, b, c, dL_dc): each edge once (a < b, global point
        indices), its FP32 cost and d(sum_b dL[b] L[b]) / dc_e."""
        offs = np.ascontiguousarray(offs, np.int64)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        n = len(offs) - 1
        p = params if params is not None else default_smooth_params()
        L = np.zeros(n, np.float64)
        gx = np.zeros(len(x), np.float32)
        gy = np.zeros(len(y), np.float32)
        cap = len(x) * int(top_k)
        a = np.zeros(cap, np.int32)
        b = np.zeros(cap, np.int32)
        c = np.zeros(cap, np.float32)
        dc = np.zeros(cap, np.float64)
        m = ctypes.c_int64()
        up = None if dL is None else np.ascontiguousarray(dL, np.float64)
        self._check(lib().f2m_smoothed_bound_bwd_edges(
            self._h, n, _ptr(offs), _ptr(x), _ptr(y), top_k, ctypes.byref(p), _ptr(up), _ptr(L),
            _ptr(gx), _ptr(gy), cap, ctypes.byref(m), _ptr(a), _ptr(b), _ptr(c), _ptr(dc)))
        k = m.value
        return L, gx, gy, (a[:k], b[:k], c[:k], dc[:k])

    def solve_graph(self, n_nodes, v1, v2, D, Do, labels=None, params=None):
        """graph_c + RUN on a caller-built graph (edges in the reference's order)."""
        v1 = np.ascontiguousarray(v1, np.int32)
        v2 = np.ascontiguousarray(v2, np.int32)
        D = np.ascontiguousarray(D, np.float64)
        Do = np.ascontiguousarray(Do, np.float64)
        lab = None if labels is None else np.ascontiguousarray(labels, np.int32)
        h = ctypes.c_void_p()
        p = params if params is not None else default_params()
        s = lib().f2m_solve_graph(self._h, int(n_nodes), len(v1), _ptr(v1), _ptr(v2), _ptr(D), _ptr(Do),
                                  _ptr(lab), ctypes.byref(p), ctypes.byref(h))
        return self._result(s, h)

    def solve_points_from(self, x, y, top_k, F0, labels=None, params=None):
        """Resume the descent from stored potentials F0 (node order of a result)."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        F0 = np.ascontiguousarray(F0, np.float64)
        lab = None if labels is None else np.ascontiguousarray(labels, np.int32)
        h = ctypes.c_void_p()
        p = params if params is not None else default_params()
        s = lib().f2m_solve_points_from(self._h, _ptr(x), _ptr(y), _ptr(lab), len(x), top_k, _ptr(F0),
                                        len(F0), ctypes.byref(p), ctypes.byref(h))
        return self._result(s, h)

    def knn(self, x, y, top_k, labels=None):
        """The kNN graph alone (edges in the reference's order; F and x are 0)."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        lab = None if labels is None else np.ascontiguousarray(labels, np.int32)
        h = ctypes.c_void_p()
        s = lib().f2m_knn(self._h, _ptr(x), _ptr(y), _ptr(lab), len(x), top_k, ctypes.byref(h))
        return self._result(s, h)

    def solve_points(self, x, y, top_k, labels=None, params=None):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        lab = None if labels is None else np.ascontiguousarray(labels, np.int32)
        h = ctypes.c_void_p()
        p = params if params is not None else default_params()
        s = lib().f2m_solve_points(self._h, _ptr(x), _ptr(y), _ptr(lab), len(x), top_k,
                                   ctypes.byref(p), ctypes.byref(h))
        return self._result(s, h)

    def solve_file(self, path, top_k, params=None, write_files=False):
        h = ctypes.c_void_p()
        p = params if params is not None else default_params()
        s = lib().f2m_solve_file(self._h, os.fsencode(path), top_k, ctypes.byref(p),
                                 1 if write_files else 0, ctypes.byref(h))
        return self._result(s, h)

    def _result(self, s, h):
        if not h:
            raise F2MError(s, self.last_error())
        try:
            if s not in (OK, ERR_NOT_CONVERGED):
                raise F2MError(s, self.last_error() or "invalid instance")
            return Result(h)
        finally:
            lib().f2m_result_free(h)


class Result:
    """Host copy of one solved instance (graph + potentials + primal)."""

    def __init__(self, h):
        L = lib()
        self.status = L.f2m_result_status(h)
        self.n_nodes = L.f2m_result_n_nodes(h)
        self.n_edges = L.f2m_result_n_edges(h)
        self.lp = L.f2m_result_lp(h)
        self.max_rank = L.f2m_result_max_rank(h)
        self.seconds = L.f2m_result_seconds(h)
        ne, nv = self.n_edges, self.n_nodes
        # every element is written by the library (its host threads fill the
        # arrays side by side), so no zero fill
        self.v1 = np.empty(ne, np.int32)
        self.v2 = np.empty(ne, np.int32)
        self.lab1 = np.empty(ne, np.int32)
        self.lab2 = np.empty(ne, np.int32)
        self.Do = np.empty(ne, np.float64)
        self.D = np.empty(ne, np.float64)
        self.x = np.empty(ne, np.float64)
        if ne:
            L.f2m_result_edges(h, *(_ptr(a) for a in (self.v1, self.v2, self.lab1, self.lab2,
                                                      self.Do, self.D, self.x)))
        self.label = np.empty(nv, np.int32)
        self.F = np.empty(nv, np.float64)
        if nv:
            L.f2m_result_nodes(h, _ptr(self.label), _ptr(self.F))
        st = Stats()
        L.f2m_result_stats(h, ctypes.byref(st))
        self.stats = st.as_dict()

    def edge_set(self):
        a = np.minimum(self.lab1, self.lab2)
        b = np.maximum(self.lab1, self.lab2)
        return set(zip(a.tolist(), b.tolist()))

    @property
    def X(self):
        """graph::X: {edge id: x} for edges in the primal solution."""
        nz = np.nonzero(self.x)[0]
        return {int(e): float(self.x[e]) for e in nz}


def solve_points_noalloc(d_x, d_y, n, top_k, d_lp, d_status, stream=0, params=None):
    """Allocation-free solve of one instance (device pointers as ints; see
    f2m_solve_points_noalloc in include/f2m.h for who needs it and its
    limits).  Only enqueues on `stream`; returns the f2m status of the call."""
    p = params if params is not None else default_params()
    return lib().f2m_solve_points_noalloc(ctypes.c_void_p(d_x), ctypes.c_void_p(d_y), n, top_k,
                                          ctypes.byref(p), ctypes.c_void_p(d_lp),
                                          ctypes.c_void_p(d_status), ctypes.c_void_p(stream))


# ---------------------------------------------------------------------------
# The reference's graph API (F2M.h) over the context
# ---------------------------------------------------------------------------
_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class graph:
    """graph(file, E_max) -- F2M.h:181.  RUN() solves and writes the report files."""

    def __init__(self, file, E_max, params=None, ctx=None):
        self.file = file
        self.E_max = int(E_max)
        self.params = params
        self.ctx = ctx or default_context()
        self.result = None
        self.X = {}

    def RUN(self):
        """graph::RUN (graph_cuda.cu:47-155)."""
        self.result = self.ctx.solve_file(self.file, self.E_max, self.params, write_files=True)
        self.X = self.result.X
        return self.result


def graph_c(g):
    """graph_c(graph*) -- F2M.h:320.  Device set-up happens inside RUN()."""
    return g
