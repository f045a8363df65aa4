"""ctypes binding of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference F2M solver on the CPU (see f2m_oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

COST_REF, COST_NINT = 0, 1
ID_REF, ID_FXY = 0, 1
KNN_LITERAL, KNN_TOPN = 0, 1
OK, ERR_INPUT, ERR_CAPACITY, ERR_NOT_CONVERGED = 0, 1, 2, 3


class Stats(ctypes.Structure):
    _fields_ = [
        ("iters_glob", ctypes.c_int64),
        ("iters_ef", ctypes.c_int64),
        ("iters_repair", ctypes.c_int64),
        ("checks", ctypes.c_int32),
        ("glob_rounds", ctypes.c_int32),
        ("ef_rounds", ctypes.c_int32),
        ("n_combs", ctypes.c_int32),
        ("irr_a", ctypes.c_int32),
        ("irr_b", ctypes.c_int32),
        ("repair_steps", ctypes.c_int32),
        ("ef_slots", ctypes.c_int64),
        ("max_grad", ctypes.c_double),
        ("d_min", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        L.orc_solve_file.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, P(vp)]
        L.orc_solve_points.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, P(vp)]
        L.orc_build_graph.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, P(vp)]
        L.orc_solve_graph.argtypes = [ctypes.c_int32, ctypes.c_int32, vp, vp, vp, vp, vp,
                                      ctypes.c_int, P(vp)]
        L.orc_free.argtypes = [vp]
        L.orc_error.argtypes = [vp]
        L.orc_error.restype = ctypes.c_char_p
        for name in ("orc_status", "orc_num_nodes", "orc_num_edges", "orc_num_points",
                     "orc_max_rank"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = ctypes.c_int32
        L.orc_lp_value.argtypes = [vp]
        L.orc_lp_value.restype = ctypes.c_double
        L.orc_size_per_node.argtypes = [vp]
        L.orc_size_per_node.restype = ctypes.c_double
        L.orc_get_edges.argtypes = [vp] * 7
        L.orc_get_nodes.argtypes = [vp] * 3
        L.orc_get_F.argtypes = [vp, vp]
        L.orc_get_x.argtypes = [vp, vp]
        L.orc_get_stats.argtypes = [vp, P(Stats)]
        L.orc_get_combs.argtypes = [vp, vp, vp]
        L.orc_get_combs.restype = ctypes.c_int32
        L.orc_get_statab.argtypes = [vp, vp, vp]
        L.orc_get_cutoffs.argtypes = [vp, vp, vp]
        L.orc_solve_batch.argtypes = [ctypes.c_int32, vp, vp, vp, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, vp, vp, vp]
        L.orc_smooth_graph.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp,
                                       ctypes.c_int64]
        L.orc_smooth_bound.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                       ctypes.c_int32, ctypes.c_double, ctypes.c_int32, vp, vp,
                                       vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Result:
    """Everything the oracle produced for one instance."""

    def __init__(self, handle):
        L = lib()
        self.status = L.orc_status(handle)
        self.error = L.orc_error(handle).decode()
        nv, ne = L.orc_num_nodes(handle), L.orc_num_edges(handle)
        npnt = L.orc_num_points(handle)
        self.n_nodes, self.n_edges = nv, ne
        self.size_per_node = L.orc_size_per_node(handle)
        self.cutoff = np.zeros(npnt, np.float64)
        self.stat = np.zeros(npnt, np.int32)
        if npnt:
            L.orc_get_cutoffs(handle, _ptr(self.cutoff), _ptr(self.stat))
        self.v1 = np.zeros(ne, np.int32)
        self.v2 = np.zeros(ne, np.int32)
        self.lab1 = np.zeros(ne, np.int32)
        self.lab2 = np.zeros(ne, np.int32)
        self.Do = np.zeros(ne, np.float64)
        self.D = np.zeros(ne, np.float64)
        if ne:
            L.orc_get_edges(handle, _ptr(self.v1), _ptr(self.v2), _ptr(self.lab1), _ptr(self.lab2),
                            _ptr(self.Do), _ptr(self.D))
        self.label = np.zeros(nv, np.int32)
        self.fxy = np.zeros(nv, np.int32)
        if nv:
            L.orc_get_nodes(handle, _ptr(self.label), _ptr(self.fxy))
        self.F = None
        self.x = None
        st = Stats()
        L.orc_get_stats(handle, ctypes.byref(st))
        self.stats = st.as_dict()
        self.lp = L.orc_lp_value(handle)
        self.max_rank = L.orc_max_rank(handle)
        if self.stats["checks"] > 0:
            self.F = np.zeros(nv, np.float64)
            L.orc_get_F(handle, _ptr(self.F))
            self.x = np.zeros(ne, np.float64)
            L.orc_get_x(handle, _ptr(self.x))
            nc = L.orc_get_combs(handle, None, None)
            self.comb_size = np.zeros(nc, np.int32)
            L.orc_get_combs(handle, _ptr(self.comb_size), None)
            self.comb_nodes = np.zeros(int(self.comb_size.sum()), np.int32)
            L.orc_get_combs(handle, _ptr(self.comb_size), _ptr(self.comb_nodes))
            self.statA = np.zeros(nv, np.int32)
            self.statB = np.zeros(nv, np.int32)
            L.orc_get_statab(handle, _ptr(self.statA), _ptr(self.statB))

    def edge_set(self):
        """Set of (label_low, label_high) pairs."""
        a = np.minimum(self.lab1, self.lab2)
        b = np.maximum(self.lab1, self.lab2)
        return set(zip(a.tolist(), b.tolist()))


def _run(fn, *args):
    L = lib()
    h = ctypes.c_void_p()
    fn(*args, ctypes.byref(h))
    try:
        return Result(h)
    finally:
        L.orc_free(h)


def solve_file(path, top_k, cost=COST_REF, id_order=ID_REF, knn=KNN_TOPN, write_files=False,
               threads=1):
    return _run(lib().orc_solve_file, path.encode(), top_k, cost, id_order, knn,
                1 if write_files else 0, threads)


def _pts(K, X, Y):
    X = np.ascontiguousarray(X, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    if K is None:
        K = np.arange(1, len(X) + 1, dtype=np.int32)
    K = np.ascontiguousarray(K, np.int32)
    return K, X, Y


def solve_points(X, Y, top_k, K=None, cost=COST_REF, id_order=ID_FXY, knn=KNN_TOPN, threads=1):
    K, X, Y = _pts(K, X, Y)
    return _run(lib().orc_solve_points, _ptr(K), _ptr(X), _ptr(Y), len(X), top_k, cost, id_order,
                knn, threads)


def build_graph(X, Y, top_k, K=None, cost=COST_REF, id_order=ID_FXY, knn=KNN_TOPN):
    K, X, Y = _pts(K, X, Y)
    return _run(lib().orc_build_graph, _ptr(K), _ptr(X), _ptr(Y), len(X), top_k, cost, id_order,
                knn)


def solve_graph(n_nodes, v1, v2, D, Do, label=None, threads=1):
    v1 = np.ascontiguousarray(v1, np.int32)
    v2 = np.ascontiguousarray(v2, np.int32)
    D = np.ascontiguousarray(D, np.float64)
    Do = np.ascontiguousarray(Do, np.float64)
    lab = None if label is None else np.ascontiguousarray(label, np.int32)
    return _run(lib().orc_solve_graph, n_nodes, len(v1), _ptr(v1), _ptr(v2), _ptr(D), _ptr(Do),
                _ptr(lab), threads)


def solve_batch(offs, X, Y, top_k, cost=COST_REF, threads=1):
    offs = np.ascontiguousarray(offs, np.int64)
    X = np.ascontiguousarray(X, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    n = len(offs) - 1
    lp = np.zeros(n, np.float64)
    status = np.zeros(n, np.int32)
    iters = np.zeros(n, np.int64)
    lib().orc_solve_batch(n, _ptr(offs), _ptr(X), _ptr(Y), top_k, cost, threads, _ptr(lp),
                          _ptr(status), _ptr(iters))
    return lp, status, iters


# -- smoothed bound (f2m_smooth_oracle.cpp) ----------------------------------
def smooth_graph(x, y, top_k):
    """(row, nbr, c) of the FP32 kNN union graph of one instance."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n = len(x)
    row = np.zeros(n + 1, np.int64)
    S = lib().orc_smooth_graph(_ptr(x), _ptr(y), n, top_k, _ptr(row), None, None, 0)
    nbr = np.zeros(S, np.int32)
    c = np.zeros(S, np.float32)
    lib().orc_smooth_graph(_ptr(x), _ptr(y), n, top_k, _ptr(row), _ptr(nbr), _ptr(c), S)
    return row, nbr, c


def smooth_bound(x, y, top_k, tau=1e-3, iters=100, omega=0.5, newton_max=60, grad=False,
                 graph_xy=None, c=None):
    """FP64 host bound of one instance; with grad=True returns (L, dLdx, dLdy,
    dLdc).  graph_xy fixes the graph (points it is built from); c replaces the
    edge costs (per slot)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n = len(x)
    gx = gy = None
    if graph_xy is not None:
        gx = np.ascontiguousarray(graph_xy[0], np.float32)
        gy = np.ascontiguousarray(graph_xy[1], np.float32)
    co = None if c is None else np.ascontiguousarray(c, np.float32)
    L = ctypes.c_double()
    dx = dy = dc = None
    if grad:
        S = int(smooth_graph(gx if gx is not None else x, gy if gy is not None else y, top_k)[1].size)
        dx, dy, dc = np.zeros(n), np.zeros(n), np.zeros(S)
    st = lib().orc_smooth_bound(_ptr(x), _ptr(y), n, top_k, tau, iters, omega, newton_max,
                                _ptr(gx), _ptr(gy), _ptr(co), ctypes.byref(L), _ptr(dx), _ptr(dy),
                                _ptr(dc))
    if st != OK:
        raise ValueError(f"orc_smooth_bound status {st}")
    return (L.value, dx, dy, dc) if grad else L.value
