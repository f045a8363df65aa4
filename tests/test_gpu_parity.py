"""CUDA path vs the CPU oracle (parity), through the C ABI.

Node ids, edge order and every FP64 expression follow the reference, so the
device potentials F must equal the oracle's bit for bit, the kNN edge list
must be identical, and the LP value must agree to rounding (the device sums
sum(x*Do) in a different order: tolerance 1e-12 relative, well inside the
1e-9 target)."""
import os

import numpy as np
import pytest

import f2m_b200
from f2m_b200 import synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LP_RTOL = 1e-12


def _close(a, b, rtol=LP_RTOL):
    return abs(a - b) <= rtol * max(abs(a), abs(b))


AXB_XTOL = 1e-6   # x of an Ax=b comb edge solved on the device (rows in another order)
AXB_LP_RTOL = 1e-9


def _check_against(r, ref_status, ref_lp, ref_max_rank, lab1, lab2, Do, F, xval):
    assert r.status == ref_status
    assert np.array_equal(r.lab1, lab1), "kNN edge list differs"
    assert np.array_equal(r.lab2, lab2)
    assert np.array_equal(r.Do, Do)
    assert np.array_equal(r.F, F), "potentials differ from the oracle"
    if ref_status == 0:
        assert r.max_rank == ref_max_rank
        if r.stats["irr_a"] == 0:
            assert np.array_equal(r.x, xval)
            assert _close(r.lp, ref_lp)
        else:
            # irregular combs, whose Ax=b the device may have solved: the
            # solution is the same, its last bits may not be (the reference
            # takes the rows in its hash map's order), so x agrees to FP32
            # rounding of a 1e-8 residual and the LP value to 1e-9
            assert np.all(np.abs(r.x - xval) <= AXB_XTOL)
            assert _close(r.lp, ref_lp, AXB_LP_RTOL)


@pytest.mark.parametrize("name", ["uniform200_n10", "config1_n20", "lattice150_s1_n8",
                                  "lattice150_s3_n8"])
def test_points_match_golden(ctx, name):
    g = np.load(os.path.join(GOLDEN, f"oracle_{name}.npz"))
    r = ctx.solve_points(g["x"], g["y"], int(g["N"]))
    _check_against(r, int(g["status"]), float(g["lp"]), int(g["max_rank"]), g["lab1"], g["lab2"],
                   g["Do"], g["F"], g["xval"])


def test_file_path_matches_golden_reference_order(ctx, tmp_path):
    """`F2M.solver.exe file N`: reference node order, report and solution files."""
    g = np.load(os.path.join(GOLDEN, "oracle_config1_ref_n20.npz"))
    path = str(tmp_path / "c1.tsp")
    synth.write_tsplib(path, g["x"], g["y"])
    r = ctx.solve_file(path, 20, write_files=True)
    _check_against(r, int(g["status"]), float(g["lp"]), int(g["max_rank"]), g["lab1"], g["lab2"],
                   g["Do"], g["F"], g["xval"])
    assert np.array_equal(r.label, g["node_label"])
    rep = open(path + ".top20.F2M_report").read().splitlines()
    assert rep[0] == "Optimal Found: Yes"
    assert rep[1] == "Optimal Value: %.15g" % r.lp
    assert rep[3] == "MAX edge rank: %d" % int(g["max_rank"])
    sol = [ln.split() for ln in open(path + ".top20.F2M_solution")]
    got = {(int(a), int(b)): float(c) for a, b, c in sol}
    want = {(int(a), int(b)): float(c) for a, b, c in zip(g["lab1"], g["lab2"], g["xval"]) if c}
    assert got == want
    assert os.path.exists(path + ".top20.DM")


def test_points_vs_oracle_live(ctx, oracle):
    """Fresh seeds: the oracle is run here next to the device."""
    for seed, n, N in [(21, 120, 6), (22, 777, 12), (23, 2500, 16), (24, 5000, 16)]:
        x, y = synth.uniform_int_points(n, seed)
        o = oracle.solve_points(x, y, N)
        r = ctx.solve_points(x, y, N)
        _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)


def test_lattice_repair_vs_oracle(ctx, oracle):
    """Many equal distances: tie order of the kNN and the comb repair loop."""
    for seed in (2, 4, 7, 11):
        x, y = synth.lattice_points(300, seed)
        o = oracle.solve_points(x, y, 8)
        r = ctx.solve_points(x, y, 8)
        _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)
        assert r.stats["repair_steps"] == o.stats["repair_steps"]


def test_duplicates_and_rounding(ctx, oracle):
    """get_KXY drops repeated points after 1e-3 rounding (FXY.hpp:252-267)."""
    x, y = synth.uniform_int_points(400, 31)
    x = np.concatenate([x, x[:40] + 0.0004])
    y = np.concatenate([y, y[:40]])
    frac = synth.uniform(31, 9, len(x)) * 0.01
    x = x + frac
    o = oracle.solve_points(x, y, 10)
    r = ctx.solve_points(x, y, 10)
    assert r.n_nodes == o.n_nodes < len(x)
    _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)


def _batch_lp_close(lp, lp_o, st_o, n_irr):
    """LP values of solved instances: to rounding (1e-12) where every comb is
    regular, to 1e-9 where an irregular comb's Ax=b ran (see _check_against)."""
    ok = st_o == 0
    tol = np.where(n_irr > 0, AXB_LP_RTOL, LP_RTOL)
    assert np.all(np.abs(lp[ok] - lp_o[ok]) <= tol[ok] * np.abs(lp_o[ok]))


def test_batch_matches_oracle(ctx, oracle):
    offs, x, y = synth.config3(seed=5, n_inst=40, hi=1500)
    # two lattice instances go through the host comb stage
    lx, ly = synth.lattice_points(150, 1)
    lx2, ly2 = synth.lattice_points(150, 3)
    x = np.concatenate([x, lx, lx2])
    y = np.concatenate([y, ly, ly2])
    offs = np.concatenate([offs, [offs[-1] + 150, offs[-1] + 300]])
    out = ctx.solve_batch(offs, x, y, 16, details=True)
    lp_o, st_o, _ = oracle.solve_batch(offs, x, y, 16, threads=os.cpu_count() or 1)
    assert np.array_equal(out["status"], st_o)
    _batch_lp_close(out["lp"], lp_o, st_o, out["n_irregular"])


def test_batch_equals_plain_path(ctx):
    """Batched LP values equal the per-instance (plain) path."""
    offs, x, y = synth.config3(seed=6, n_inst=16, hi=900)
    lp, st = ctx.solve_batch(offs, x, y, 16)
    for b in range(16):
        r = ctx.solve_points(x[offs[b]:offs[b + 1]], y[offs[b]:offs[b + 1]], 16)
        assert r.status == st[b]
        assert _close(r.lp, lp[b])


def test_primal_is_feasible_and_gap_closed(ctx):
    x, y = synth.config1(8)
    r = ctx.solve_points(x, y, 20)
    assert r.status == 0
    deg = np.zeros(r.n_nodes)
    np.add.at(deg, r.v1, r.x)
    np.add.at(deg, r.v2, r.x)
    assert np.allclose(deg, 2.0)
    assert set(np.unique(r.x)).issubset({0.0, 0.5, 1.0})
    assert r.stats["degree_violations"] == 0
    assert abs(r.stats["dual_value"] - r.lp) <= 1e-9 * r.lp
    assert r.stats["max_grad"] < 1e-7


def test_input_errors(ctx):
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_points(np.array([0.0, 1, 2]), np.array([0.0, 1, 5]), 3)
    assert e.value.status == f2m_b200.ERR_INPUT
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_points(*synth.uniform_int_points(50, 1), 2)
    assert e.value.status == f2m_b200.ERR_INPUT
    with pytest.raises(f2m_b200.F2MError):
        ctx.solve_file("/nonexistent/file.tsp", 10)


def test_zero_x_span_is_solved(ctx, oracle):
    """A vertical line of points: the reference's ring radius is 0 and its
    stat pass never ends (FXY.hpp:305,528); here the y-span takes over."""
    y = np.arange(60, dtype=np.float64) * 3.0 + synth.uniform(3, 1, 60).round(3)
    x = np.zeros(60)
    o = oracle.solve_points(x, y, 6)
    r = ctx.solve_points(x, y, 6)
    _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)


# --- the grid-wide solver (single instances above 10,000 points, or forced) ---

def test_grid_solver_forced_matches_oracle(ctx, oracle):
    x, y = synth.uniform_int_points(3000, 41)
    o = oracle.solve_points(x, y, 16)
    r = ctx.solve_points(x, y, 16, params=f2m_b200.default_params(solver=2))
    _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)


def test_grid_solver_repair_matches_oracle(ctx, oracle):
    """The repair loop's device refits on the grid-wide solver."""
    for seed in (1, 2):
        x, y = synth.lattice_points(300, seed)
        o = oracle.solve_points(x, y, 8)
        r = ctx.solve_points(x, y, 8, params=f2m_b200.default_params(solver=2))
        _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)
        assert r.stats["repair_steps"] == o.stats["repair_steps"] > 0


def test_grid_solver_file_and_graph_paths(ctx, tmp_path):
    """The grid-wide solver orders its nodes by their points: on the file path
    (nodes in the reference's order, mapped to file points) and on the graph
    path (no coordinates, the caller's order) it must give the per-team
    solver's potentials bit for bit."""
    x, y = synth.uniform_int_points(4000, 43)
    path = str(tmp_path / "g4000.tsp")
    synth.write_tsplib(path, x, y)
    team = ctx.solve_file(path, 14)
    grid = ctx.solve_file(path, 14, params=f2m_b200.default_params(solver=2))
    assert team.status == grid.status == 0
    assert np.array_equal(team.F, grid.F)
    assert _close(team.lp, grid.lp) and team.max_rank == grid.max_rank
    g = ctx.knn(x, y, 14)
    gt = ctx.solve_graph(len(g.F), g.v1, g.v2, g.D, g.Do)
    gg = ctx.solve_graph(len(g.F), g.v1, g.v2, g.D, g.Do, params=f2m_b200.default_params(solver=2))
    assert gt.status == gg.status == 0
    assert np.array_equal(gt.F, gg.F)


def test_large_instance_uses_grid_solver(ctx, oracle):
    """20,000 clustered points (the large-instance shape at 1/5 size)."""
    x, y = synth.config2(2, n=20000)
    o = oracle.solve_points(x, y, 16, threads=os.cpu_count() or 1)
    r = ctx.solve_points(x, y, 16)
    _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)


def test_config2_100k_n50(ctx, oracle):
    """100,000 points, 64 Gaussian clusters + 10% background, N=50."""
    x, y = synth.config2(2)
    o = oracle.solve_points(x, y, 50, threads=os.cpu_count() or 1)
    r = ctx.solve_points(x, y, 50)
    _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)
    assert abs(r.stats["dual_value"] - r.lp) <= 1e-9 * r.lp


def test_knn_only_matches_oracle_graph(ctx, oracle):
    """f2m_knn: the graph stage alone, edge for edge."""
    x, y = synth.uniform_int_points(1500, 77)
    o = oracle.build_graph(x, y, 14)
    r = ctx.knn(x, y, 14)
    assert r.status == 0 and np.isnan(r.lp)
    assert np.array_equal(r.lab1, o.lab1) and np.array_equal(r.lab2, o.lab2)
    assert np.array_equal(r.Do, o.Do) and np.array_equal(r.D, o.D)


# --- TSPLIB EUC_2D costs: nint(distance) as the edge cost --------------------

def test_nint_cost_mode_matches_oracle(ctx, oracle):
    """Integer costs tie often: the nint key order and the widened candidate
    search (ties with the N-th cost out to cost + 0.5)."""
    p = f2m_b200.default_params(cost_mode=1)
    for seed, n, N in [(51, 1000, 20), (52, 400, 8), (53, 2500, 16)]:
        x, y = synth.uniform_int_points(n, seed)
        o = oracle.solve_points(x, y, N, cost=oracle.COST_NINT)
        r = ctx.solve_points(x, y, N, params=p)
        _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)
    x, y = synth.lattice_points(300, 5)
    o = oracle.solve_points(x, y, 8, cost=oracle.COST_NINT)
    r = ctx.solve_points(x, y, 8, params=p)
    _check_against(r, o.status, o.lp, o.max_rank, o.lab1, o.lab2, o.Do, o.F, o.x)


def test_nint_batch_matches_oracle(ctx, oracle):
    offs, x, y = synth.config3(seed=8, n_inst=30, hi=1200)
    p = f2m_b200.default_params(cost_mode=1)
    out = ctx.solve_batch(offs, x, y, 16, params=p, details=True)
    lp_o, st_o, _ = oracle.solve_batch(offs, x, y, 16, cost=oracle.COST_NINT,
                                       threads=os.cpu_count() or 1)
    assert np.array_equal(out["status"], st_o)
    _batch_lp_close(out["lp"], lp_o, st_o, out["n_irregular"])


def test_class_bounds_change_speed_not_results(ctx):
    """The size classes only decide which team size runs an instance."""
    offs, x, y = synth.config3(seed=12, n_inst=24, hi=2500)
    start = f2m_b200.get_class_bounds()
    lp0, st0 = ctx.solve_batch(offs, x, y, 16)
    try:
        f2m_b200.set_class_bounds([100, 200, 300])
        lp1, st1 = ctx.solve_batch(offs, x, y, 16)
        with pytest.raises(f2m_b200.F2MError):
            f2m_b200.set_class_bounds([500, 400, 900])
    finally:
        f2m_b200.set_class_bounds(start)
    # the potentials are the same bits; the LP value is a team-wide sum whose
    # order follows the team size
    assert np.array_equal(st0, st1)
    assert np.all(np.abs(lp0 - lp1) <= LP_RTOL * np.abs(lp0))


def test_batch_edge_cases_match_oracle(ctx, oracle):
    """Ragged batch: instances of 4-12 points (N clamped to V-1), repeated and
    collinear points, one all-identical instance (an input error), and one
    instance of 10,000 points (the largest the batched solver takes)."""
    parts = []
    for n in (4, 5, 6, 8, 12):
        parts.append(synth.uniform_int_points(n, 100 + n))
    parts.append((np.array([0, 0, 0, 1, 1, 2, 2, 3, 5, 8], float),
                  np.array([0, 0, 0, 1, 1, 2, 2, 3, 5, 8], float)))
    x, y = synth.uniform_int_points(30, 7)
    parts.append((np.concatenate([x, x]), np.concatenate([y, y])))
    parts.append((np.zeros(10), np.zeros(10)))
    parts.append(synth.uniform_int_points(10000, 99))
    offs = np.concatenate([[0], np.cumsum([len(p[0]) for p in parts])]).astype(np.int64)
    X = np.concatenate([p[0] for p in parts])
    Y = np.concatenate([p[1] for p in parts])
    out = ctx.solve_batch(offs, X, Y, 16, details=True)
    st = out["status"]
    lp_o, st_o, _ = oracle.solve_batch(offs, X, Y, 16, threads=os.cpu_count() or 1)
    assert np.array_equal(st, st_o)
    assert st[7] == f2m_b200.ERR_INPUT
    assert (st_o == 0).sum() == len(parts) - 1
    _batch_lp_close(out["lp"], lp_o, st_o, out["n_irregular"])


def test_batch_argument_errors(ctx):
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_batch(np.array([0], np.int64), np.zeros(0), np.zeros(0), 16)
    assert e.value.status == f2m_b200.ERR_INPUT
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_batch(np.array([0, 50], np.int64), *synth.uniform_int_points(50, 1), 300)
    assert e.value.status == f2m_b200.ERR_CAPACITY
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_batch(np.array([0, 60, 40], np.int64), *synth.uniform_int_points(60, 1), 8)
    assert e.value.status == f2m_b200.ERR_INPUT


def test_solve_graph_matches_oracle(ctx, oracle):
    """graph_c + RUN on a caller-built graph (here the oracle's kNN graph),
    including a lattice graph that needs the repair loop."""
    cases = [(synth.uniform_int_points(900, 61), 12), (synth.lattice_points(300, 2), 8)]
    for (x, y), N in cases:
        g = oracle.build_graph(x, y, N)
        o = oracle.solve_graph(g.n_nodes, g.v1, g.v2, g.D, g.Do, label=g.label)
        r = ctx.solve_graph(g.n_nodes, g.v1, g.v2, g.D, g.Do, labels=g.label)
        assert r.status == o.status
        assert np.array_equal(r.F, o.F), "potentials differ from the oracle"
        if o.status == 0:
            assert _close(r.lp, o.lp)
            assert r.max_rank == o.max_rank
            assert np.array_equal(r.x, o.x)
        p = ctx.solve_points(x, y, N)  # the same graph through the points path
        assert np.array_equal(p.F, r.F)


# --- failures made on the host: caps, bad files, zero-length edges ----------

def test_iteration_cap_reports_not_converged(ctx, oracle):
    x, y = synth.uniform_int_points(400, 3)
    p = f2m_b200.default_params(max_iters=50)
    r = ctx.solve_points(x, y, 10, params=p)  # raises only for hard errors
    assert r.status == f2m_b200.ERR_NOT_CONVERGED
    lp, st = ctx.solve_batch(np.array([0, 400]), x, y, 10, params=p)
    assert st[0] == f2m_b200.ERR_NOT_CONVERGED and np.isnan(lp[0])


def test_malformed_files_are_input_errors(ctx, tmp_path):
    bad = tmp_path / "bad.tsp"
    bad.write_text("NAME : bad\nNODE_COORD_SECTION\n1 0 0\n2 x 7\nEOF\n")
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_file(str(bad), 5)
    assert e.value.status == f2m_b200.ERR_INPUT
    empty = tmp_path / "empty.tsp"
    empty.write_text("NAME : empty\nNODE_COORD_SECTION\nEOF\n")
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_file(str(empty), 5)
    assert e.value.status == f2m_b200.ERR_INPUT


def test_zero_length_nint_edge_is_an_input_error(ctx, oracle):
    """Two points 0.3 apart (distinct after the 1e-3 rounding) have nint cost 0."""
    x, y = synth.uniform_int_points(60, 12)
    x = np.concatenate([x, [x[0] + 0.3]])
    y = np.concatenate([y, [y[0]]])
    p = f2m_b200.default_params(cost_mode=1)
    o = oracle.solve_points(x, y, 6, cost=oracle.COST_NINT)
    assert o.status == oracle.ERR_INPUT
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_points(x, y, 6, params=p)
    assert e.value.status == f2m_b200.ERR_INPUT


def test_resume_from_stored_potentials(ctx):
    """Checkpoint/resume: the potentials of a result restart the descent; from
    the optimum the same LP comes back in far fewer iterations."""
    for (x, y), N in [(synth.uniform_int_points(1200, 81), 12), (synth.config2(3, n=15000), 16)]:
        r1 = ctx.solve_points(x, y, N)
        r2 = ctx.solve_points_from(x, y, N, r1.F)
        assert r1.status == r2.status == 0
        assert _close(r1.lp, r2.lp)
        assert r2.stats["iterations"] < r1.stats["iterations"] / 2
        with pytest.raises(f2m_b200.F2MError) as e:
            ctx.solve_points_from(x, y, N, r1.F[:-1])
        assert e.value.status == f2m_b200.ERR_INPUT


def test_grid_block_depths_give_identical_potentials(tmp_path):
    """Halo blocks recompute the nodes within k EF hops of each CTA's own
    nodes so that one grid barrier covers k Jacobi steps: the potentials must
    not depend on k (0 = one grid barrier per step).  Depth 0 also launches
    without halo storage (no shared scratch), so its partitions take the
    thread-per-node global-memory path; depths 2 and 8 take the warp path in
    shared memory.  The depth is read once per process, so each depth runs in
    a child process."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import f2m_b200; from f2m_b200 import synth; "
            "x, y = synth.config2(5, n=20000); r = f2m_b200.Context(0).solve_points(x, y, 16, "
            "params=f2m_b200.default_params(solver=2)); np.savez(sys.argv[1], F=r.F, x=r.x, lp=r.lp, "
            "it=r.stats['iterations'])" % root)
    out = {}
    for k in (0, 2, 8):
        f = str(tmp_path / f"k{k}.npz")
        env = dict(os.environ, F2M_GRID_BLOCK=str(k))
        subprocess.run([sys.executable, "-c", code, f], env=env, check=True, timeout=600)
        out[k] = np.load(f)
    for k in (2, 8):
        assert np.array_equal(out[k]["F"], out[0]["F"]), f"depth {k} changed the potentials"
        assert np.array_equal(out[k]["x"], out[0]["x"])
        assert int(out[k]["it"]) == int(out[0]["it"])
        assert _close(float(out[k]["lp"]), float(out[0]["lp"]))


def test_grid_l1_reserve_gives_identical_potentials(tmp_path):
    """The whole-GPU solver leaves part of the shared-memory carve-out to L1
    (F2M_GRID_L1_KB), which changes how many halo entries fit and so the
    block depth of each phase and whether the partitions run in shared
    memory -- never the potentials, the primal or the iteration count (at
    160 KB the halo no longer fits and every step meets a grid barrier).
    The reserve is read once per process, so each setting runs in a child
    process."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import f2m_b200; from f2m_b200 import synth; "
            "x, y = synth.config2(5, n=20000); r = f2m_b200.Context(0).solve_points(x, y, 16, "
            "params=f2m_b200.default_params(solver=2)); np.savez(sys.argv[1], F=r.F, x=r.x, lp=r.lp, "
            "it=r.stats['iterations'])" % root)
    out = {}
    for kb in (0, 64, 160):
        f = str(tmp_path / f"kb{kb}.npz")
        env = dict(os.environ, F2M_GRID_L1_KB=str(kb))
        subprocess.run([sys.executable, "-c", code, f], env=env, check=True, timeout=600)
        out[kb] = np.load(f)
    for kb in (64, 160):
        assert np.array_equal(out[kb]["F"], out[0]["F"]), f"L1 reserve {kb} KB changed the potentials"
        assert np.array_equal(out[kb]["x"], out[0]["x"])
        assert int(out[kb]["it"]) == int(out[0]["it"])
        assert _close(float(out[kb]["lp"]), float(out[0]["lp"]))


def test_repeated_calls_are_bit_identical(ctx):
    """Replays: every reduction here has a fixed order (team sums, the grid
    solver's per-CTA partials read in CTA order), so the same call gives the
    same bits, LP values included -- the check that stands in for a race
    detector on this GPU."""
    offs, x, y = synth.config3(seed=9, n_inst=96, hi=3000)
    a = ctx.solve_batch(offs, x, y, 16, details=True)
    b = ctx.solve_batch(offs, x, y, 16, details=True)
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]), equal_nan=True), k
    gx, gy = synth.config2(6, n=20000)
    r1 = ctx.solve_points(gx, gy, 16)
    r2 = ctx.solve_points(gx, gy, 16)
    assert np.array_equal(r1.F, r2.F) and np.array_equal(r1.x, r2.x)
    assert r1.lp == r2.lp and r1.stats == r2.stats


def test_grid_barrier_wait_runs_out_and_the_context_recovers(ctx):
    """The whole-GPU solver's grid barrier is a bounded wait.  With a limit of
    one poll the first CTA to arrive gives up (nothing releases the barrier
    that early), raises the error flag, every CTA leaves the solve and the
    call fails with F2M_ERR_CUDA -- no fault, no trap.  The same context then
    solves the instance normally, bit for bit as a fresh context does."""
    import f2m_b200
    x, y = synth.config2(7, n=12000)
    short = f2m_b200.default_params(solver=2, grid_spin_limit=1)
    with pytest.raises(f2m_b200.F2MError) as e:
        ctx.solve_points(x, y, 16, params=short)
    assert e.value.status == f2m_b200.ERR_CUDA
    assert "barrier" in ctx.last_error()
    r = ctx.solve_points(x, y, 16, params=f2m_b200.default_params(solver=2))
    fresh = f2m_b200.Context(0)
    try:
        r2 = fresh.solve_points(x, y, 16, params=f2m_b200.default_params(solver=2))
    finally:
        fresh.close()
    assert r.status == 0 and np.array_equal(r.F, r2.F) and r.lp == r2.lp


def test_warp_partition_equals_the_serial_loop(ctx):
    """The whole-GPU solver partitions a node's list with a whole warp
    (qpart_ptr_EF, graph_cuda_partition.hpp:27-54, restated as a fixed
    pairing of swaps ranked by ballots).  On the device, 200,000 seeded lists
    (0-128 entries, ties, thresholds that need the raise-by-one loop, NaN)
    must come out in the serial loop's order with its count."""
    assert ctx.partition_selfcheck(200000, 7) == 0
    assert ctx.partition_selfcheck(200000, 8) == 0
