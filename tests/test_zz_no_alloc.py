"""The allocation-free entry point against the regular one.

f2m_solve_points_noalloc serves callers that cannot allocate device memory
while they run (a host application that owns the GPU through its own pool, or
a latency-bound loop that cannot wait for cudaMalloc).  It takes its scratch
from a fixed device array.  This test calls it through the C ABI twice in a
row -- the array keeps the first call's contents -- and checks both results
against f2m_solve_batch_device on the same inputs.  The file is named to be
collected last.
"""
import numpy as np
import pytest

import f2m_b200
from f2m_b200 import synth

pytestmark = pytest.mark.gpu
LP_RTOL = 1e-12


def _regular(ctx, torch, x, y, top_k):
    dev = torch.device("cuda", 0)
    offs = np.array([0, len(x)], np.int64)
    d_offs = torch.from_numpy(offs).to(dev)
    d_x = torch.from_numpy(x).to(dev)
    d_y = torch.from_numpy(y).to(dev)
    d_lp = torch.empty(1, dtype=torch.float64, device=dev)
    d_st = torch.empty(1, dtype=torch.int32, device=dev)
    ctx.solve_batch_device(offs, d_offs.data_ptr(), d_x.data_ptr(), d_y.data_ptr(), top_k,
                           d_lp.data_ptr(), d_st.data_ptr())
    ctx.sync()
    return float(d_lp.item()), int(d_st.item())


def test_noalloc_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    ctx = f2m_b200.Context(0)
    # the largest size the array takes (2,048 points, N = 24) included
    cases = [(synth.uniform_int_points(1800, 71), 16), (synth.uniform_int_points(600, 72), 20),
             (synth.uniform_int_points(2048, 73), 24)]
    stream = torch.cuda.Stream(device=dev)
    for (x, y), top_k in cases:
        d_x = torch.from_numpy(x).to(dev)
        d_y = torch.from_numpy(y).to(dev)
        d_lp = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
        d_st = torch.full((1,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        s = f2m_b200.solve_points_noalloc(d_x.data_ptr(), d_y.data_ptr(), len(x), top_k,
                                          d_lp.data_ptr(), d_st.data_ptr(), stream.cuda_stream)
        assert s == f2m_b200.OK
        stream.synchronize()
        lp, st = float(d_lp.item()), int(d_st.item())
        lp_ref, st_ref = _regular(ctx, torch, x, y, top_k)
        assert st == st_ref == f2m_b200.OK
        assert abs(lp - lp_ref) <= LP_RTOL * abs(lp_ref)
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    s = f2m_b200.solve_points_noalloc(1, 1, 2049, 16, 1, 1)
    assert s == f2m_b200.ERR_CAPACITY
    s = f2m_b200.solve_points_noalloc(1, 1, 100, 25, 1, 1)
    assert s == f2m_b200.ERR_CAPACITY


def test_noalloc_reports_instances_that_need_the_host_stage():
    """The entry point runs the device stages only: a lattice instance whose
    combs need the host Ax=b stage comes back as F2M_ERR_CAPACITY with a NaN
    LP value, while the regular entry point completes it on the host."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x, y = synth.lattice_points(150, 1)
    d_x = torch.from_numpy(x).to(dev)
    d_y = torch.from_numpy(y).to(dev)
    d_lp = torch.zeros(1, dtype=torch.float64, device=dev)
    d_st = torch.full((1,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    s = f2m_b200.solve_points_noalloc(d_x.data_ptr(), d_y.data_ptr(), len(x), 8,
                                      d_lp.data_ptr(), d_st.data_ptr(), 0)
    assert s == f2m_b200.OK
    torch.cuda.synchronize()
    assert int(d_st.item()) == f2m_b200.ERR_CAPACITY
    assert np.isnan(float(d_lp.item()))
    ctx = f2m_b200.Context(0)
    lp_ref, st_ref = _regular(ctx, torch, x, y, 8)
    ctx.close()
    assert st_ref == f2m_b200.OK and np.isfinite(lp_ref)


def test_noalloc_rejects_the_whole_gpu_solver():
    p = f2m_b200.default_params(solver=2)
    assert f2m_b200.solve_points_noalloc(1, 1, 100, 16, 1, 1, params=p) == f2m_b200.ERR_INPUT
