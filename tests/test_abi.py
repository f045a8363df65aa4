"""The C-ABI library loads and exports every entry point include/f2m.h
declares; argument checks and the no-device path need no GPU."""
import ctypes
import os
import re

import pytest

import f2m_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "f2m.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(f2m_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(f2m_b200.LIB_PATH)
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert sorted(f2m_b200.EXPORTS) == names


def test_default_params_are_the_reference_constants():
    p = f2m_b200.default_params()
    assert p.error_B == 1e-7 and p.error_B_comb == 1e2          # graph_cuda.cu:56-57
    assert (p.glob_K, p.glob_rounds, p.glob_inner, p.glob_tol) == (5, 200, 50, 0.01)
    assert (p.factor0, p.factor_step, p.factor_cap, p.max_rounds) == (100, 300, 5000, 10000)
    assert (p.fix_rounds, p.fix_factor, p.frozen_iters) == (100, 500, 20)
    assert (p.ef_thr, p.ef_small_deg, p.ef_min, p.comb_thr) == (1.0, 10, 3, 0.25)
    assert (p.shift0, p.shift_max) == (0.5, 32)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(f2m_b200.F2MError) as e:
        f2m_b200.Context(0)
    assert e.value.status == f2m_b200.ERR_NO_DEVICE


def test_cli_usage_without_arguments():
    import subprocess
    exe = os.path.join(ROOT, "f2m_b200", "bin", "F2M.solver.exe")
    if not os.path.exists(exe):
        pytest.skip("CLI not built")
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and "usage" in out.stdout


def test_noalloc_array_holds_its_documented_maximum():
    """The no-alloc entry point's fixed array must hold its largest documented
    instance (2,048 points, N = 24): the size check comes before any device
    call, so without a GPU that size gets past it (and fails only on the
    device), while one point or one neighbour more is a capacity error."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (the GPU suite runs these sizes for real)")
    assert f2m_b200.solve_points_noalloc(8, 8, 2048, 24, 8, 8) not in (f2m_b200.OK,
                                                                        f2m_b200.ERR_CAPACITY)
    assert f2m_b200.solve_points_noalloc(8, 8, 2049, 24, 8, 8) == f2m_b200.ERR_CAPACITY
    assert f2m_b200.solve_points_noalloc(8, 8, 2048, 25, 8, 8) == f2m_b200.ERR_CAPACITY
