"""Parity against the reference program itself.

tests/golden/reference_runs.npz holds the outputs of the reference (built from
its own sources by oracle/ref.mk and run on a B200 by
tests/golden/make_reference_runs.py) on seeded uniform inputs: the report's
LP text and MAX rank, the solution lines, and the SHA-256 of its .F2M_solution,
.DM and _duplicates files.  The inputs are rebuilt here from their seeds.

* the CPU oracle must print the same LP text and MAX rank and write a
  byte-identical solution file;
* the CUDA path (`f2m_solve_file`, the `F2M.solver.exe file N` drop-in) must
  write byte-identical solution, .DM and _duplicates files and the same report
  lines (the Time line aside).
"""
import hashlib
import os
import re
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_reference_runs as MR  # noqa: E402

FIX = os.path.join(HERE, "golden", "reference_runs.npz")
pytestmark = pytest.mark.skipif(not os.path.exists(FIX), reason="no reference runs recorded")


def _fixture():
    return np.load(FIX)


def _cases():
    if not os.path.exists(FIX):
        return []
    return [str(c) for c in _fixture()["cases"]]


def _sha(path):
    if not os.path.exists(path):
        return ""
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def _report(path):
    txt = open(path).read()
    m = re.search(r"Optimal Value: (\S+)", txt)
    r = re.search(r"MAX edge rank: (\d+)", txt)
    return (m.group(1) if m else None), (int(r.group(1)) if r else None)


@pytest.mark.parametrize("name", _cases())
def test_oracle_matches_reference_program(name, tmp_path):
    from oracle import oracle as O
    g = _fixture()
    N = MR.CASES[name][2]
    path = MR.write_input(name, str(tmp_path))
    o = O.solve_file(path, N, id_order=O.ID_REF, write_files=True)
    assert o.status == O.OK
    lp_text, rank = _report(f"{path}.top{N}.F2M_report")
    assert lp_text == str(g[name + "/lp_text"])
    assert rank == int(g[name + "/max_rank"])
    assert _sha(f"{path}.top{N}.F2M_solution") == str(g[name + "/sha_solution"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", _cases())
def test_cuda_path_matches_reference_program(ctx, name, tmp_path):
    g = _fixture()
    N = MR.CASES[name][2]
    path = MR.write_input(name, str(tmp_path))
    r = ctx.solve_file(path, N, write_files=True)
    assert r.status == 0
    base = f"{path}.top{N}"
    lp_text, rank = _report(base + ".F2M_report")
    assert lp_text == str(g[name + "/lp_text"])
    assert rank == int(g[name + "/max_rank"])
    pairs = g[name + "/pairs"]
    got = {(int(a), int(b)) for a, b in zip(np.minimum(r.lab1, r.lab2), np.maximum(r.lab1, r.lab2))}
    want = {(int(a), int(b)) for a, b in pairs}
    assert want <= got, "a solution edge of the reference is missing from the kNN graph"
    assert _sha(base + ".F2M_solution") == str(g[name + "/sha_solution"])
    assert _sha(base + ".DM") == str(g[name + "/sha_dm"])
    assert _sha(path + "_duplicates") == str(g[name + "/sha_duplicates"])


CLI = os.path.join(os.path.dirname(HERE), "f2m_b200", "bin", "F2M.solver.exe")


@pytest.mark.gpu
@pytest.mark.parametrize("name", _cases()[:4])
def test_cli_binary_matches_reference_program(name, tmp_path):
    """The drop-in binary itself (`F2M.solver.exe file N`, RUN.cpp:12-31) run
    as a subprocess: the files it writes next to the input are byte-identical
    to the reference program's and its report lines equal the reference's."""
    import subprocess
    assert os.path.exists(CLI), "F2M.solver.exe is not built (f2m_b200/build.py)"
    g = _fixture()
    N = MR.CASES[name][2]
    path = MR.write_input(name, str(tmp_path))
    r = subprocess.run([CLI, path, str(N)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Optimal Found: Yes" in r.stdout
    base = f"{path}.top{N}"
    lp_text, rank = _report(base + ".F2M_report")
    assert lp_text == str(g[name + "/lp_text"])
    assert rank == int(g[name + "/max_rank"])
    assert f"Optimal Value: {lp_text}" in r.stdout
    assert _sha(base + ".F2M_solution") == str(g[name + "/sha_solution"])
    assert _sha(base + ".DM") == str(g[name + "/sha_dm"])
    assert _sha(path + "_duplicates") == str(g[name + "/sha_duplicates"])
