"""The CUDA path on the reference's own published instances, 10^5 to 2.4 x 10^5
points, against the values the reference reports for them.

* examples/vsli/ara238025.tsp.top20.F2M_report:2 -- 563655.760603988 (N = 20)
* examples/vsli/ara238025.tsp.top50.F2M_report:2 -- 563655.760603754 (N = 50)
* examples/vsli/sra104815.tsp.top50.F2M_report:2 -- 246329.098557781 (N = 50)
  (with the reports' MAX edge rank, 18 / 18 / 25)
* report_dir.txt:1-4,6 -- five TSP-art instances; the report does not record
  N, the values are reproduced with N = 50 (the oracle matches them within
  7e-15 relative, tests/test_oracle.py)

The instances are read from gzip copies in tests/golden/_instances, staged from
a reference checkout by tests/golden/stage_instances.py (run by build()); the
tests skip where they were not staged.  Each goes through f2m_solve_file, the
drop-in for `F2M.solver.exe file N`.
"""
import gzip
import json
import os
import shutil

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
INST = os.path.join(HERE, "golden", "_instances")
REPORTS = json.load(open(os.path.join(HERE, "golden", "reference_reports.json")))

pytestmark = pytest.mark.gpu


def _instance(rel, tmp_path):
    src = os.path.join(INST, os.path.basename(rel) + ".gz")
    if not os.path.exists(src):
        pytest.skip(f"{os.path.basename(rel)} not staged (tests/golden/stage_instances.py)")
    dst = tmp_path / os.path.basename(rel)
    with gzip.open(src, "rb") as f, open(dst, "wb") as g:
        shutil.copyfileobj(f, g)
    return str(dst)


VSLI = [(r["file"], r["N"], r["lp_text"], r["max_rank"]) for r in REPORTS if r["N"] is not None]
ART = [(r["file"], r["lp"]) for r in REPORTS if r["N"] is None and "earring" not in r["file"]]


@pytest.mark.parametrize("rel,N,lp_text,rank", VSLI, ids=[f"{os.path.basename(f)}-N{n}" for f, n, _, _ in VSLI])
def test_vlsi_report_digits(ctx, tmp_path, rel, N, lp_text, rank):
    path = _instance(rel, tmp_path)
    r = ctx.solve_file(path, N)
    assert r.status == 0
    assert "%.15g" % r.lp == lp_text
    assert r.max_rank == rank


@pytest.mark.parametrize("rel,lp", ART, ids=[os.path.basename(f) for f, _ in ART])
def test_art_report_values(ctx, tmp_path, rel, lp):
    path = _instance(rel, tmp_path)
    r = ctx.solve_file(path, 50)
    assert r.status == 0
    assert abs(r.lp - lp) <= 1e-9 * abs(lp), (r.lp, lp)
