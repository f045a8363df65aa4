"""Generate the golden fixtures under tests/golden/.

1. reference_reports.json: the known answers shipped with the reference
   (examples/vsli/*.F2M_report and report_dir.txt), read from a local copy of
   the reference repository (argument 1; default $F2M_REFERENCE, else a sibling
   checkout named "reference" next to this repository).
2. oracle_*.npz: outputs of the CPU oracle (oracle/) on small seeded
   synthetic instances; the oracle is pinned to (1) by tests/test_oracle.py.

Run from the repository root:  python tests/golden/make_golden.py [reference_dir]
"""
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from f2m_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def reports(ref):
    out = []
    for name in sorted(os.listdir(os.path.join(ref, "examples", "vsli"))):
        m = re.match(r"(.+\.tsp)\.top(\d+)\.F2M_report$", name)
        if not m:
            continue
        txt = open(os.path.join(ref, "examples", "vsli", name)).read()
        out.append({
            "file": "examples/vsli/" + m.group(1),
            "N": int(m.group(2)),
            "lp": float(re.search(r"Optimal Value: (\S+)", txt).group(1)),
            "lp_text": re.search(r"Optimal Value: (\S+)", txt).group(1),
            "max_rank": int(re.search(r"MAX edge rank: (\d+)", txt).group(1)),
            "time_s": float(re.search(r"Time: (\S+)", txt).group(1)),
        })
    for line in open(os.path.join(ref, "report_dir.txt")):
        m = re.match(r"(\S+) Time: (\S+) Optimal Value: (\S+)", line.strip())
        if m:
            out.append({"file": "examples/art/" + m.group(1) + ".tsp", "N": None,
                        "lp": float(m.group(3)), "lp_text": m.group(3), "max_rank": None,
                        "time_s": float(m.group(2))})
    return out


CASES = {
    # name: (points generator, N, id order)
    "uniform200_n10": (lambda: synth.uniform_int_points(200, 11), 10, O.ID_FXY),
    "config1_n20": (lambda: synth.config1(1), 20, O.ID_FXY),
    "lattice150_s1_n8": (lambda: synth.lattice_points(150, 1), 8, O.ID_FXY),
    "lattice150_s3_n8": (lambda: synth.lattice_points(150, 3), 8, O.ID_FXY),
    "config1_ref_n20": (lambda: synth.config1(5), 20, O.ID_REF),
}


def save_case(name, gen, N, id_order):
    x, y = gen()
    r = O.solve_points(x, y, N, id_order=id_order, knn=O.KNN_LITERAL)
    np.savez_compressed(
        os.path.join(HERE, f"oracle_{name}.npz"),
        x=x, y=y, N=N, id_order=id_order, status=r.status, lp=r.lp, max_rank=r.max_rank,
        lab1=r.lab1, lab2=r.lab2, Do=r.Do, D=r.D, node_label=r.label, F=r.F, xval=r.x,
        n_combs=r.stats["n_combs"], irr_a=r.stats["irr_a"], repair_steps=r.stats["repair_steps"],
        iterations=r.stats["iters_glob"] + r.stats["iters_ef"] + r.stats["iters_repair"],
        cutoff=r.cutoff, stat=r.stat)
    print(name, "status", r.status, "V", r.n_nodes, "E", r.n_edges, "lp %.15g" % r.lp,
          "repair", r.stats["repair_steps"])


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    default = os.environ.get("F2M_REFERENCE") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(here))), "reference")
    ref = sys.argv[1] if len(sys.argv) > 1 else default
    if os.path.isdir(ref):
        with open(os.path.join(HERE, "reference_reports.json"), "w") as f:
            json.dump(reports(ref), f, indent=1)
    for name, (gen, N, idord) in CASES.items():
        save_case(name, gen, N, idord)


if __name__ == "__main__":
    main()
