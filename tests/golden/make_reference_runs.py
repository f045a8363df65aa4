"""Record the outputs of the reference program itself on seeded inputs.

The reference (aav-antonov/F2M) is built from its own sources by
`make -C oracle -f ref.mk` into oracle/_ref/F2M.solver.exe (a checker, never
shipped).  This script, run on a machine with a GPU:

1. writes each seeded TSPLIB input (f2m_b200.synth, so the tests can rebuild
   it bit for bit);
2. screens it with the CPU oracle and keeps it only where the reference is
   well defined: x-span within its int area (<= 46340), no point exactly on a
   ring radius (its candidate block overflows), no repair loop (a stale comb
   index is read there), combs well below its fixed 150/550 local arrays,
   at least 300 points (the reference's host code died with SIGSEGV on a
   50-point input with N=16; such inputs are not run again);
3. runs the reference on a copy of the input in a scratch directory under
   `timeout` and stores its four output files: the report (LP text, MAX
   rank), the solution (label pairs and x), and the SHA-256 of the solution,
   .DM and _duplicates files byte for byte.

Output: tests/golden/reference_runs.npz (or the path given as argument 1).
Run from the repository root:  python tests/golden/make_reference_runs.py [out.npz]
"""
import hashlib
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from f2m_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF_EXE = os.path.join(ROOT, "oracle", "_ref", "F2M.solver.exe")

# name: (n points, seed, N); integer coordinates uniform in [0, 10^4)^2
CASES = {
    "u1000_s1_n20": (1000, 1, 20),
    "u1000_s2_n20": (1000, 2, 20),
    "u1000_s3_n20": (1000, 3, 20),
    "u1000_s4_n8": (1000, 4, 8),
    "u800_s5_n30": (800, 5, 30),
    "u300_s7_n16": (300, 7, 16),
    "u1500_s8_n16": (1500, 8, 16),
    "u3000_s9_n16": (3000, 9, 16),
    "u5000_s10_n16": (5000, 10, 16),
    "u2000_s11_n10": (2000, 11, 10),
}


def case_points(name):
    n, seed, _ = CASES[name]
    return synth.uniform_int_points(n, 7000 + seed)


def write_input(name, directory):
    x, y = case_points(name)
    path = os.path.join(directory, name + ".tsp")
    synth.write_tsplib(path, x, y)
    return path


def sha(path):
    if not os.path.exists(path):
        return ""
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def read_solution(path):
    rows = [ln.split() for ln in open(path) if ln.strip()]
    pairs = np.array([[int(a), int(b)] for a, b, _ in rows], np.int32).reshape(-1, 2)
    x = np.array([float(c) for _, _, c in rows], np.float64)
    return pairs, x


def screen(name, path):
    """Why the reference would be undefined on this input, or None."""
    _, _, N = CASES[name]
    x, _ = case_points(name)
    if len(x) < 300:
        return "fewer than 300 points"
    if np.ptp(x) > 46340 or np.ptp(x) == 0:
        return "x-span outside the reference's int area"
    lit = O.solve_file(path, N, knn=O.KNN_LITERAL)
    if lit.status == O.ERR_INPUT:
        return "a point lies exactly on a ring radius"
    if lit.stats["repair_steps"] > 0:
        return "repair loop (stale comb index in the reference)"
    if lit.status != O.OK:
        return "oracle status %d" % lit.status
    cs = getattr(lit, "comb_size", np.zeros(0))
    if len(cs) and cs.max() > 100:
        return "comb larger than 100 nodes"
    return None


def run_reference(path, N, timeout=300):
    """Exit status of the reference on `path` (0 = ran to its end)."""
    return subprocess.run(["timeout", "-k", "10", str(timeout), REF_EXE, path, str(N)],
                          stdout=subprocess.DEVNULL, stderr=subprocess.STDOUT).returncode


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden",
                                                              "reference_runs.npz")
    if not os.path.exists(REF_EXE):
        sys.exit("build the reference first: make -C oracle -f ref.mk")
    rec = {}
    names = []
    work = tempfile.mkdtemp(prefix="f2m_ref_")
    try:
        for name, (n, seed, N) in CASES.items():
            d = os.path.join(work, name)
            os.makedirs(d)
            path = write_input(name, d)
            why = screen(name, path)
            if why:
                print(f"{name}: skipped ({why})")
                continue
            rc = run_reference(path, N)
            if rc != 0:
                print(f"{name}: the reference exited with status {rc}; not recorded")
                continue
            base = f"{path}.top{N}"
            rep = open(base + ".F2M_report").read()
            m = re.search(r"Optimal Value: (\S+)", rep)
            if not m:
                print(f"{name}: reference found no optimum: {rep.strip()!r}")
                continue
            pairs, x = read_solution(base + ".F2M_solution")
            rec[name + "/lp_text"] = np.array(m.group(1))
            rec[name + "/max_rank"] = np.array(int(re.search(r"MAX edge rank: (\d+)", rep).group(1)))
            rec[name + "/pairs"] = pairs
            rec[name + "/x"] = x
            rec[name + "/sha_solution"] = np.array(sha(base + ".F2M_solution"))
            rec[name + "/sha_dm"] = np.array(sha(base + ".DM"))
            rec[name + "/sha_duplicates"] = np.array(sha(path + "_duplicates"))
            rec[name + "/time_s"] = np.array(float(re.search(r"Time: (\S+)", rep).group(1)))
            names.append(name)
            print(f"{name}: LP {m.group(1)}, {len(x)} solution lines")
    finally:
        shutil.rmtree(work, ignore_errors=True)
    rec["cases"] = np.array(names)
    np.savez_compressed(out, **rec)
    print("wrote", out)


if __name__ == "__main__":
    main()
