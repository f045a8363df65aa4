"""Autotuner for the size classes and CTA shape of the batched solver.

The batched solver runs each instance on a team of 128, 256, 512 or 1024
threads (8, 4, 2 or 1 teams per CTA) chosen by its point count; the three
bounds between the classes decide how shared memory and SMs are split
across a batch of uneven instances, and the shared memory a CTA takes
decides how much of each SM stays L1 cache for the list slices that spill
to global memory.  The potentials never depend on either (the LP value only
through the order of a sum).  This script times the solve phase (CUDA
events) of a workload under a grid of candidate bounds, re-times the five
fastest with more repetitions, then times the best few under each
shared-memory target, and records the fastest pair in a JSON file that
`f2m_b200.load_tuning()` applies:

    python -m f2m_b200.autotune                    # 4,096-instance synthetic batch
    python -m f2m_b200.autotune --out my_tuning.json --n-inst 1024 --hi 3000
"""
import argparse
import itertools
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuned_classes.json")

GRID = {
    "a": (320, 448, 576),
    "b": (768, 896, 1152, 1408),
    "c": (1536, 1792, 2304, 2816, 3328),
}
SMEM_KB = (100, 132, 164, 0)  # 0: the whole opt-in limit


def time_bounds(ctx, offs, x, y, top_k, bounds, reps):
    """Median solve-phase ms over `reps` calls after one warm-up call."""
    import f2m_b200
    f2m_b200.set_class_bounds(bounds)
    ctx.solve_batch(offs, x, y, top_k)  # warm-up (and arena growth)
    t = []
    for _ in range(reps):
        ctx.solve_batch(offs, x, y, top_k)
        ms, _ = ctx.phase_times()
        t.append(float(ms[3]))
    return float(np.median(t))


def autotune(offs, x, y, top_k, reps=2, grid=GRID, ctx=None, log=None, final_reps=5, finalists=5):
    """Time every increasing combination of the grid, then the fastest few
    again; returns (best bounds, its median solve ms, table of (bounds, ms))."""
    import f2m_b200
    own = ctx is None
    ctx = ctx or f2m_b200.Context(0)
    start = f2m_b200.get_class_bounds()
    table = []
    try:
        for a, b, c in itertools.product(grid["a"], grid["b"], grid["c"]):
            if not a < b < c:
                continue
            try:
                ms = time_bounds(ctx, offs, x, y, top_k, [a, b, c], reps)
            except f2m_b200.F2MError:
                continue  # a class cannot hold instances that large
            table.append(([a, b, c], ms))
            if log:
                log(f"bounds {a:5d} {b:5d} {c:5d}: solve {ms:8.2f} ms")
        final = []
        for bounds, _ in sorted(table, key=lambda t: t[1])[:finalists]:
            ms = time_bounds(ctx, offs, x, y, top_k, bounds, final_reps)
            final.append((bounds, ms))
            if log:
                log(f"final  {bounds}: solve {ms:8.2f} ms (median of {final_reps})")
    finally:
        f2m_b200.set_class_bounds(start)
        if own:
            ctx.close()
    bounds, ms = min(final, key=lambda t: t[1])
    return bounds, ms, table


def autotune_smem(offs, x, y, top_k, candidates, smem=SMEM_KB, reps=5, ctx=None, log=None):
    """Times each of `candidates` (bounds) under each shared-memory target;
    returns (bounds, smem_kb, median ms)."""
    import f2m_b200
    own = ctx is None
    ctx = ctx or f2m_b200.Context(0)
    start = f2m_b200.get_solver_smem_kb()
    best = None
    try:
        for kb in smem:
            f2m_b200.set_solver_smem_kb(kb)
            for bounds in candidates:
                try:
                    ms = time_bounds(ctx, offs, x, y, top_k, bounds, reps)
                except f2m_b200.F2MError:
                    continue
                if log:
                    log(f"smem {kb:4d} KB, bounds {bounds}: solve {ms:8.2f} ms")
                if best is None or ms < best[2]:
                    best = (bounds, kb, ms)
    finally:
        f2m_b200.set_solver_smem_kb(start)
        if own:
            ctx.close()
    return best


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--n-inst", type=int, default=4096)
    ap.add_argument("--lo", type=int, default=50)
    ap.add_argument("--hi", type=int, default=5000)
    ap.add_argument("--top-k", type=int, default=16)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(HERE))
    from f2m_b200 import synth
    offs, x, y = synth.config3(seed=args.seed, n_inst=args.n_inst, lo=args.lo, hi=args.hi)
    import f2m_b200
    ctx = f2m_b200.Context(0)
    bounds, ms, table = autotune(offs, x, y, args.top_k, reps=args.reps, log=print, ctx=ctx)
    top = [b for b, _ in sorted(table, key=lambda t: t[1])[:3]]
    if bounds not in top:
        top = [bounds] + top[:2]
    bounds, smem_kb, ms = autotune_smem(offs, x, y, args.top_k, top, ctx=ctx, log=print)
    ctx.close()
    rec = {"bounds": bounds, "smem_kb": smem_kb, "solve_ms": ms,
           "workload": {"n_inst": args.n_inst, "sizes": "log-uniform", "lo": args.lo, "hi": args.hi,
                        "top_k": args.top_k, "seed": args.seed},
           "table": [{"bounds": b, "solve_ms": t} for b, t in table]}
    with open(args.out, "w") as f:
        json.dump(rec, f, indent=1)
    print(f"best bounds {bounds}, smem {smem_kb} KB: solve {ms:.2f} ms -> {args.out}")


if __name__ == "__main__":
    main()
