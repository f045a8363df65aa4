#!/usr/bin/env python
"""Benchmark: batched F2M solves/s on one B200 (and N GPUs, weak scaling).

Workload (one step): 4,096 independent instances, node counts log-uniform in
[50, 5000], integer coordinates uniform in [0, 10^4)^2, N = 16 neighbours,
reference cost mode (FP64 Euclidean) -- the batched benchmark configuration.
A step is one full solve of the whole batch: rounding and de-duplication, kNN
graph, dual descent, comb extraction and the primal value of every instance.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload large      # one 100,000-point clustered instance, N = 50

Under torchrun each rank solves its own 4,096-instance batch (seed 3 + rank);
the job time is the max over ranks.  `--impl reference` times the CPU
restatement of the reference solver (oracle/) on the host cores instead.

On one GPU the line also checks the metric's precision clause: the oracle's
LP value of every sampled instance (the whole batch by default) against the
GPU's, exiting with status 3 above 1e-9 relative.  It carries two more
workloads as sub-objects, each with its own roofline, end-to-end figure, CPU
baseline and parity check: `large` (one 100,000-point clustered instance,
N = 50, the grid-wide solver) and `smooth` (smoothed bound + adjoint of 1,024
jittered-lattice instances, N = 24).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from f2m_b200 import synth  # noqa: E402

METRIC = "batched F2M solves/s vs plain per-instance loop on B200 at LP rel err<=1e-9"
N_INST = 4096
TOP_K = 16
FLUSH_BYTES = 256 << 20
LP_TOL = 1e-9

# FP64 pipe operations of the persistent solver's Jacobi step, counted from
# its source (f2m_kernels.cu Solver::step / slice_hgrad / half_grad,
# f2m_device.cuh top3_insert):
#   per list entry a warp lane sweeps (padding of the 32-node slices
#   included): 2 DADD for the reduced cost (D + H[lo]) + H[hi] and 3 DSETP
#   for the top-3 insertion;
#   per lane updating a node: 1 DSETP (first value below the 1e6 sentinels),
#   1 DADD (v1 + v2), 2 DMUL (/2, *0.5) and 1 DADD (H + grad/2).
# Partitions, gradient checks and comb extraction are not counted, so the
# fraction is a lower bound.
FP64_PER_ENTRY = 5
FP64_PER_LANE = 5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch", choices=["batch", "large", "smooth", "smooth1"],
                    help="batch: 4,096 mixed-size instances (the headline); large: one "
                         "100,000-point Gaussian-mixture instance with N=50 (grid-wide solver); "
                         "smooth: smoothed bound + adjoint of 1,024 jittered-lattice instances "
                         "(N=24); smooth1: the same on 10,000 uniform FP32 points (N=30)")
    ap.add_argument("--large-n", type=int, default=100_000, help="points of the large instance")
    ap.add_argument("--smooth-solver", type=int, default=0, choices=[0, 1, 2],
                    help="smoothed bound: 0 auto, 1 one CTA per instance, 2 one launch per step")
    ap.add_argument("--n-inst", type=int, default=N_INST)
    ap.add_argument("--plain-sample", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sub", action="store_true",
                    help="leave out the large and smooth sub-objects of the batch line")
    ap.add_argument("--size-range", type=int, nargs=2, default=None,
                    help="keep only instances with lo <= points <= hi (profiling one solver class)")
    return ap.parse_args()


def workload(rank, n_inst, size_range=None):
    offs, x, y = synth.config3(seed=3 + rank, n_inst=n_inst)
    if size_range is not None:
        n = np.diff(offs)
        keep = np.nonzero((n >= size_range[0]) & (n <= size_range[1]))[0]
        xs = [x[offs[b]:offs[b + 1]] for b in keep]
        ys = [y[offs[b]:offs[b + 1]] for b in keep]
        offs = np.concatenate([[0], np.cumsum(n[keep])]).astype(np.int64)
        x, y = np.concatenate(xs), np.concatenate(ys)
    return offs, x, y


def config(args, world):
    return {"workload": f"config3: {args.n_inst} instances/GPU, V log-uniform [50,5000], "
                        f"int coords uniform [0,1e4)^2, N={TOP_K}, reference FP64 Euclidean cost",
            "n_inst_per_gpu": args.n_inst, "top_k": TOP_K, "seed": "3 + rank",
            "l2": f"flushed between timed steps ({FLUSH_BYTES >> 20} MiB write)",
            "parallelism": f"instance sharding over {world} GPU(s), no collective"}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (a restatement of the reference solver)
# ---------------------------------------------------------------------------
def cpu_sample(offs, n_sample):
    n = len(offs) - 1
    idx = np.linspace(0, n - 1, n_sample).astype(np.int64)
    return idx


def run_cpu(offs, x, y, idx, threads):
    from oracle import oracle as O
    sub_offs = [0]
    xs, ys = [], []
    for b in idx:
        xs.append(x[offs[b]:offs[b + 1]])
        ys.append(y[offs[b]:offs[b + 1]])
        sub_offs.append(sub_offs[-1] + offs[b + 1] - offs[b])
    so = np.array(sub_offs, np.int64)
    xx, yy = np.concatenate(xs), np.concatenate(ys)
    t0 = time.perf_counter()
    lp, st, it = O.solve_batch(so, xx, yy, TOP_K, threads=threads)
    dt = time.perf_counter() - t0
    return lp, st, dt


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def sample_size(offs, x, y, threads, target_s):
    """Instances (spread evenly over the batch) that keep the CPU busy for
    about target_s seconds: grow a pilot sample until it takes a quarter of
    that, then extrapolate (at most the whole batch)."""
    total = len(offs) - 1
    n = min(total, 4 * threads)
    while True:
        _, _, dt = run_cpu(offs, x, y, cpu_sample(offs, n), threads)
        if dt >= target_s / 4 or n >= total:
            break
        n = min(total, 4 * n)
    return int(min(total, max(n, n * target_s / max(dt, 1e-3))))


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def lp_parity(lp_gpu, st_gpu, lp_cpu, st_cpu):
    """Largest relative LP difference over instances both sides solved, and
    whether the statuses agree instance by instance."""
    both = (st_gpu == 0) & (st_cpu == 0)
    rel = np.abs(lp_gpu[both] - lp_cpu[both]) / np.maximum(np.abs(lp_cpu[both]), 1e-300)
    return {"max_lp_rel_err_vs_oracle": float(rel.max()) if rel.size else None,
            "n_checked": int(both.sum()), "status_equal": bool(np.array_equal(st_gpu, st_cpu)),
            "tolerance": LP_TOL}


def cpu_baseline(offs, x, y, lp_gpu=None, st_gpu=None, target_s=15.0):
    """The oracle on all host threads over a bounded sample of the batch (the
    whole batch when it fits in target_s), plus one core on a smaller sample.
    With the GPU's results given, also the LP parity of the sampled instances."""
    threads = cpu_threads()
    n = sample_size(offs, x, y, threads, target_s)
    idx = cpu_sample(offs, n)
    lp, st, dt = run_cpu(offs, x, y, idx, threads)
    # one core: about 5 s of work, spread over the batch the same way
    per_inst = dt * threads / len(idx)
    n1 = int(max(4, min(len(idx), 5.0 / max(per_inst, 1e-6))))
    idx1 = cpu_sample(offs, n1)
    _, _, dt1 = run_cpu(offs, x, y, idx1, 1)
    out = {"value": len(idx) / dt, "unit": "solves/s", "cores": threads, "kind": "port",
           "cpu_model": cpu_model(),
           "sample": f"{len(idx)} instances spread evenly over the batch (same size "
                     f"distribution), CPU oracle restating the reference solver, "
                     f"{threads} threads, {dt:.1f} s",
           "one_core": {"value": len(idx1) / dt1, "unit": "solves/s", "cores": 1,
                        "sample": f"{len(idx1)} instances spread evenly over the batch, "
                                  f"{dt1:.1f} s"}}
    parity = None
    if lp_gpu is not None:
        parity = lp_parity(np.asarray(lp_gpu)[idx], np.asarray(st_gpu)[idx], lp, st)
    return out, parity


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def alg_bytes(work):
    """Algorithmic bytes of the dual iterations: per swept (active) slot the
    12-byte (D, neighbour) record, per node 28 bytes (F in, F out, list offset,
    gathered F counted once per node)."""
    return 12.0 * work["slot_iters"] + 28.0 * work["node_iters"]


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(workload, work):
    """DRAM bytes of the solve phase, scaled from the committed ncu summary of a
    smaller case by the dual-iteration work (node iterations), or None.  The
    summary holds a line `traffic_per_node_iter <workload> <bytes>`."""
    p = os.path.join(ROOT, "profiles", "k_solve_dram_traffic.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) == 3 and f[0] == "traffic_per_node_iter" and f[1] == workload:
            return float(f[2]) * work["node_iters"]
    return None


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def reference_arm(args, rank, world):
    if rank != 0:
        return
    offs, x, y = workload(0, args.n_inst)
    threads = cpu_threads()
    # each step is a bounded sample (about 5 s of CPU work) of the same batch
    idx = cpu_sample(offs, sample_size(offs, x, y, threads, 5.0))
    for _ in range(args.warmup):
        run_cpu(offs, x, y, idx[: max(4, len(idx) // 8)], threads)
    times = []
    for _ in range(args.steps):
        _, st, dt = run_cpu(offs, x, y, idx, threads)
        times.append(dt)
    tot = sum(times)
    value = len(idx) * args.steps / tot
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config(args, world), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                             "cpu_model": cpu_model(),
                             "sample": f"{len(idx)} instances spread over the batch per step, "
                                       f"CPU restatement of the reference solver (oracle/), "
                                       f"{threads} threads"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ours_arm(args, rank, world, local_rank):
    import torch

    import f2m_b200
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    tuned = f2m_b200.load_tuning()  # size-class bounds from f2m_b200/autotune.py
    offs, x, y = workload(rank, args.n_inst, args.size_range)
    n_inst = len(offs) - 1
    ctx = f2m_b200.Context(local_rank)
    d_offs = torch.from_numpy(offs).to(dev)
    d_x = torch.from_numpy(x).to(dev)
    d_y = torch.from_numpy(y).to(dev)
    d_lp = torch.empty(n_inst, dtype=torch.float64, device=dev)
    d_st = torch.empty(n_inst, dtype=torch.int32, device=dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def step():
        ctx.solve_batch_device(offs, d_offs.data_ptr(), d_x.data_ptr(), d_y.data_ptr(), TOP_K,
                               d_lp.data_ptr(), d_st.data_ptr())
        ctx.sync()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        step()
    st = d_st.cpu().numpy()
    lp = d_lp.cpu().numpy()
    assert np.all(st == 0), f"instances not solved: {np.unique(st, return_counts=True)}"
    assert np.all(np.isfinite(lp))

    clk = Clocks(local_rank)
    l0 = ctx.kernel_launches()
    ms_steps, phase = [], np.zeros(4)
    work = None
    clk.start()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        ms_steps.append(e0.elapsed_time(e1))
        ph, work = ctx.phase_times()
        phase += ph
    clocks = clk.stop()
    launches = ctx.kernel_launches() - l0
    ms = float(np.mean(ms_steps))
    t_job = ms
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_job = float(t.item())
    value = n_inst * world / (t_job / 1e3)
    phase /= args.steps

    # end to end through the public API with host buffers (pinned)
    hx = torch.from_numpy(x).pin_memory().numpy()
    hy = torch.from_numpy(y).pin_memory().numpy()
    ho = torch.from_numpy(offs).pin_memory().numpy()
    ctx.solve_batch(ho, hx, hy, TOP_K)
    e2e_ms = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.fill_(1)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        lp_h, st_h = ctx.solve_batch(ho, hx, hy, TOP_K)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e = float(np.mean(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e = float(t.item())
    assert np.array_equal(st_h, st) and np.array_equal(lp_h, lp)

    # plain per-instance loop on a sample (one instance per call, device-resident)
    sample = cpu_sample(offs, min(args.plain_sample, n_inst))
    plain_ms = 0.0
    for b in sample:
        o1 = np.array([0, offs[b + 1] - offs[b]], np.int64)
        d_o1 = torch.from_numpy(o1).to(dev)
        xb, yb = d_x[offs[b]:offs[b + 1]], d_y[offs[b]:offs[b + 1]]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.solve_batch_device(o1, d_o1.data_ptr(), xb.data_ptr(), yb.data_ptr(), TOP_K,
                               d_lp[b:b + 1].data_ptr(), d_st[b:b + 1].data_ptr())
        ctx.sync()
        plain_ms += 1e3 * (time.perf_counter() - t0)
    plain = len(sample) / (plain_ms / 1e3)
    lp_plain = d_lp.cpu().numpy()[sample]
    plain_err = float(np.max(np.abs(lp_plain - lp[sample]) / np.abs(lp[sample])))

    # FP64 pipe peak of this GPU (the solver's roofline), measured after the
    # timed region on the same context
    fp64_dadd = ctx.fp64_rate(0)
    fp64_dsetp = ctx.fp64_rate(1)
    if rank != 0:
        return
    # roofline of the dominant kernel: the persistent solver, bound by the
    # FP64 pipe (its working set stays in shared memory)
    solve_ms = phase[3]
    ops = FP64_PER_ENTRY * work["pad_iters"] + FP64_PER_LANE * work["lane_iters"]
    achieved = ops / (solve_ms / 1e3) / 1e12
    peak_fp64 = min(fp64_dadd, fp64_dsetp) / 1e12
    hbm_peak, peak_kind = measured_peak()
    ab = alg_bytes(work)
    tr = profile_traffic("batch", work)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_job,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": config(args, world),
        "roofline": {"bound": "fp64", "kernel": "k_solve (persistent CTA-per-instance solver)",
                     "achieved": achieved, "peak": peak_fp64, "unit": "T FP64 lane-ops/s",
                     "frac": achieved / peak_fp64,
                     "peak_kind": "measured in this run (f2m_fp64_rate: best of 3 launches, "
                                  "every SM at full occupancy; min of the DADD and DSETP rates)",
                     "peak_dadd": fp64_dadd / 1e12, "peak_dsetp": fp64_dsetp / 1e12,
                     "fp64_ops_per_launch": ops,
                     "fp64_ops_model": f"{FP64_PER_ENTRY} per swept list entry (pad_iters) + "
                                       f"{FP64_PER_LANE} per node lane (lane_iters), from the source",
                     "time": "solve phase (CUDA events), all four size classes",
                     "traffic": tr,
                     "smem_gbs": ab / (solve_ms / 1e3) / 1e9,
                     "smem_bytes_per_launch": ab,
                     "hbm_peak_gbs": hbm_peak, "hbm_peak_kind": peak_kind,
                     "dram_gbs": (tr / (solve_ms / 1e3) / 1e9) if tr else None,
                     "note": "the active set and potentials stay in shared memory; smem_gbs is "
                             "the algorithmic byte rate (12 B per active slot + 28 B per node "
                             "per iteration), served on chip; traffic is the DRAM bytes"},
        "e2e": {"value": n_inst * world / (e2e / 1e3), "unit": "solves/s",
                "h2d_bytes_per_step": int(ho.nbytes + hx.nbytes + hy.nbytes),
                "d2h_bytes_per_step": int(n_inst * (8 + 4))},
        "clocks": clocks,
        "gpu_launches": int(launches // max(args.steps, 1)),
        "gpu_launches_total": int(launches),
        "phases_ms": {"prep": phase[0], "knn": phase[1], "graph": phase[2], "solve": phase[3],
                      "host_and_copies": ms - float(np.sum(phase))},
        "work": work,
        "plain_loop": {"value": plain, "unit": "solves/s", "sample": f"{len(sample)} instances, "
                       "one f2m_solve_batch_device call each", "speedup": value / world / plain,
                       "max_lp_rel_err_vs_batched": plain_err},
        "iterations_mean": float(work["node_iters"] / max(work["points"], 1)),
        "class_bounds": f2m_b200.get_class_bounds(), "class_bounds_tuned": tuned is not None,
    }
    bad = False
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"], line["parity"] = cpu_baseline(offs, x, y, lp, st)
        p = line["parity"]
        bad = (p["max_lp_rel_err_vs_oracle"] is None or p["max_lp_rel_err_vs_oracle"] > LP_TOL
               or not p["status_equal"])
    if world == 1 and not args.no_sub:
        ctx.close()
        line["large"] = large_sub(args, local_rank)
        line["smooth"] = smooth_sub(args, local_rank)
        for k in ("large", "smooth"):
            p = line[k].get("parity") or {}
            bad |= bool(p.get("fail"))
    print(json.dumps(line), flush=True)
    if bad:
        print("parity check failed (LP values differ from the oracle's)", file=sys.stderr)
        sys.exit(3)


def _pool_map(fn, items, threads):
    """fn over items on `threads` host threads (the oracle releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(fn, items))


def large_sub(args, local_rank, steps=3, warmup=2):
    """Sub-object of the batch line: one 100,000-point clustered instance
    (64 Gaussian clusters, sigma 0.5% of a 10^6 box, 10% uniform background,
    rounded to integers), N = 50, through f2m_solve_points (host arrays in,
    full result out), solved by the grid-wide solver.  Roofline of
    k_solve_grid against the measured HBM copy rate; the oracle on all host
    threads is its CPU baseline and parity check (LP value, potentials)."""
    import torch

    import f2m_b200
    dev = torch.device("cuda", local_rank)
    x, y = synth.config2(2, n=args.large_n)
    n_large = 50
    ctx = f2m_b200.Context(local_rank)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(warmup):
        r = ctx.solve_points(x, y, n_large)
    clk = Clocks(local_rank)
    l0 = ctx.kernel_launches()
    wall, phase = [], np.zeros(4)
    clk.start()
    for _ in range(steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = ctx.solve_points(x, y, n_large)
        wall.append(1e3 * (time.perf_counter() - t0))
        ph, work = ctx.phase_times()
        phase += ph
    clocks = clk.stop()
    launches = ctx.kernel_launches() - l0
    ctx.close()
    phase /= steps
    dev_ms = float(np.sum(phase))
    e2e_ms = float(np.mean(wall))
    peak, peak_kind = measured_peak()
    ab = alg_bytes(work)
    achieved = ab / (phase[3] / 1e3) / 1e9
    out = {
        "metric": "F2M solves/s, one large clustered instance (device phases)",
        "value": 1e3 / dev_ms, "unit": "solves/s", "steps": steps, "warmup": warmup,
        "ms_per_step": dev_ms,
        "config": {"workload": f"{args.large_n:,} points: 64 Gaussian clusters (sigma 0.5% of a "
                               "10^6 box) + 10% uniform background, rounded; N=50, reference FP64 "
                               "Euclidean cost", "top_k": n_large, "seed": 2,
                   "l2": f"flushed between timed steps ({FLUSH_BYTES >> 20} MiB write)"},
        "roofline": {"bound": "hbm", "kernel": "k_solve_grid (grid-wide dual descent)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": profile_traffic("large", work),
                     "algorithmic_bytes_per_launch": ab,
                     "bytes_model": "12 B per active slot + 28 B per node, per Jacobi iteration",
                     "time": "solve phase (CUDA events)"},
        "e2e": {"value": 1e3 / e2e_ms, "unit": "solves/s",
                "h2d_bytes_per_step": int(x.nbytes + y.nbytes),
                "d2h_bytes_per_step": int(r.n_edges * 40 + r.n_nodes * 12)},
        "clocks": clocks, "gpu_launches": int(launches // max(steps, 1)),
        "phases_ms": {"prep": phase[0], "knn": phase[1], "graph": phase[2], "solve": phase[3],
                      "host_and_copies": e2e_ms - dev_ms},
        "work": work, "lp": r.lp, "n_nodes": r.n_nodes, "n_edges": r.n_edges,
        "iterations": int(r.stats["iterations"]),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        threads = cpu_threads()
        t0 = time.perf_counter()
        o = O.solve_points(x, y, n_large, threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "solves/s", "cores": threads,
                               "kind": "port", "cpu_model": cpu_model(),
                               "sample": f"the whole instance once, CPU oracle, {threads} threads, "
                                         f"{dt:.1f} s"}
        rel = abs(r.lp - o.lp) / abs(o.lp)
        same_f = bool(o.F is not None and np.array_equal(r.F, o.F))
        out["parity"] = {"lp_rel_err_vs_oracle": rel, "F_bit_identical": same_f,
                         "status_equal": r.status == o.status, "tolerance": LP_TOL,
                         "fail": bool(rel > LP_TOL or not same_f or r.status != o.status)}
    return out


def smooth_sub(args, local_rank, steps=3, warmup=1):
    """Sub-object of the batch line: smoothed bound + coordinate gradient of
    1,024 jittered-lattice instances (200-2,000 points, spacing 1, jitter
    +-0.3, FP32), N = 24, tau = 1e-3, 100 damped Jacobi steps, adjoint with
    checkpoints every 16 steps; host arrays in and out through the C ABI.
    The FP64 host oracle on a bounded sample is the CPU baseline and the
    parity check (bound and gradient)."""
    import torch

    import f2m_b200
    offs, x, y = synth.config5(5)
    N = 24
    n_inst = len(offs) - 1
    ctx = f2m_b200.Context(local_rank)
    p = f2m_b200.default_smooth_params()
    for _ in range(warmup):
        ctx.smoothed_bound(offs, x, y, N, params=p, grad=True)
    clk = Clocks(local_rank)
    l0 = ctx.kernel_launches()
    ms, kterms, kms = [], [], []
    clk.start()
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L, gx, gy = ctx.smoothed_bound(offs, x, y, N, params=p, grad=True)
        ms.append(1e3 * (time.perf_counter() - t0))
        tr, km = ctx.smooth_work()  # logistic terms and time of the persistent kernel
        kterms.append(tr)
        kms.append(km)
    clocks = clk.stop()
    launches = ctx.kernel_launches() - l0
    # roofline: the persistent kernel (one CTA per instance) evaluates
    # logistic terms (one FP64 exp and two divisions each: the Newton sums
    # of every node root, softplus, sigma and sigma'); its peak is the same
    # term measured at full occupancy on this GPU
    peak_terms = ctx.fp64_rate(2, repeats=3)
    ctx.close()
    t = float(np.mean(ms))
    achieved = float(np.mean(kterms)) / (float(np.mean(kms)) / 1e3)
    out = {
        "metric": "smoothed F2M bound + coordinate gradient, instances/s",
        "value": n_inst / (t / 1e3), "unit": "instances/s", "steps": steps, "warmup": warmup,
        "ms_per_step": t, "dtype": "f64 (FP32 coordinates)",
        "config": {"workload": "1,024 instances, sizes uniform in [200,2000], jittered unit "
                               "lattice (+-0.3), FP32", "top_k": N, "tau": p.tau, "iters": p.iters,
                   "damping": p.damping, "checkpoint": p.checkpoint, "seed": 5},
        "e2e": {"value": n_inst / (t / 1e3), "unit": "instances/s",
                "h2d_bytes_per_step": int(offs.nbytes + x.nbytes + y.nbytes),
                "d2h_bytes_per_step": int(L.nbytes + gx.nbytes + gy.nbytes)},
        "clocks": clocks, "gpu_launches": int(launches // max(steps, 1)),
        "L_mean": float(np.mean(L)),
        "roofline": {"bound": "fp64 exp+div", "kernel": "k_sbound (persistent, one CTA per instance)",
                     "achieved": achieved / 1e9, "peak": peak_terms / 1e9, "unit": "G logistic terms/s",
                     "frac": achieved / peak_terms if peak_terms > 0 else None,
                     "peak_kind": "measured in this run (f2m_fp64_rate kind 2: the same term, four "
                                  "independent sums per thread, every SM at full occupancy)",
                     "terms_per_launch": float(np.mean(kterms)), "kernel_ms": float(np.mean(kms)),
                     "traffic": None},
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        threads = cpu_threads()

        def host(b):
            s_, e_ = offs[b], offs[b + 1]
            return O.smooth_bound(x[s_:e_], y[s_:e_], N, tau=p.tau, iters=p.iters,
                                  omega=p.damping, newton_max=p.newton_max, grad=True)
        # pilot: size the sample for about 10 s of host work
        pilot = list(range(0, n_inst, max(1, n_inst // (2 * threads))))[: 2 * threads]
        t0 = time.perf_counter()
        _pool_map(host, pilot, threads)
        per = (time.perf_counter() - t0) / len(pilot)
        n_s = int(min(n_inst, max(len(pilot), 10.0 / max(per, 1e-6))))
        idx = np.linspace(0, n_inst - 1, n_s).astype(np.int64)
        t0 = time.perf_counter()
        res = _pool_map(host, list(idx), threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(idx) / dt, "unit": "instances/s", "cores": threads,
                               "kind": "port", "cpu_model": cpu_model(),
                               "sample": f"{len(idx)} instances spread over the batch, FP64 host "
                                         f"oracle (bound + adjoint), {threads} threads, {dt:.1f} s"}
        l_err, g_err = 0.0, 0.0
        for b, (Lo, dx, dy, _) in zip(idx, res):
            s_, e_ = offs[b], offs[b + 1]
            l_err = max(l_err, abs(L[b] - Lo) / abs(Lo))
            scale = max(np.abs(dx).max(), np.abs(dy).max(), 1e-300)
            g_err = max(g_err, float(max(np.abs(gx[s_:e_] - dx).max(),
                                         np.abs(gy[s_:e_] - dy).max()) / scale))
        out["parity"] = {"n_checked": len(idx), "max_L_rel_err_vs_oracle": l_err,
                         "max_grad_err_rel_to_max": g_err,
                         "tolerance": {"L": 1e-9, "grad": 1e-5},
                         "fail": bool(l_err > 1e-9 or g_err > 1e-5)}
    return out


def large_arm(args, rank, world, local_rank):
    """One 100,000-point instance (64 Gaussian clusters + 10% background), N=50:
    replicas only (the instance does not shard); the grid-wide solver."""
    import torch

    import f2m_b200
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    x, y = synth.config2(2 + rank, n=args.large_n)
    n_large = 50
    ctx = f2m_b200.Context(local_rank)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        r = ctx.solve_points(x, y, n_large)
    assert r.status == 0
    clk = Clocks(local_rank)
    l0 = ctx.kernel_launches()
    wall, phase = [], np.zeros(4)
    clk.start()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = ctx.solve_points(x, y, n_large)
        wall.append(1e3 * (time.perf_counter() - t0))
        ph, work = ctx.phase_times()
        phase += ph
    clocks = clk.stop()
    launches = ctx.kernel_launches() - l0
    phase /= args.steps
    dev_ms = float(np.sum(phase))
    e2e_ms = float(np.mean(wall))
    t = [dev_ms, e2e_ms]
    if world > 1:
        tt = torch.tensor(t, dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = tt.tolist()
    if rank != 0:
        return
    peak, peak_kind = measured_peak()
    ab = alg_bytes(work)
    achieved = ab / (phase[3] / 1e3) / 1e9
    line = {
        "metric": "F2M solves/s, one large clustered instance", "value": world * 1e3 / t[0],
        "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t[0], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.large_n:,} points: 64 Gaussian clusters (sigma 0.5% of a "
                               "10^6 box) + 10% uniform background, rounded; N=50", "top_k": n_large,
                   "seed": "2 + rank", "parallelism": f"replicas on {world} GPU(s)",
                   "l2": f"flushed between timed steps ({FLUSH_BYTES >> 20} MiB write)"},
        "roofline": {"bound": "hbm", "kernel": "k_solve_grid (grid-wide dual descent)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": profile_traffic("large", work),
                     "algorithmic_bytes_per_launch": ab},
        "e2e": {"value": world * 1e3 / t[1], "unit": "solves/s",
                "h2d_bytes_per_step": int(x.nbytes + y.nbytes), "d2h_bytes_per_step": None},
        "clocks": clocks, "gpu_launches": int(launches // max(args.steps, 1)),
        "phases_ms": {"prep": phase[0], "knn": phase[1], "graph": phase[2], "solve": phase[3]},
        "work": work, "lp": r.lp, "n_nodes": r.n_nodes, "n_edges": r.n_edges,
        "iterations": int(r.stats["iterations"]) if "iterations" in r.stats else None,
    }
    print(json.dumps(line), flush=True)


def smooth_arm(args, rank, world, local_rank):
    """Smoothed bound + adjoint (tau = 1e-3, 100 damped Jacobi steps,
    checkpoints every 16): `smooth` = 1,024 jittered-lattice instances of
    200-2,000 points (N=24), `smooth1` = 10,000 uniform FP32 points (N=30).
    Host arrays in and out through the C ABI (the entry points copy)."""
    import torch

    import f2m_b200
    torch.cuda.set_device(local_rank)
    if args.workload == "smooth":
        offs, x, y = synth.config5(5 + rank)
        N, desc = 24, "1,024 instances, sizes uniform in [200,2000], jittered unit lattice (+-0.3), FP32"
    else:
        x, y = synth.config4(4 + rank)
        offs, N, desc = np.array([0, len(x)], np.int64), 30, "10,000 FP32 points uniform in [0,1)^2"
    n_inst = len(offs) - 1
    ctx = f2m_b200.Context(local_rank)
    p = f2m_b200.default_smooth_params(solver=args.smooth_solver)
    for _ in range(args.warmup):
        ctx.smoothed_bound(offs, x, y, N, params=p, grad=True)
    clk = Clocks(local_rank)
    l0 = ctx.kernel_launches()
    ms, kterms, kms = [], [], []
    clk.start()
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L, gx, gy = ctx.smoothed_bound(offs, x, y, N, params=p, grad=True)
        ms.append(1e3 * (time.perf_counter() - t0))
        tr, km = ctx.smooth_work()
        kterms.append(tr)
        kms.append(km)
    clocks = clk.stop()
    launches = ctx.kernel_launches() - l0
    roof = None
    if min(kterms) >= 0 and np.mean(kms) > 0:  # the persistent kernel ran (its terms are counted)
        peak_terms = ctx.fp64_rate(2, repeats=3)
        ach = float(np.mean(kterms)) / (float(np.mean(kms)) / 1e3)
        roof = {"bound": "fp64 exp+div", "kernel": "k_sbound (persistent, one CTA per instance)",
                "achieved": ach / 1e9, "peak": peak_terms / 1e9, "unit": "G logistic terms/s",
                "frac": ach / peak_terms if peak_terms > 0 else None,
                "peak_kind": "measured in this run (f2m_fp64_rate kind 2)",
                "terms_per_launch": float(np.mean(kterms)), "kernel_ms": float(np.mean(kms)),
                "traffic": None}
    t = float(np.mean(ms))
    if world > 1:
        tt = torch.tensor([t], dtype=torch.float64, device=torch.device("cuda", local_rank))
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = float(tt.item())
    if rank != 0:
        return
    line = {
        "metric": "smoothed F2M bound + coordinate gradient, instances/s", "value": n_inst * world / (t / 1e3),
        "unit": "instances/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (FP32 coordinates)", "data": "synthetic (seeded)",
        "config": {"workload": desc, "top_k": N, "tau": p.tau, "iters": p.iters,
                   "damping": p.damping, "checkpoint": p.checkpoint,
                   "parallelism": f"instance sharding over {world} GPU(s), no collective"},
        "roofline": roof,
        "e2e": {"value": n_inst * world / (t / 1e3), "unit": "instances/s",
                "h2d_bytes_per_step": int(offs.nbytes + x.nbytes + y.nbytes),
                "d2h_bytes_per_step": int(L.nbytes + gx.nbytes + gy.nbytes)},
        "clocks": clocks, "gpu_launches": int(launches // max(args.steps, 1)),
        "L_mean": float(np.mean(L)), "grad_rms": float(np.sqrt(np.mean(gx.astype(np.float64) ** 2))),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        elif args.workload == "large":
            large_arm(args, rank, world, local_rank)
        elif args.workload in ("smooth", "smooth1"):
            smooth_arm(args, rank, world, local_rank)
        else:
            ours_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
