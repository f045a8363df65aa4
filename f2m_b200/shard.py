"""Instance sharding of a batch over the ranks of a process group.

Instances of a batch are independent, so a batch spreads over GPUs with no
exchange on the data path: each rank solves its own share of the instances
on its own GPU, and the per-instance results are gathered once at the end.
The shares are balanced by a greedy longest-processing-time bin pack on the
estimated work of an instance (points x neighbours).

    lp, status = solve_batch_sharded(offs, x, y, top_k)     # under torchrun

`solve_fn(offs, x, y, top_k) -> (lp, status)` defaults to the CUDA path of
this rank's GPU (f2m_b200.Context(local rank).solve_batch).
"""
import os

import numpy as np


def plan_shards(offs, n_ranks, top_k=16):
    """Instance indices per rank (ascending within a rank), balanced by
    points x top_k with the largest instances placed first."""
    offs = np.asarray(offs, np.int64)
    work = np.diff(offs) * max(int(top_k), 1)
    order = np.argsort(-work, kind="stable")
    load = np.zeros(n_ranks, np.int64)
    owner = np.empty(len(work), np.int64)
    for b in order:
        r = int(np.argmin(load))
        owner[b] = r
        load[r] += work[b]
    return [np.nonzero(owner == r)[0] for r in range(n_ranks)]


def take_instances(offs, x, y, idx):
    """(offs, x, y) of the instances idx of a batch, in that order."""
    offs = np.asarray(offs, np.int64)
    sizes = offs[idx + 1] - offs[idx]
    sub = np.zeros(len(idx) + 1, np.int64)
    sub[1:] = np.cumsum(sizes)
    if len(idx) == 0:
        return sub, np.zeros(0, x.dtype), np.zeros(0, y.dtype)
    xs = np.concatenate([x[offs[b]:offs[b + 1]] for b in idx])
    ys = np.concatenate([y[offs[b]:offs[b + 1]] for b in idx])
    return sub, xs, ys


def _default_solve(offs, x, y, top_k):
    import f2m_b200
    ctx = f2m_b200.Context(int(os.environ.get("LOCAL_RANK", "0")))
    try:
        return ctx.solve_batch(offs, x, y, top_k)
    finally:
        ctx.close()


def solve_batch_sharded(offs, x, y, top_k, solve_fn=None, group=None):
    """Solve a batch over all ranks of `group` (torch.distributed); every rank
    passes the whole batch and gets back the whole batch's (lp, status)."""
    import torch
    import torch.distributed as dist
    solve_fn = solve_fn or _default_solve
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shards = plan_shards(offs, world, top_k)
    mine = shards[rank]
    lp = np.zeros(len(mine), np.float64)
    st = np.zeros(len(mine), np.int32)
    if len(mine):
        so, sx, sy = take_instances(offs, x, y, mine)
        lp, st = solve_fn(so, sx, sy, top_k)
    n = len(offs) - 1
    # one gather of the results: a rank's values scattered into a full-size
    # buffer, then summed (every instance has exactly one owner)
    full_lp = torch.zeros(n, dtype=torch.float64)
    full_st = torch.zeros(n, dtype=torch.int64)
    full_lp[torch.from_numpy(mine)] = torch.from_numpy(np.asarray(lp, np.float64))
    full_st[torch.from_numpy(mine)] = torch.from_numpy(np.asarray(st, np.int64))
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
        full_lp, full_st = full_lp.to(dev), full_st.to(dev)
    dist.all_reduce(full_lp, group=group)
    dist.all_reduce(full_st, group=group)
    return full_lp.cpu().numpy(), full_st.cpu().numpy().astype(np.int32)
