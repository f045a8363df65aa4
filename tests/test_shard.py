"""Instance sharding over ranks (the multi-GPU path of a batch), tested with
world_size-2 gloo process groups on CPU; the per-rank solver is the CPU
oracle here (the CUDA path plugs in the same way, one GPU per rank)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from f2m_b200 import shard, synth


def test_plan_shards_cover_every_instance_once():
    offs, _, _ = synth.config3(seed=9, n_inst=97)
    for world in (1, 2, 3, 8):
        parts = shard.plan_shards(offs, world, 16)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(97))
        work = [int(np.sum(np.diff(offs)[p])) for p in parts]
        assert max(work) - min(work) <= int(np.max(np.diff(offs)))  # LPT bound


def test_take_instances_round_trip():
    offs, x, y = synth.config3(seed=2, n_inst=10, hi=300)
    idx = np.array([7, 2, 5])
    so, sx, sy = shard.take_instances(offs, x, y, idx)
    for k, b in enumerate(idx):
        assert np.array_equal(sx[so[k]:so[k + 1]], x[offs[b]:offs[b + 1]])
        assert np.array_equal(sy[so[k]:so[k + 1]], y[offs[b]:offs[b + 1]])


def _oracle_solve(offs, x, y, top_k):
    from oracle import oracle as O
    lp, st, _ = O.solve_batch(offs, x, y, top_k, threads=1)
    return lp, st


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        offs, x, y = synth.config3(seed=11, n_inst=12, hi=400)
        lp, st = shard.solve_batch_sharded(offs, x, y, 10, solve_fn=_oracle_solve)
        np.savez(f"{out}_{rank}.npz", lp=lp, st=st)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_two_ranks_gloo_match_single_process():
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "res")
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
        offs, x, y = synth.config3(seed=11, n_inst=12, hi=400)
        lp0, st0 = _oracle_solve(offs, x, y, 10)
        for r in range(2):
            g = np.load(f"{out}_{r}.npz")
            assert np.array_equal(g["st"], st0)
            assert np.array_equal(g["lp"], lp0)  # every instance solved by exactly one rank
