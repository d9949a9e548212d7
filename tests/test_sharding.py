"""Multi-GPU host logic on CPU: partition of a ragged batch, scatter back, and
two gloo ranks exchanging shard results and taking the max over ranks."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from xtbloom_b200 import sharding as S
from xtbloom_b200 import workloads as W


def fake_compute(b):
    """Deterministic per-system stand-in for a compute call (host only)."""
    off = np.asarray(b.atom_offsets)
    z = np.asarray(b.atomic_numbers, float)
    x = np.asarray(b.positions)
    e = np.array([z[off[i]:off[i + 1]].sum() + 1e-3 * x[3 * off[i]:3 * off[i + 1]].sum()
                  for i in range(b.batch_size)])
    return {"energies": e, "forces": 2.0 * x, "atomic_charges": 0.1 * z,
            "scc_iterations": np.full(b.batch_size, 7, np.int32),
            "scc_converged": np.ones(b.batch_size, np.uint8),
            "per_system_status": np.zeros(b.batch_size, np.int32)}


def test_plan_covers_every_system_once_and_balances_cost():
    b = W.config1(300)
    cost = S.predicted_cost(b)
    for world in (1, 2, 3, 8):
        shards = S.plan_shards(b, world)
        allidx = np.sort(np.concatenate(shards))
        assert np.array_equal(allidx, np.arange(b.batch_size))
        loads = [cost[s].sum() for s in shards]
        assert max(loads) - min(loads) <= cost.max()
        assert all(np.all(np.diff(s) > 0) for s in shards)


def test_shard_then_scatter_back_equals_the_whole_batch():
    b = W.config1(97)
    direct = fake_compute(b)
    shards = S.plan_shards(b, 4)
    parts = [fake_compute(S.shard(b, idx)) for idx in shards]
    back = S.scatter_back(b, shards, parts)
    for k in direct:
        assert np.array_equal(back[k], direct[k]), k


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        b = W.config1(64)
        shards = S.plan_shards(b, world)
        mine = fake_compute(S.shard(b, shards[rank]))
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        tmax = bench.allreduce_max(float(rank + 1), world)
        bench.barrier(world)
        if rank == 0:
            back = S.scatter_back(b, shards, gathered)
            direct = fake_compute(b)
            q.put((tmax, all(np.array_equal(back[k], direct[k]) for k in direct)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_shards_and_take_max():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    tmax, ok = q.get(timeout=5)
    assert tmax == 2.0 and ok
