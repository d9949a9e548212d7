"""Multi-GPU host logic on CPU: the cost model, the partition of a ragged
batch with its attachments (spin channels, point charges, fields, charge
response), scatter back, and gloo ranks running one batch through
``sharding.distributed_compute`` and taking the max over ranks."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from xtbloom_b200 import sharding as S
from xtbloom_b200 import workloads as W


def fake_compute(b):
    """Deterministic per-system stand-in for a compute call (host only): every
    output depends on the system's own atoms and attachments only."""
    off = np.asarray(b.atom_offsets)
    z = np.asarray(b.atomic_numbers, float)
    x = np.asarray(b.positions)
    e = np.array([z[off[i]:off[i + 1]].sum() + 1e-3 * x[3 * off[i]:3 * off[i + 1]].sum()
                  for i in range(b.batch_size)])
    if b.spin_channels is not None:
        e = e + 0.5 * np.asarray(b.spin_channels)
    q = 0.1 * z
    out = {"scc_iterations": np.full(b.batch_size, 7, np.int32),
           "scc_converged": np.ones(b.batch_size, np.uint8),
           "per_system_status": np.zeros(b.batch_size, np.int32)}
    if b.point_charge_offsets is not None:
        po = np.asarray(b.point_charge_offsets)
        v = np.asarray(b.point_charge_values)
        e = e + np.array([v[po[i]:po[i + 1]].sum() for i in range(b.batch_size)])
        out["point_charge_forces"] = 3.0 * np.asarray(b.point_charge_positions) * np.repeat(v, 3)
    if b.efields is not None:
        f = np.nan_to_num(np.asarray(b.efields).reshape(-1, 3))
        e = e + f.sum(axis=1)
        out["dipole_moments"] = (f * 2.0).ravel()
    if b.charge_response_matrix is not None:
        ro = np.asarray(b.charge_response_offsets)
        a = np.asarray(b.charge_response_matrix)
        e = e + np.array([a[ro[i]:ro[i + 1]].sum() for i in range(b.batch_size)])
        q = q + np.asarray(b.atomic_potential_shifts)
    out.update({"energies": e, "forces": 2.0 * x, "atomic_charges": q})
    return out


def with_attachments(b, seed=3):
    """Every kind of attachment on a batch: spin channels, point charges,
    fields (NaN rows: none) and charge-response blocks."""
    rng = np.random.default_rng(seed)
    B, off = b.batch_size, np.asarray(b.atom_offsets)
    na = np.diff(off)
    b.spin_channels = rng.integers(1, 3, B).astype(np.int32)
    npc = rng.integers(0, 6, B)
    b.point_charge_offsets = np.concatenate([[0], np.cumsum(npc)]).astype(np.int64)
    b.point_charge_values = rng.standard_normal(int(npc.sum()))
    b.point_charge_positions = rng.standard_normal(3 * int(npc.sum()))
    b.point_charge_gammas = np.abs(rng.standard_normal(int(npc.sum())))
    f = rng.standard_normal((B, 3)) * 1e-3
    f[rng.random(B) < 0.3] = np.nan
    b.efields = f
    b.atomic_potential_shifts = rng.standard_normal(int(off[-1]))
    b.charge_response_offsets = np.concatenate([[0], np.cumsum(na * na)]).astype(np.int64)
    b.charge_response_matrix = rng.standard_normal(int((na * na).sum()))
    return b


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


def test_shard_carries_every_attachment():
    b = with_attachments(W.config1(41))
    direct = fake_compute(b)
    shards = S.plan_shards(b, 3)
    subs = [S.shard(b, idx) for idx in shards]
    for idx, sb in zip(shards, subs):
        assert sb.batch_size == len(idx)
        assert np.array_equal(sb.spin_channels, b.spin_channels[idx])
        po, spo = b.point_charge_offsets, sb.point_charge_offsets
        for k, i in enumerate(idx):
            assert np.array_equal(sb.point_charge_values[spo[k]:spo[k + 1]],
                                  b.point_charge_values[po[i]:po[i + 1]])
            assert np.array_equal(sb.point_charge_gammas[spo[k]:spo[k + 1]],
                                  b.point_charge_gammas[po[i]:po[i + 1]])
        assert np.array_equal(sb.efields, b.efields[idx], equal_nan=True)
    back = S.scatter_back(b, shards, [fake_compute(sb) for sb in subs])
    assert set(back) == set(direct)
    for k in direct:
        assert np.array_equal(back[k], direct[k], equal_nan=True), k


def test_cost_model_counts_channels_iterations_and_the_model_basis():
    b = W.config4(12, seed=4)               # radicals: two spin channels each
    n2 = S.orbital_counts(b, S.MODEL_GFN2)
    n1 = S.orbital_counts(b, S.MODEL_GFN1)
    nh = np.add.reduceat((np.asarray(b.atomic_numbers) == 1).astype(int), b.atom_offsets[:-1])
    assert np.array_equal(n1 - n2, nh)       # GFN1 gives H a 2s shell
    c = S.predicted_cost(b)
    one = S.shard(b, np.arange(12))
    one.spin_channels = None
    assert np.allclose(c / S.predicted_cost(one), (2 * S.DEFAULT_ITERATIONS + 2) / (S.DEFAULT_ITERATIONS + 2))
    it = np.full(12, 20)
    it[5] = 250
    ci = S.predicted_cost(b, iterations=it)
    assert ci[5] / ci[4] > 5 * (n2[5] / n2[4]) ** 3
    with pytest.raises(ValueError):
        S.predicted_cost(b, iterations=[1, 2])


def test_known_iteration_counts_balance_the_real_cost():
    b = W.config1(400)
    it = np.full(400, 22)
    slow = [3, 50, 101, 207, 333, 390]
    it[slow] = 250
    world = 4
    cost = S.predicted_cost(b, iterations=it)
    shards = S.plan_shards(b, world, cost)
    loads = np.array([cost[s].sum() for s in shards])
    assert loads.max() / loads.mean() < 1.05
    # the partition that ignores the counts leaves a rank with more of the real cost
    blind = S.plan_shards(b, world)
    assert max(cost[s].sum() for s in blind) > 1.1 * loads.max()


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
        b = with_attachments(W.config1(64))
        seen = []

        def compute(sb):
            seen.append(sb.batch_size)
            return fake_compute(sb)

        whole = S.distributed_compute(b, compute)
        tmax = bench.allreduce_max(float(rank + 1), world)
        bench.barrier(world)
        direct = fake_compute(b)
        ok = all(np.array_equal(whole[k], direct[k], equal_nan=True) for k in direct)
        q.put((rank, tmax, ok, seen[0], len(S.plan_shards(b, world)[rank])))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_one_batch_with_attachments():
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
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, tmax, ok, computed, owned in got:
        assert tmax == 2.0 and ok
        assert computed == owned < 64     # each rank computed only its own shard


class _FakeLibrary:
    """Stands in for one device's context: records the systems it computed."""

    def __init__(self, device):
        self.device = device
        self.seen = []

    def make_options(self, **kw):
        return kw

    def compute(self, b, options):
        self.seen.append(b.batch_size)
        out = fake_compute(b)
        n = np.diff(np.asarray(b.atom_offsets))
        out["scc_iterations"] = (10 + (n % 7) * 30).astype(np.int32)   # some slow systems
        return out


def test_batch_calculator_spreads_one_batch_over_devices(monkeypatch):
    from xtbloom_b200 import interface
    fakes = {d: _FakeLibrary(d) for d in (0, 1, 2)}
    monkeypatch.setattr(interface, "_library", lambda d: fakes[d])
    b = W.config1(50)
    nums = [W.molecule(b, i)[0] for i in range(50)]
    pos = [W.molecule(b, i)[1] for i in range(50)]
    calc = interface.BatchCalculator("GFN2-xTB", nums, pos, device_ids=[0, 1, 2])
    r1 = calc.singlepoint()
    assert sum(f.seen[0] for f in fakes.values()) == 50 and all(f.seen[0] > 0 for f in fakes.values())
    direct = fake_compute(b)
    assert np.allclose(r1.get("energies"), direct["energies"])
    for i in range(50):
        assert np.array_equal(r1.get("charges")[i], direct["atomic_charges"][b.atom_offsets[i]:b.atom_offsets[i + 1]])
    # the second call is partitioned with the first call's iteration counts
    first = [f.seen[0] for f in fakes.values()]
    calc.singlepoint()
    second = [f.seen[1] for f in fakes.values()]
    assert sum(second) == 50
    assert calc._last_iterations is not None and len(calc._last_iterations) == 50
    assert first != second or len(set(calc._last_iterations)) == 1
    with pytest.raises(ValueError):
        interface.BatchCalculator("GFN2-xTB", nums, pos, device_ids=[0, 0])
