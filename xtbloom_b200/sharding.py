"""Splitting one ragged batch over the GPUs of a node, and gathering it back.

Systems are independent, so a multi-GPU call is a partition of the systems
with no collective in the data path.  Each rank gets a contiguous ragged
sub-batch of its own systems (with their point charges, field and
charge-response attachments); results are scattered back into system order.

Cost model.  One SCC iteration of a system costs about n_AO^3 per spin
channel (the eigensolver and the basis-transform products dominate), and a
system runs as many iterations as it needs to meet the gate, up to the cap.
Before anything is known every system is charged the same iteration count;
once a previous call on the same systems reported its ``scc_iterations``
(an MD loop, a scan, a plan reused with new positions), those counts replace
it, so a system that ran to the cap -- a few such systems are a quarter of a
4096-system step -- weighs as much as the hundred systems it costs.  The
partition is longest-processing-time-first greedy (within 4/3 of the
optimal makespan), so the heaviest systems land on different ranks first.
"""
from __future__ import annotations

import heapq
from functools import lru_cache
from pathlib import Path
from typing import Callable, Sequence

import numpy as np

from .abi import MODEL_GFN1, MODEL_GFN2, RaggedBatch

# Iterations charged to a system whose count is not known yet.
DEFAULT_ITERATIONS = 24.0

_RESULT_PER_SYSTEM = {"energies": 1, "scc_iterations": 1, "scc_converged": 1,
                      "per_system_status": 1, "dipole_moments": 3, "quadrupole_moments": 6}
_RESULT_PER_ATOM = {"forces": 3, "atomic_charges": 1, "spin_populations": 1}


@lru_cache(maxsize=2)
def _nao_table(model: int) -> np.ndarray:
    """Spherical AOs per element (index Z) of a model's basis: sum over shells of 2l+1."""
    p = np.load(Path(__file__).resolve().parent / "data" / "params.npz")
    key = "gfn1" if model == MODEL_GFN1 else "gfn2"
    nsh, ls = p[f"{key}_nshell"], p[f"{key}_shell_l"]    # row Z-1
    nao = np.zeros(len(nsh) + 1, dtype=np.int64)
    for z in range(1, len(nsh) + 1):
        nao[z] = sum(2 * int(ls[z - 1, k]) + 1 for k in range(int(nsh[z - 1])))
    return nao


def orbital_counts(batch: RaggedBatch, model: int = MODEL_GFN2) -> np.ndarray:
    """AOs per system of the batch in the model's basis."""
    off = np.asarray(batch.atom_offsets, dtype=np.int64)
    nao = _nao_table(model)[np.asarray(batch.atomic_numbers, dtype=np.int64)]
    if batch.batch_size == 0:
        return np.zeros(0, np.int64)
    csum = np.concatenate([[0], np.cumsum(nao)])
    return csum[off[1:]] - csum[off[:-1]]


def predicted_cost(batch: RaggedBatch, model: int = MODEL_GFN2,
                   iterations: Sequence[int] | None = None) -> np.ndarray:
    """Predicted device time per system (arbitrary units): n_AO^3 per spin
    channel and iteration.  ``iterations``: SCC iterations reported for these
    systems by an earlier call (``scc_iterations``), else the default count."""
    n = orbital_counts(batch, model).astype(np.float64)
    channels = np.ones_like(n)
    if batch.spin_channels is not None:
        channels = np.asarray(batch.spin_channels, dtype=np.float64).reshape(-1)
    if iterations is None:
        it = np.full_like(n, DEFAULT_ITERATIONS)
    else:
        it = np.asarray(iterations, dtype=np.float64).reshape(-1)
        if len(it) != len(n):
            raise ValueError("iterations must have one entry per system")
        it = np.where(it > 0, it, DEFAULT_ITERATIONS)
    # setup, Löwdin and forces: about two iterations' worth per system
    return n ** 3 * (channels * it + 2.0)


def plan_shards(batch: RaggedBatch, world: int, cost: np.ndarray | None = None) -> list[np.ndarray]:
    """System indices per rank (ascending within a rank), balanced by cost
    (``predicted_cost(batch)`` unless given)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = predicted_cost(batch) if cost is None else np.asarray(cost, dtype=np.float64)
    if len(cost) != batch.batch_size:
        raise ValueError("cost must have one entry per system")
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    owned: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        owned[r].append(int(i))
        heapq.heappush(heap, (load + float(cost[i]), r))
    return [np.asarray(sorted(o), dtype=np.int64) for o in owned]


def _segments(values: np.ndarray, off: np.ndarray, idx: np.ndarray, width: int) -> tuple[np.ndarray, np.ndarray]:
    """Concatenated rows off[i]..off[i+1] (each `width` wide) of systems idx,
    with the rebased offsets."""
    counts = (off[idx + 1] - off[idx]).astype(np.int64)
    new_off = np.zeros(len(idx) + 1, np.int64)
    new_off[1:] = np.cumsum(counts)
    if len(idx) == 0 or new_off[-1] == 0:
        return values[:0].copy(), new_off
    parts = [values[width * off[i]:width * off[i + 1]] for i in idx]
    return np.ascontiguousarray(np.concatenate(parts)), new_off


def shard(batch: RaggedBatch, idx: np.ndarray) -> RaggedBatch:
    """The sub-batch of systems idx (host arrays), offsets rebased to zero,
    with every attachment of those systems: spin channels, point charges,
    fields and charge-response blocks."""
    idx = np.asarray(idx, dtype=np.int64)
    off = np.asarray(batch.atom_offsets, dtype=np.int64)
    z, new_off = _segments(np.asarray(batch.atomic_numbers), off, idx, 1)
    x, _ = _segments(np.asarray(batch.positions, dtype=np.float64).reshape(-1), off, idx, 3)
    sub = RaggedBatch(
        atom_offsets=new_off,
        atomic_numbers=np.ascontiguousarray(z.astype(np.int32)),
        positions=x,
        molecular_charges=np.ascontiguousarray(np.asarray(batch.molecular_charges, float)[idx]),
        unpaired_electrons=np.ascontiguousarray(np.asarray(batch.unpaired_electrons, np.int32)[idx]),
    )
    if batch.spin_channels is not None:
        sub.spin_channels = np.ascontiguousarray(np.asarray(batch.spin_channels, np.int32)[idx])
    if batch.point_charge_offsets is not None:
        poff = np.asarray(batch.point_charge_offsets, dtype=np.int64)
        sub.point_charge_values, sub.point_charge_offsets = _segments(
            np.asarray(batch.point_charge_values, float), poff, idx, 1)
        sub.point_charge_positions, _ = _segments(
            np.asarray(batch.point_charge_positions, float).reshape(-1), poff, idx, 3)
        if batch.point_charge_gammas is not None:
            sub.point_charge_gammas, _ = _segments(np.asarray(batch.point_charge_gammas, float), poff, idx, 1)
    if batch.efields is not None:
        sub.efields = np.ascontiguousarray(np.asarray(batch.efields, float).reshape(-1, 3)[idx])
    if batch.charge_response_matrix is not None:
        sub.atomic_potential_shifts, _ = _segments(np.asarray(batch.atomic_potential_shifts, float), off, idx, 1)
        roff = np.asarray(batch.charge_response_offsets, dtype=np.int64)
        sub.charge_response_matrix, sub.charge_response_offsets = _segments(
            np.asarray(batch.charge_response_matrix, float), roff, idx, 1)
    return sub


def scatter_back(batch: RaggedBatch, shards: list[np.ndarray], results: list[dict]) -> dict:
    """Per-rank result dicts (in shard order) -> one dict in the batch's system
    order.  Outputs that no shard returned are absent; systems of a shard that
    returned nothing keep NaN (status 0 stays only where a shard reported it)."""
    off = np.asarray(batch.atom_offsets, dtype=np.int64)
    B, N = batch.batch_size, batch.total_atoms
    poff = None if batch.point_charge_offsets is None else np.asarray(batch.point_charge_offsets, np.int64)
    keys = set().union(*[r.keys() for r in results]) if results else set()
    out: dict = {}
    for key in keys:
        ref = next(r[key] for r in results if key in r)
        dt = np.asarray(ref).dtype
        if key in _RESULT_PER_SYSTEM:
            size = B * _RESULT_PER_SYSTEM[key]
        elif key in _RESULT_PER_ATOM:
            size = N * _RESULT_PER_ATOM[key]
        elif key == "point_charge_forces" and poff is not None:
            size = 3 * int(poff[-1])
        else:
            continue
        fill = np.nan if np.issubdtype(dt, np.floating) else 0
        out[key] = np.full(size, fill, dtype=dt)
    for idx, res in zip(shards, results):
        idx = np.asarray(idx, dtype=np.int64)
        for key, w in _RESULT_PER_SYSTEM.items():
            if key in res and key in out:
                out[key].reshape(-1, w)[idx] = np.asarray(res[key]).reshape(-1, w)
        counts = off[idx + 1] - off[idx]
        local = np.concatenate([[0], np.cumsum(counts)])
        for key, w in _RESULT_PER_ATOM.items():
            if key in res and key in out:
                src = np.asarray(res[key]).reshape(-1, w)
                dst = out[key].reshape(-1, w)
                for k, i in enumerate(idx):
                    dst[off[i]:off[i + 1]] = src[local[k]:local[k + 1]]
        if "point_charge_forces" in res and "point_charge_forces" in out:
            pc = poff[idx + 1] - poff[idx]
            plocal = np.concatenate([[0], np.cumsum(pc)])
            src = np.asarray(res["point_charge_forces"]).reshape(-1, 3)
            dst = out["point_charge_forces"].reshape(-1, 3)
            for k, i in enumerate(idx):
                dst[poff[i]:poff[i + 1]] = src[plocal[k]:plocal[k + 1]]
    return out


def distributed_compute(batch: RaggedBatch, compute: Callable[[RaggedBatch], dict],
                        group=None, cost: np.ndarray | None = None) -> dict:
    """One batch over the ranks of a ``torch.distributed`` group: every rank
    computes its own shard with ``compute`` (this rank's library context on
    this rank's GPU) and receives the whole result in system order.  The only
    exchange is one object all-gather of the shards' host results after the
    computes; nothing crosses ranks inside a compute."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shards = plan_shards(batch, world, cost)
    mine = compute(shard(batch, shards[rank]))
    mine = {k: np.asarray(v) for k, v in mine.items()}
    gathered: list = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    return scatter_back(batch, shards, gathered)


def threaded_compute(batch: RaggedBatch, computes: Sequence[Callable[[RaggedBatch], dict]],
                     cost: np.ndarray | None = None) -> dict:
    """One batch over several contexts of one process (one per GPU): the
    shards run concurrently on threads (each call releases the interpreter
    lock while the library works) and are scattered back in system order."""
    from concurrent.futures import ThreadPoolExecutor
    shards = plan_shards(batch, len(computes), cost)
    subs = [shard(batch, s) for s in shards]
    with ThreadPoolExecutor(max_workers=len(computes)) as ex:
        futs = [ex.submit(fn, sb) for fn, sb in zip(computes, subs)]
        results = [f.result() for f in futs]
    return scatter_back(batch, shards, results)


__all__ = ["DEFAULT_ITERATIONS", "orbital_counts", "predicted_cost", "plan_shards", "shard",
           "scatter_back", "distributed_compute", "threaded_compute", "MODEL_GFN1", "MODEL_GFN2"]
