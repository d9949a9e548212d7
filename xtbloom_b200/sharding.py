"""Splitting one ragged batch over the GPUs of a node, and gathering it back.

Systems are independent, so a multi-GPU call is a partition of the systems
with no collective in the data path.  Each rank gets a contiguous ragged
sub-batch of its own systems; results are scattered back into system order.
Cost per system is predicted as n_AO^3 (the eigensolver term that dominates
the SCC); the partition is longest-processing-time-first greedy, which is
within 4/3 of the optimal makespan.
"""
from __future__ import annotations

import heapq
from functools import lru_cache
from pathlib import Path

import numpy as np

from .abi import RaggedBatch, ragged_from_lists


@lru_cache(maxsize=1)
def _gfn2_nao() -> np.ndarray:
    """Spherical AOs per element (index Z) of the GFN2 basis: sum over shells of 2l+1."""
    p = np.load(Path(__file__).resolve().parent / "data" / "params.npz")
    nsh, ls = p["gfn2_nshell"], p["gfn2_shell_l"]    # row Z-1
    nao = np.zeros(len(nsh) + 1, dtype=np.int64)
    for z in range(1, len(nsh) + 1):
        nao[z] = sum(2 * int(ls[z - 1, k]) + 1 for k in range(int(nsh[z - 1])))
    return nao


def predicted_cost(batch: RaggedBatch) -> np.ndarray:
    """n_AO^3 per system (float64)."""
    off = np.asarray(batch.atom_offsets, dtype=np.int64)
    nao = _gfn2_nao()[np.asarray(batch.atomic_numbers, dtype=np.int64)]
    per = np.add.reduceat(nao, off[:-1]) if len(nao) else np.zeros(0, np.int64)
    return per.astype(np.float64) ** 3


def plan_shards(batch: RaggedBatch, world: int) -> list[np.ndarray]:
    """System indices per rank (ascending within a rank), balanced by predicted cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = predicted_cost(batch)
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    owned: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        owned[r].append(int(i))
        heapq.heappush(heap, (load + float(cost[i]), r))
    return [np.asarray(sorted(o), dtype=np.int64) for o in owned]


def shard(batch: RaggedBatch, idx: np.ndarray) -> RaggedBatch:
    """The sub-batch of systems idx (host arrays), offsets rebased to zero."""
    off = np.asarray(batch.atom_offsets, dtype=np.int64)
    z = np.asarray(batch.atomic_numbers)
    x = np.asarray(batch.positions)
    nums = [z[off[i]:off[i + 1]] for i in idx]
    poss = [x[3 * off[i]:3 * off[i + 1]] for i in idx]
    return ragged_from_lists(nums, poss, np.asarray(batch.molecular_charges)[idx],
                             np.asarray(batch.unpaired_electrons)[idx])


def scatter_back(batch: RaggedBatch, shards: list[np.ndarray], results: list[dict]) -> dict:
    """Per-rank result dicts (in shard order) -> one dict in the batch's system order."""
    off = np.asarray(batch.atom_offsets, dtype=np.int64)
    B, N = batch.batch_size, batch.total_atoms
    out = {"energies": np.full(B, np.nan), "forces": np.full(3 * N, np.nan),
           "atomic_charges": np.full(N, np.nan), "scc_iterations": np.zeros(B, np.int32),
           "scc_converged": np.zeros(B, np.uint8), "per_system_status": np.zeros(B, np.int32)}
    for idx, res in zip(shards, results):
        a = 0
        for k, i in enumerate(idx):
            n = int(off[i + 1] - off[i])
            for key in ("energies", "scc_iterations", "scc_converged", "per_system_status"):
                if key in res:
                    out[key][i] = res[key][k]
            if "forces" in res:
                out["forces"][3 * off[i]:3 * off[i + 1]] = res["forces"][3 * a:3 * (a + n)]
            if "atomic_charges" in res:
                out["atomic_charges"][off[i]:off[i + 1]] = res["atomic_charges"][a:a + n]
            a += n
    return out
