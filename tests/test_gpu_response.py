"""Charge response b + A q (periodic QM/MM coupling) against the reference library.

Per-atom shifts b and per-system symmetric response blocks A add
(b + A q)_A to every atom's potential in the SCC (mixed charges) and
q.b + q^T A q / 2 to the energy (raw charges); forces exclude coordinate
derivatives of the caller-owned b and A, which the result flag
FORCES_EXCLUDE_EXTERNAL_OPERATOR_DERIVATIVES reports.  Goldens:
``tests/golden/response_fixtures.json`` (reference library).
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, TOL_E, TOL_F, TOL_Q
from xtbloom_b200 import abi

pytestmark = pytest.mark.gpu


def pack(systems, asym=None):
    b = abi.ragged_from_lists([np.asarray(s["numbers"], np.int32) for s in systems],
                              [np.asarray(s["positions"]).reshape(-1, 3) for s in systems],
                              [s["charge"] for s in systems], [s["uhf"] for s in systems],
                              [s["spin_channels"] for s in systems])
    na = np.diff(b.atom_offsets)
    b.atomic_potential_shifts = np.concatenate([s["shifts"] for s in systems])
    b.charge_response_offsets = np.concatenate([[0], np.cumsum(na * na)]).astype(np.int64)
    blocks = [np.asarray(s["response"]) for s in systems]
    if asym is not None:
        blocks[asym] = blocks[asym].copy()
        blocks[asym][1] += 1e-3    # element (0, 1) only: no longer symmetric
    b.charge_response_matrix = np.concatenate(blocks)
    return b


def test_response_matches_reference(cuda_lib):
    systems = json.loads((GOLDEN / "response_fixtures.json").read_text())["systems"]
    b = pack(systems)
    out = cuda_lib.compute(b)
    assert cuda_lib.last_result_flags & 1   # forces exclude derivatives of b and A
    for i, s in enumerate(systems):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == s["status"] == 0
        assert abs(out["energies"][i] - s["energy"]) < TOL_E, s["name"]
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(s["forces"])).max() < TOL_F, s["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(s["charges"])).max() < TOL_Q, s["name"]
        assert abs(int(out["scc_iterations"][i]) - s["scc_iterations"]) <= 1


def test_nonsymmetric_response_is_rejected(cuda_lib):
    systems = json.loads((GOLDEN / "response_fixtures.json").read_text())["systems"][:2]
    b = pack(systems, asym=1)
    sentinel = {"energies": np.full(2, 7.0), "scc_iterations": np.empty(2, np.int32),
                "scc_converged": np.empty(2, np.uint8), "per_system_status": np.empty(2, np.int32)}
    with pytest.raises(abi.XtbloomError) as e:
        cuda_lib.compute(b, cuda_lib.make_options(flags=abi.COMPUTE_ENERGY), sentinel)
    assert e.value.status == abi.INVALID_ARGUMENT
    assert (sentinel["energies"] == 7.0).all()
