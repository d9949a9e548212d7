"""Uniform external electric field and dipole moments against the reference library.

The field enters as the atomic potential -E.R_A and the dipole potential -E
of every atom in the SCC, the energy -E.(sum_A q_A R_A + d_A) of the raw
multipoles and the explicit force q_A E; dipole moments are
sum_A q_A R_A + d_A.  Goldens: ``tests/golden/field_fixtures.json`` (reference
library on restricted fixtures and unrestricted radicals, with and without a
field; the water case is the reference's ``water_efield`` conformance input,
whose energy the reference library reproduces from tblite).
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, TOL_E, TOL_F, TOL_Q
from xtbloom_b200 import abi

pytestmark = pytest.mark.gpu

FLAGS = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES | abi.COMPUTE_CHARGES | abi.COMPUTE_DIPOLES


@pytest.fixture(scope="module")
def gold():
    return json.loads((GOLDEN / "field_fixtures.json").read_text())


def run(lib, systems, with_field=True):
    b = abi.ragged_from_lists([np.asarray(s["numbers"], np.int32) for s in systems],
                              [np.asarray(s["positions"]).reshape(-1, 3) for s in systems],
                              [s["charge"] for s in systems], [s["uhf"] for s in systems],
                              [s["spin_channels"] for s in systems])
    if with_field:
        b.efields = np.array([s["field"] if s["field"] is not None else [np.nan] * 3 for s in systems])
    nb, na = b.batch_size, b.total_atoms
    out = {"energies": np.empty(nb), "forces": np.empty(3 * na), "atomic_charges": np.empty(na),
           "dipole_moments": np.empty(3 * nb), "scc_iterations": np.empty(nb, np.int32),
           "scc_converged": np.empty(nb, np.uint8), "per_system_status": np.empty(nb, np.int32)}
    return b, lib.compute(b, lib.make_options(flags=FLAGS), out)


def test_field_and_dipoles_match_reference(cuda_lib, gold):
    # one ragged batch: systems with a field next to systems without one
    systems = gold["systems"]
    b, out = run(cuda_lib, systems)
    assert cuda_lib.last_result_flags & (1 << 4)   # dipole moments published
    for i, s in enumerate(systems):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == s["status"] == 0
        assert abs(out["energies"][i] - s["energy"]) < TOL_E, (s["name"], s["case"])
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(s["forces"])).max() < TOL_F, s["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(s["charges"])).max() < TOL_Q, s["name"]
        assert np.abs(out["dipole_moments"][3 * i:3 * i + 3] - np.asarray(s["dipole"])).max() < 1e-5
        assert abs(int(out["scc_iterations"][i]) - s["scc_iterations"]) <= 1
    water = next(i for i, s in enumerate(systems) if s["name"] == "water_efield" and s["case"] == "field")
    assert abs(out["energies"][water] - gold["tblite_water_efield_energy"]) < 5e-7


def test_field_force_is_energy_derivative(cuda_lib, gold):
    """Central differences (h = 1e-4 bohr) of the energy in a field."""
    s = next(x for x in gold["systems"] if x["name"] == "water_efield" and x["case"] == "field")
    base = np.asarray(s["positions"]).reshape(-1, 3)
    _, out = run(cuda_lib, [s])
    h = 1e-4
    for atom in range(3):
        for c in range(3):
            e = []
            for sg in (+1, -1):
                x = base.copy()
                x[atom, c] += sg * h
                _, o = run(cuda_lib, [dict(s, positions=x.reshape(-1).tolist())])
                e.append(o["energies"][0])
            assert abs(-(e[0] - e[1]) / (2 * h) - out["forces"][3 * atom + c]) < 2e-6


def test_unknown_and_duplicate_attachments_are_refused(cuda_lib, gold):
    s = gold["systems"][0]
    b = abi.ragged_from_lists([np.asarray(s["numbers"], np.int32)],
                              [np.asarray(s["positions"]).reshape(-1, 3)])
    batch = cuda_lib.make_batch(b)
    desc = (abi.Interaction * 2)(abi.Interaction(abi.INTERACTION_ELECTRIC_FIELD, 0, 0, 0, 32),
                                 abi.Interaction(abi.INTERACTION_ELECTRIC_FIELD, 0, 0, 32, 32))
    payload = np.zeros(64, np.uint8)
    payload[0] = payload[32] = 1   # block_version 1, zero fields
    import ctypes as C
    batch.total_interactions = 2
    batch.interaction_descriptors = abi.ConstBuffer(C.addressof(desc), C.sizeof(desc), abi.MEMORY_HOST, 0)
    batch.interaction_payload = abi.ConstBuffer(payload.ctypes.data, payload.nbytes, abi.MEMORY_HOST, 0)
    outs = {"energies": np.empty(1), "scc_iterations": np.empty(1, np.int32),
            "scc_converged": np.empty(1, np.uint8), "per_system_status": np.empty(1, np.int32)}
    res = cuda_lib.make_result(outs)
    opts = cuda_lib.make_options(flags=abi.COMPUTE_ENERGY)
    st = cuda_lib.lib.xtbloom_compute(cuda_lib.ctx, C.byref(batch), C.byref(opts), C.byref(res))
    assert st == abi.INVALID_ARGUMENT                     # two fields on one system
    desc[1] = abi.Interaction(0x0201, 0, 0, 32, 32)       # a reserved tag (solvation)
    st = cuda_lib.lib.xtbloom_compute(cuda_lib.ctx, C.byref(batch), C.byref(opts), C.byref(res))
    assert st == abi.NOT_IMPLEMENTED
