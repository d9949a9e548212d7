"""Strict WARM SCC start against the reference library.

A WARM call seeds the SCC with the converged electronic state (shell charges,
atomic dipoles and quadrupoles; for unrestricted systems also the
magnetisation block) of the latest fully converged call with the same
identity, on new coordinates; every accepted call consumes that checkpoint.
A WARM request without a compatible checkpoint is rejected with
INVALID_ARGUMENT before any output is written.  The same FRESH -> WARM sequence
is run through the reference library (the oracle) and through the CUDA path.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, REF_LIB, TOL_E, TOL_F, TOL_Q, as_molecule
from xtbloom_b200 import abi, library_path
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu


def batches(fixtures, uhf, shift=0.02, seed=11):
    """Restricted fixtures plus two unrestricted radicals, and the same
    molecules displaced by N(0, shift) bohr (an MD-like next step)."""
    mols = [as_molecule(s) + (1,) for s in fixtures[:8]]
    full = W.config4(2048, seed=4)
    for c in uhf["radicals"]["systems"][:2]:
        z, x = W.molecule(full, c["index"])
        mols.append((z, x, 0.0, 1, 2))
    rng = np.random.default_rng(seed)

    def pack(ms):
        return abi.ragged_from_lists([m[0] for m in ms], [m[1] for m in ms], [m[2] for m in ms],
                                     [m[3] for m in ms], [m[4] for m in ms])
    moved = [(m[0], m[1] + rng.normal(0.0, shift, m[1].shape), m[2], m[3], m[4]) for m in mols]
    return pack(mols), pack(moved)


@pytest.fixture(scope="module")
def uhf():
    return json.loads((GOLDEN / "uhf_fixtures.json").read_text())


def fresh_then_warm(lib, b1, b2):
    one = lib.compute(b1, lib.make_options(start=abi.START_FRESH))
    two = lib.compute(b2, lib.make_options(start=abi.START_WARM))
    return one, two


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference library not built")
def test_warm_sequence_matches_reference(fixtures, uhf):
    b1, b2 = batches(fixtures, uhf)
    gpu = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=0)
    ref = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=0)
    try:
        g1, g2 = fresh_then_warm(gpu, b1, b2)
        r1, r2 = fresh_then_warm(ref, b1, b2)
        cold = gpu.compute(b2)   # FRESH on the moved geometry, for the iteration count
    finally:
        gpu.close()
        ref.close()
    assert (g2["per_system_status"] == 0).all() and (r2["per_system_status"] == 0).all()
    assert np.abs(g2["energies"] - r2["energies"]).max() < TOL_E
    assert np.abs(g2["forces"] - r2["forces"]).max() < TOL_F
    assert np.abs(g2["atomic_charges"] - r2["atomic_charges"]).max() < TOL_Q
    assert np.abs(g2["scc_iterations"].astype(int) - r2["scc_iterations"]).max() <= 1
    # the warm start needs fewer iterations than a fresh start on the same geometry
    assert g2["scc_iterations"].sum() < cold["scc_iterations"].sum()
    assert np.abs(g2["energies"] - cold["energies"]).max() < TOL_E


def test_warm_requires_a_compatible_converged_call(fixtures, uhf):
    b1, b2 = batches(fixtures, uhf)
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=0)
    try:
        warm = lib.make_options(start=abi.START_WARM)
        sentinel = {"energies": np.full(b1.batch_size, 7.0)}
        with pytest.raises(abi.XtbloomError) as e:   # no checkpoint yet
            lib.compute(b1, warm, sentinel)
        assert e.value.status == abi.INVALID_ARGUMENT
        assert (sentinel["energies"] == 7.0).all()   # nothing written
        lib.compute(b1)                               # FRESH, fully converged: checkpoint
        charged = abi.ragged_from_lists(
            [b1.atomic_numbers[b1.atom_offsets[i]:b1.atom_offsets[i + 1]] for i in range(b1.batch_size)],
            [b1.positions[3 * b1.atom_offsets[i]:3 * b1.atom_offsets[i + 1]] for i in range(b1.batch_size)],
            b1.molecular_charges + 2.0, b1.unpaired_electrons, b1.spin_channels)
        with pytest.raises(abi.XtbloomError) as e:   # other molecular charges
            lib.compute(charged, warm, sentinel)
        assert e.value.status == abi.INVALID_ARGUMENT
        assert (sentinel["energies"] == 7.0).all()
        with pytest.raises(abi.XtbloomError):         # other SCC settings
            lib.compute(b2, lib.make_options(start=abi.START_WARM, ctol=2e-6))
        out = lib.compute(b2, warm)                   # rejected calls leave the checkpoint
        assert (out["per_system_status"] == 0).all()
        lib.compute(b1, lib.make_options(max_iter=2))  # accepted, not converged: consumed
        with pytest.raises(abi.XtbloomError):
            lib.compute(b1, lib.make_options(start=abi.START_WARM, max_iter=2))
        with pytest.raises(abi.XtbloomError):
            lib.compute(b1, warm)
    finally:
        lib.close()
