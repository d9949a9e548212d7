"""Unrestricted (two spin channel) GFN2 against the reference library.

Spin polarisation: alpha and beta Hamiltonians H0 - S (v +- v_mag)/2 with the
spin potential v_mag = W m of the atom-local tblite couplings, separate
eigensolves and Fermi occupations per channel, the magnetisation block in the
Broyden vector, E_spin = m W m / 2, and the magnetisation term of the
analytic forces.  Goldens: ``tests/golden/uhf_fixtures.json`` (reference
library, spin_channels = 2).
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, TOL_E, TOL_F, TOL_Q, as_molecule
from xtbloom_b200 import abi
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uhf():
    return json.loads((GOLDEN / "uhf_fixtures.json").read_text())


# Radicals whose SCC needs more than this many Broyden iterations follow a
# trajectory that rounding differences (summation order) move: both runs stop
# somewhere inside the convergence gate (charge residual rms < 1e-6, |dF| < 1e-8)
# after different iteration counts.  Such a run can only be held to the fixed
# point: its forces and charges lie no farther from the reference's than the
# reference's own default-gate result lies from its fixed point (charge
# tolerance 1e-10, the ``tight_*`` goldens), plus the public tolerance; the
# energy (variational) is compared at 1e-6 Eh, the iteration count is not.
# ``test_radicals_at_the_fixed_point`` compares every output at the public
# tolerances with both sides converged to the fixed point.
SLOW = 60


def check(out, b, i, ref):
    a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
    assert out["per_system_status"][i] == ref["status"], (i, out["per_system_status"][i], ref["status"])
    if ref["status"] != 0:
        assert np.isnan(out["energies"][i])
        return
    f, q = out["forces"][3 * a0:3 * a1], out["atomic_charges"][a0:a1]
    rf, rq = np.asarray(ref["forces"]), np.asarray(ref["charges"])
    tf, tq = TOL_F, TOL_Q
    slow = ref["scc_iterations"] > SLOW
    if slow:
        tf += np.abs(rf - np.asarray(ref["tight_forces"])).max()
        tq += np.abs(rq - np.asarray(ref["tight_charges"])).max()
    assert abs(out["energies"][i] - ref["energy"]) < TOL_E, (i, out["energies"][i], ref["energy"])
    assert np.abs(f - rf).max() < tf, i
    assert np.abs(q - rq).max() < tq, i
    if not slow:
        assert abs(int(out["scc_iterations"][i]) - ref["scc_iterations"]) <= 1, \
            (i, out["scc_iterations"][i], ref["scc_iterations"])


def test_oh_radical(cuda_lib, uhf):
    r = uhf["oh_radical"]
    b = abi.ragged_from_lists([np.asarray(r["numbers"], np.int32)],
                              [np.asarray(r["positions"]).reshape(-1, 3)], [0.0], [1], [2])
    out = cuda_lib.compute(b)
    check(out, b, 0, r)
    # the tblite UHF trace's final charges (its SCC stops at a residual of 1e-5)
    assert np.abs(out["atomic_charges"] - np.asarray(r["tblite_final_charges"])).max() < 2e-5


def test_radicals_in_one_batch(cuda_lib, uhf):
    cases = uhf["radicals"]["systems"]
    full = W.config4(2048, seed=4)
    b = W.subset(full, [c["index"] for c in cases])
    out = cuda_lib.compute(b)
    for i, c in enumerate(cases):
        check(out, b, i, c)
    assert sum(c["scc_iterations"] <= SLOW for c in cases) >= 8


def test_restricted_and_unrestricted_share_a_batch(cuda_lib, uhf, fixtures):
    """Restricted fixtures and unrestricted radicals interleaved in one call."""
    rad = uhf["radicals"]["systems"][:4]
    full = W.config4(2048, seed=4)
    mols = []
    refs = []
    for k, s in enumerate(fixtures[:6]):
        z, x, q, u = as_molecule(s)
        mols.append((z, x, q, u, 1))
        refs.append(s)
        if k < len(rad):
            zr, xr = W.molecule(full, rad[k]["index"])
            mols.append((zr, xr, 0.0, 1, 2))
            refs.append(rad[k])
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols], [m[2] for m in mols],
                              [m[3] for m in mols], [m[4] for m in mols])
    out = cuda_lib.compute(b)
    for i, r in enumerate(refs):
        check(out, b, i, r)


def test_radicals_at_the_fixed_point(cuda_lib, uhf):
    """Both sides converged to the fixed point (charge tolerance 1e-10): every
    output of every converging radical at the public tolerances."""
    cases = [c for c in uhf["radicals"]["systems"] if c["tight_status"] == 0]
    full = W.config4(2048, seed=4)
    b = W.subset(full, [c["index"] for c in cases])
    out = cuda_lib.compute(b, cuda_lib.make_options(ctol=1e-10, etol=1e-13))
    assert len(cases) >= 10
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, c["index"]
        assert abs(out["energies"][i] - c["tight_energy"]) < TOL_E, c["index"]
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["tight_forces"])).max() < TOL_F, c["index"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["tight_charges"])).max() < TOL_Q, c["index"]
