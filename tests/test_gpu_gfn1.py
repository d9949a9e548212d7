"""GFN1-xTB on the CUDA path against the reference.

GFN1 (model/gfn1/ of the reference): an H 1s+2s basis with the legacy STO-6G
4s/4p rows, the exponential coordination number, its own H0 shell-pair
scaling (valence/polarisation rules, element-pair kpair, electronegativity
factor), harmonic-mean ES2 hardness, atom-resolved third order, D3(BJ)
dispersion, the halogen-bond correction, and (for radicals) tblite spin
polarisation.  Goldens: ``tests/golden/gfn1_fixtures.json`` (made by
``tests/golden/make_gfn1.py``): the reference's committed tblite/xTB GFN1
conformance values and the reference library's own outputs.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, REF_LIB, TOL_E, TOL_F, TOL_Q
from xtbloom_b200 import abi
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gfn1():
    return json.loads((GOLDEN / "gfn1_fixtures.json").read_text())


def batch_of(cases):
    return abi.ragged_from_lists([np.asarray(c["numbers"], np.int32) for c in cases],
                                 [np.asarray(c["positions"]).reshape(-1, 3) for c in cases],
                                 [c["charge"] for c in cases], [c["uhf"] for c in cases],
                                 [c.get("spin_channels", 1) for c in cases])


def gfn1_options(lib, **kw):
    return lib.make_options(model=abi.MODEL_GFN1, **kw)


def test_gfn1_tblite_goldens(cuda_lib, gfn1):
    """The reference's committed GFN1 conformance values (xTB 6.7.1 / tblite,
    produced with a tight SCC), at their tolerance of 5e-7 (H3+, ketene,
    Ne-Na-Cl, SiF5-, OH radical, a halogen bond), with the SCC converged to
    charge tolerance 1e-10."""
    cases = gfn1["tblite"]
    b = batch_of(cases)
    out = cuda_lib.compute(b, gfn1_options(cuda_lib, ctol=1e-10, etol=1e-13))
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, c["name"]
        assert abs(out["energies"][i] - c["energy"]) < 5e-7, (c["name"], out["energies"][i], c["energy"])
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["forces"])).max() < 5e-7, c["name"]
        if c["charges"] is not None:
            assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["charges"])).max() < 5e-7, c["name"]


def test_gfn1_reference_fixtures_in_one_batch(cuda_lib, gfn1):
    """Conformance molecules, hetero-alkane chains and spin-polarised radicals
    (with Cl/Br) in one ragged GFN1 batch, against the reference library.
    Systems that converge within 60 iterations are compared with the
    reference at the default SCC settings; slower ones, whose result anywhere
    inside the gate depends on the trajectory, with the reference's fixed point
    (no farther than the reference itself is from it, plus the tolerance)."""
    cases = [c for c in gfn1["reference"] if c["status"] == 0 and c["tight_status"] == 0]
    assert len(cases) >= 20
    b = batch_of(cases)
    out = cuda_lib.compute(b, gfn1_options(cuda_lib))
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, c["name"]
        assert abs(out["energies"][i] - c["energy"]) < TOL_E, (c["name"], out["energies"][i], c["energy"])
        f, q = out["forces"][3 * a0:3 * a1], out["atomic_charges"][a0:a1]
        if c["scc_iterations"] <= 60:
            assert np.abs(f - np.asarray(c["forces"])).max() < TOL_F, c["name"]
            assert np.abs(q - np.asarray(c["charges"])).max() < TOL_Q, c["name"]
            assert abs(int(out["scc_iterations"][i]) - c["scc_iterations"]) <= 1, c["name"]
        else:
            gate_f = np.abs(np.asarray(c["forces"]) - np.asarray(c["tight_forces"])).max()
            gate_q = np.abs(np.asarray(c["charges"]) - np.asarray(c["tight_charges"])).max()
            assert np.abs(f - np.asarray(c["tight_forces"])).max() < gate_f + TOL_F, c["name"]
            assert np.abs(q - np.asarray(c["tight_charges"])).max() < gate_q + TOL_Q, c["name"]


def test_gfn1_fixed_point_matches_tight_reference(cuda_lib, gfn1):
    """Converged to the fixed point on both sides (charge tolerance 1e-10):
    every output at the public tolerances, slow radicals included."""
    cases = [c for c in gfn1["reference"] if c["tight_status"] == 0]
    b = batch_of(cases)
    out = cuda_lib.compute(b, gfn1_options(cuda_lib, ctol=1e-10, etol=1e-13))
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        if out["per_system_status"][i] != 0:
            continue   # a chaotic trajectory may not reach the tight gate here
        assert abs(out["energies"][i] - c["tight_energy"]) < TOL_E, c["name"]
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["tight_forces"])).max() < TOL_F, c["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["tight_charges"])).max() < TOL_Q, c["name"]


def test_gfn1_finite_difference_forces(cuda_lib):
    """Central differences (h = 1e-4 bohr) of GFN1 energies on a brominated
    radical (D3, spin polarisation, 4s/4p legacy basis) and on the halogen-bond
    golden (halogen-bond correction) match the analytic forces."""
    b4 = W.config4(2048, seed=4)
    idx = next(i for i in range(2048) if np.isin(W.molecule(b4, i)[0], (35,)).any()
               and len(W.molecule(b4, i)[0]) < 20)
    z, x = W.molecule(b4, idx)
    h = 1e-4
    mols = [(z, x)]
    atoms = list(range(len(z)))[:6]
    for a in atoms:
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, c] += h
            xm[a, c] -= h
            mols += [(z, xp), (z, xm)]
    n = len(mols)
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols], [0.0] * n, [1] * n, [2] * n)
    out = cuda_lib.compute(b, gfn1_options(cuda_lib, ctol=1e-10, etol=1e-12))
    assert (out["per_system_status"] == 0).all()
    e = out["energies"]
    fd = -(e[1::2] - e[2::2]) / (2 * h)
    assert np.abs(fd - out["forces"][:3 * len(atoms)]).max() < 1e-5


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference library not built")
def test_gfn1_live_reference_on_radical_workload(cuda_lib):
    """24 radicals of the 2048-radical workload (12 with Cl/Br), two spin
    channels, against the reference library run live.

    Radicals that converge within 60 iterations follow the reference's path:
    every output at the public tolerances at the default settings, and at the
    fixed point (charge tolerance 1e-10).  Slower ones follow a trajectory
    that rounding moves, and an open-shell SCC can have more than one
    solution: such a system is compared at the fixed point when both sides
    reach the same one; at most one of the sample may settle on another
    solution, which must then be a converged fixed point of its own (default
    and tight results agree), and at most three may end on the other side of
    the iteration cap."""
    full = W.config4(2048, seed=4)
    halo = [i for i in range(2048) if np.isin(W.molecule(full, i)[0], (17, 35)).any()]
    plain = [i for i in range(2048) if i not in set(halo)]
    rng = np.random.default_rng(11)
    idx = np.sort(np.concatenate([rng.choice(halo, 12, replace=False), rng.choice(plain, 12, replace=False)]))
    b = W.subset(full, idx)
    ref = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=0)
    r_t = ref.compute(b, ref.make_options(model=abi.MODEL_GFN1, ctol=1e-10, etol=1e-13))
    r_d = ref.compute(b, ref.make_options(model=abi.MODEL_GFN1))
    out = cuda_lib.compute(b, gfn1_options(cuda_lib))
    out_t = cuda_lib.compute(b, gfn1_options(cuda_lib, ctol=1e-10, etol=1e-13))
    o = b.atom_offsets
    fast = (r_d["per_system_status"] == 0) & (r_d["scc_iterations"] <= 60)
    assert fast.sum() >= 12
    assert (out["per_system_status"][fast] == 0).all()
    # a trajectory of more than 60 iterations can end either side of the
    # 250-iteration cap; at most three of the sample may differ in status
    assert np.sum((out["per_system_status"] == 0) != (r_d["per_system_status"] == 0)) <= 3
    other_solution = 0
    for i in np.where((r_d["per_system_status"] == 0) & (out["per_system_status"] == 0))[0]:
        sl3, sl = slice(3 * o[i], 3 * o[i + 1]), slice(o[i], o[i + 1])
        if fast[i]:
            assert abs(out["energies"][i] - r_d["energies"][i]) < TOL_E, i
            assert np.abs(out["forces"][sl3] - r_d["forces"][sl3]).max() < TOL_F, i
            assert np.abs(out["atomic_charges"][sl] - r_d["atomic_charges"][sl]).max() < TOL_Q, i
            assert abs(int(out["scc_iterations"][i]) - int(r_d["scc_iterations"][i])) <= 1, i
        if out_t["per_system_status"][i] != 0 or r_t["per_system_status"][i] != 0:
            assert not fast[i], i
            continue
        if abs(out_t["energies"][i] - r_t["energies"][i]) < TOL_E:
            assert np.abs(out_t["forces"][sl3] - r_t["forces"][sl3]).max() < TOL_F, i
            assert np.abs(out_t["atomic_charges"][sl] - r_t["atomic_charges"][sl]).max() < TOL_Q, i
        else:
            assert not fast[i], i
            other_solution += 1
            assert abs(out["energies"][i] - out_t["energies"][i]) < TOL_E, i
    assert other_solution <= 1


def pc_batch(cases):
    b = batch_of(cases)
    counts = [len(c["pc_charges"]) for c in cases]
    b.point_charge_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    b.point_charge_positions = np.concatenate([np.asarray(c["pc_positions"], float) for c in cases])
    b.point_charge_values = np.concatenate([np.asarray(c["pc_charges"], float) for c in cases])
    b.point_charge_gammas = np.concatenate([np.asarray(c["pc_gammas"], float) for c in cases])
    return b


PC_FLAGS = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES | abi.COMPUTE_CHARGES | abi.COMPUTE_POINT_CHARGE_FORCES


def test_gfn1_qmmm_goldens(cuda_lib, gfn1):
    """The reference's GFN1 QM/MM goldens (xTB 6.7.1: water dimer in six point
    charges with GFN1 hardnesses and with gamma = 999; harmonic-mean softening
    of the shell-charge coupling) at 5e-7, point-charge forces included."""
    cases = gfn1["tblite_qmmm"]
    assert len(cases) == 2
    b = pc_batch(cases)
    out = cuda_lib.compute(b, gfn1_options(cuda_lib, flags=PC_FLAGS, ctol=1e-10, etol=1e-13))
    po = b.point_charge_offsets
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, c["name"]
        assert abs(out["energies"][i] - c["energy"]) < 5e-7, (c["name"], out["energies"][i], c["energy"])
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["forces"]).ravel()).max() < 5e-7, c["name"]
        pcf = out["point_charge_forces"][3 * po[i]:3 * po[i + 1]]
        assert np.abs(pcf - np.asarray(c["point_charge_forces"]).ravel()).max() < 5e-7, c["name"]
        if c["charges"] is not None:
            assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["charges"])).max() < 5e-7, c["name"]


def test_gfn1_point_charges_against_reference(cuda_lib, gfn1):
    """GFN1 chains, radicals and the QM/MM waters in point-charge shells, one
    ragged batch, against the reference library at the default settings
    (slow systems: within the reference's own distance from its fixed point)."""
    cases = [c for c in gfn1["reference_pc"] if c["status"] == 0]
    assert len(cases) >= 6
    b = pc_batch(cases)
    out = cuda_lib.compute(b, gfn1_options(cuda_lib, flags=PC_FLAGS))
    po = b.point_charge_offsets
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, c["name"]
        assert abs(out["energies"][i] - c["energy"]) < TOL_E, (c["name"], out["energies"][i], c["energy"])
        slack_f = slack_q = 0.0
        if c["scc_iterations"] > 60:
            slack_f = np.abs(np.asarray(c["forces"]) - np.asarray(c["tight_forces"])).max()
            slack_q = np.abs(np.asarray(c["charges"]) - np.asarray(c["tight_charges"])).max()
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["forces"])).max() < TOL_F + slack_f, c["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["charges"])).max() < TOL_Q + slack_q, c["name"]
        pcf = out["point_charge_forces"][3 * po[i]:3 * po[i + 1]]
        assert np.abs(pcf - np.asarray(c["point_charge_forces"])).max() < TOL_F + slack_f, c["name"]


def test_gfn1_charge_response_against_reference(cuda_lib, gfn1):
    """GFN1 with the charge response b + A q, against the reference library."""
    cases = [c for c in gfn1["reference_response"] if c["status"] == 0]
    assert len(cases) >= 4
    b = batch_of(cases)
    na = np.diff(b.atom_offsets)
    b.atomic_potential_shifts = np.concatenate([np.asarray(c["shifts"]) for c in cases])
    b.charge_response_offsets = np.concatenate([[0], np.cumsum(na * na)]).astype(np.int64)
    b.charge_response_matrix = np.concatenate([np.asarray(c["response"]) for c in cases])
    out = cuda_lib.compute(b, gfn1_options(cuda_lib))
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, c["name"]
        assert abs(out["energies"][i] - c["energy"]) < TOL_E, (c["name"], out["energies"][i], c["energy"])
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["forces"])).max() < TOL_F, c["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["charges"])).max() < TOL_Q, c["name"]


def test_gfn1_fields_and_dipoles_are_not_implemented(cuda_lib, gfn1):
    """As in the reference (src/runtime/validation.cpp:1428-1437): GFN1 refuses
    interaction attachments and the dipole publication before any output."""
    cases = gfn1["tblite"][:2]
    b = batch_of(cases)
    with pytest.raises(abi.XtbloomError) as e:
        cuda_lib.compute(b, gfn1_options(cuda_lib, flags=abi.COMPUTE_ENERGY | abi.COMPUTE_DIPOLES))
    assert e.value.status == abi.NOT_IMPLEMENTED
    b.efields = np.array([[0.0, 0.0, 1e-3], [np.nan] * 3])
    with pytest.raises(abi.XtbloomError) as e:
        cuda_lib.compute(b, gfn1_options(cuda_lib))
    assert e.value.status == abi.NOT_IMPLEMENTED
