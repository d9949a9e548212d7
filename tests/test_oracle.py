"""Pins of the CPU oracle (numpy restatement) against the reference's own outputs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import as_molecule, as_pc
from oracle import gfn2

FAST = ["c10h22_conformer_0", "c10h22_conformer_3", "hetero_chain_7", "h3_plus", "ketene",
        "nenacl", "sif5_minus", "oh_radical", "zn_atom", "i_anion", "rn_atom"]


@pytest.mark.parametrize("name", FAST)
def test_oracle_matches_reference_library(fixtures, name):
    """Energy, forces, charges and iteration count equal the compiled reference library."""
    sys_ = next(s for s in fixtures if s["name"] == name)
    z, x, q, u = as_molecule(sys_)
    r = gfn2.singlepoint(z, x, charge=q, uhf=u)
    assert r.converged
    assert abs(r.energy - sys_["energy"]) < 1e-9
    assert np.abs(-r.gradient.ravel() - np.asarray(sys_["forces"])).max() < 1e-8
    assert np.abs(r.charges - np.asarray(sys_["charges"])).max() < 1e-8
    assert r.iterations == sys_["scc_iterations"]


def test_oracle_matches_tblite_goldens(fixtures, tblite_goldens):
    """The oracle reproduces the pinned tblite 0.7.0 conformance energies and forces (5e-7)."""
    for case in tblite_goldens:
        sys_ = next(s for s in fixtures if s["name"] == case["name"])
        z, x, q, u = as_molecule(sys_)
        r = gfn2.singlepoint(z, x, charge=q, uhf=u)
        assert abs(r.energy - case["energy"]) < 5e-7, case["name"]
        assert np.abs(-r.gradient.ravel() - np.asarray(case["forces"])).max() < 5e-7, case["name"]


def test_oracle_gradient_is_derivative_of_energy(fixtures):
    """Central finite differences (h = 1e-4 bohr) of the oracle energy match its analytic gradient."""
    sys_ = next(s for s in fixtures if s["name"] == "ketene")
    z, x, q, u = as_molecule(sys_)
    r = gfn2.singlepoint(z, x, charge=q, uhf=u, ctol=1e-10, etol=1e-12)
    h = 1e-4
    fd = np.zeros_like(x)
    for a in range(len(z)):
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, c] += h
            xm[a, c] -= h
            ep = gfn2.singlepoint(z, xp, q, u, ctol=1e-10, etol=1e-12, forces=False).energy
            em = gfn2.singlepoint(z, xm, q, u, ctol=1e-10, etol=1e-12, forces=False).energy
            fd[a, c] = (ep - em) / (2 * h)
    assert np.abs(fd - r.gradient).max() < 2e-6


def test_integer_layout_of_basis():
    """AO/shell counts per element follow the GFN2 basis (H: 1s; C, N, O: 2s2p; Cl: 3s3p3d)."""
    for z, nsh, nao in [(1, 1, 1), (6, 2, 4), (7, 2, 4), (8, 2, 4), (17, 3, 9)]:
        b = gfn2.make_basis(np.array([z]))
        assert len(b.sh_l) == nsh and b.nao == nao


PC_FAST = ["water_one_pc_gamma999", "water_one_pc_close_hardness", "water_one_pc_coincident_hardness",
           "water_dimer_6pc_hardness", "water_dimer_6pc_gamma999", "hetero_chain_7_pc30_gamma999",
           "hetero_chain_3001_pc30_gamma0.8"]


@pytest.mark.parametrize("name", PC_FAST)
def test_oracle_point_charges_match_reference_library(pc_fixtures, name):
    """Embedded energies, forces, charges and point-charge forces equal the compiled reference."""
    sys_ = next(s for s in pc_fixtures if s["name"] == name)
    z, x, q, u = as_molecule(sys_)
    pp, pq, pg = as_pc(sys_)
    r = gfn2.singlepoint(z, x, charge=q, uhf=u, pc_pos=pp, pc_q=pq, pc_gam=pg)
    assert r.converged and r.iterations == sys_["scc_iterations"]
    assert abs(r.energy - sys_["energy"]) < 1e-9
    assert np.abs(-r.gradient.ravel() - np.asarray(sys_["forces"])).max() < 1e-8
    assert np.abs(r.charges - np.asarray(sys_["charges"])).max() < 1e-8
    assert np.abs(-r.pc_gradient.ravel() - np.asarray(sys_["pc_forces"])).max() < 1e-8
    if "xtb_energy" in sys_:   # the reference's xTB 6.7.1 QM/MM goldens
        assert abs(r.energy - sys_["xtb_energy"]) < 5e-7
        assert np.abs(-r.gradient.ravel() - np.asarray(sys_["xtb_forces"])).max() < 5e-7
        assert np.abs(-r.pc_gradient.ravel() - np.asarray(sys_["xtb_pc_forces"])).max() < 5e-7


def test_oracle_point_charge_derivatives_are_finite_differences(pc_fixtures):
    """dE/dQ_p and dE/dR_p from central differences (h = 1e-4) of the oracle energy."""
    sys_ = next(s for s in pc_fixtures if s["name"] == "water_dimer_6pc_hardness")
    z, x, q, u = as_molecule(sys_)
    pp, pq, pg = as_pc(sys_)
    tight = dict(charge=q, uhf=u, ctol=1e-10, etol=1e-12, pc_gam=pg)
    r = gfn2.singlepoint(z, x, pc_pos=pp, pc_q=pq, **tight)
    h = 1e-4
    for p in range(len(pq)):
        qp, qm = pq.copy(), pq.copy()
        qp[p] += h
        qm[p] -= h
        ep = gfn2.singlepoint(z, x, pc_pos=pp, pc_q=qp, forces=False, **tight).energy
        em = gfn2.singlepoint(z, x, pc_pos=pp, pc_q=qm, forces=False, **tight).energy
        assert abs((ep - em) / (2 * h) - r.pc_dq[p]) < 1e-6
    for p, c in [(0, 0), (3, 2)]:
        xp, xm = pp.copy(), pp.copy()
        xp[p, c] += h
        xm[p, c] -= h
        ep = gfn2.singlepoint(z, x, pc_pos=xp, pc_q=pq, forces=False, **tight).energy
        em = gfn2.singlepoint(z, x, pc_pos=xm, pc_q=pq, forces=False, **tight).energy
        assert abs((ep - em) / (2 * h) - r.pc_gradient[p, c]) < 1e-6


def test_unrestricted_goldens_pinned_to_tblite_trace():
    """The unrestricted goldens come from the reference library; its OH radical
    (spin_channels = 2) reproduces the reference's tblite UHF SCC trace: same
    iteration count, final charges within the trace's own residual (1e-5)."""
    import json

    from conftest import GOLDEN
    oh = json.loads((GOLDEN / "uhf_fixtures.json").read_text())["oh_radical"]
    assert oh["status"] == 0
    assert oh["scc_iterations"] == oh["tblite_iterations"]
    assert np.abs(np.asarray(oh["charges"]) - np.asarray(oh["tblite_final_charges"])).max() < 2e-5


def test_field_goldens_pinned_to_tblite():
    """The electric-field goldens come from the reference library, whose water
    energy in the field (0.003, -0.004, 0.005) equals the reference's committed
    tblite value of its water_efield conformance case."""
    import json

    from conftest import GOLDEN
    g = json.loads((GOLDEN / "field_fixtures.json").read_text())
    w = next(s for s in g["systems"] if s["name"] == "water_efield" and s["case"] == "field")
    assert w["status"] == 0
    assert abs(w["energy"] - g["tblite_water_efield_energy"]) < 1e-9


def test_gfn1_goldens_pinned_to_tblite():
    """The GFN1 goldens come from the reference library; converged to its fixed
    point (charge tolerance 1e-10; the committed values were produced with
    xTB's tight SCC accuracy 1e-4) it reproduces the reference's six
    molecular GFN1 conformance cases (xTB 6.7.1 / tblite energies, forces and
    charges) and its two QM/MM cases (energies, forces, point-charge forces)
    at their tolerance (5e-7)."""
    import json

    from conftest import GOLDEN
    g = json.loads((GOLDEN / "gfn1_fixtures.json").read_text())
    ref = {c["name"]: c for c in g["reference"]}
    assert len(g["tblite"]) == 6
    for c in g["tblite"]:
        r = ref[c["name"]]
        assert r["tight_status"] == 0, c["name"]
        assert abs(r["tight_energy"] - c["energy"]) < 5e-7, c["name"]
        assert np.abs(np.asarray(r["tight_forces"]) - np.asarray(c["forces"])).max() < 5e-7, c["name"]
        if c["charges"] is not None:
            assert np.abs(np.asarray(r["tight_charges"]) - np.asarray(c["charges"])).max() < 5e-7, c["name"]
    # the two QM/MM cases (xTB 6.7.1, water dimer in six point charges)
    pcref = {c["name"]: c for c in g["reference_pc"]}
    assert len(g["tblite_qmmm"]) == 2
    for c in g["tblite_qmmm"]:
        r = pcref[c["name"]]
        assert r["tight_status"] == 0, c["name"]
        assert abs(r["tight_energy"] - c["energy"]) < 5e-7, c["name"]
        assert np.abs(np.asarray(r["tight_forces"]) - np.asarray(c["forces"]).ravel()).max() < 5e-7, c["name"]
        assert np.abs(np.asarray(r["tight_point_charge_forces"])
                      - np.asarray(c["point_charge_forces"]).ravel()).max() < 5e-7, c["name"]
