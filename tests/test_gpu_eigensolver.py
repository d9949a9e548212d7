"""The SCC eigensolver on its own, for both Householder kernels.

After a compute the engine retains the last Fock matrix H and the Loewdin
orthogonaliser X; the eigenvalues it kept must be those of X H X (LAPACK
through numpy), whichever tridiagonalisation ran: the register-resident
cluster kernel (few systems, n <= 256) or the shared-memory kernel
(XTBLOOM_B200_TRIDIAG=smem).  Whole computes through either kernel agree.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from xtbloom_b200 import abi, library_path
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu


def batch():
    full = W.config1(4096, seed=1)
    # sizes from 2 to ~240 orbitals, and a few molecules below 16 orbitals
    b = W.subset(full, [0, 7, 100, 1164, 2048, 4000])
    small = [([1, 1], [[0, 0, 0], [0, 0, 1.4]]),
             ([8, 1, 1], [[0, 0, 0], [0, 1.43, 1.1], [0, -1.43, 1.1]]),
             ([1], [[0, 0, 0]])]
    nums = [b.atomic_numbers[b.atom_offsets[i]:b.atom_offsets[i + 1]] for i in range(b.batch_size)]
    pos = [b.positions[3 * b.atom_offsets[i]:3 * b.atom_offsets[i + 1]].reshape(-1, 3)
           for i in range(b.batch_size)]
    for z, r in small:
        nums.append(np.array(z))
        pos.append(np.array(r, float))
    uhf = [0] * b.batch_size + [0, 0, 1]
    return abi.ragged_from_lists(nums, pos, None, uhf)


def run(kernel: str | None, tight: bool = False):
    if kernel is None:
        os.environ.pop("XTBLOOM_B200_TRIDIAG", None)
    else:
        os.environ["XTBLOOM_B200_TRIDIAG"] = kernel
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=0)
    try:
        b = batch()
        out = lib.compute(b, lib.make_options(ctol=1e-10, etol=1e-13) if tight else None)
        eig = []
        for i in range(b.batch_size):
            h = lib.fetch("hamiltonian", i)
            x = lib.fetch("x", i)
            ev = lib.fetch("eigenvalues", i)
            n = len(ev)
            eig.append((h.reshape(n, n), x.reshape(n, n), ev))
        return out, eig
    finally:
        os.environ.pop("XTBLOOM_B200_TRIDIAG", None)
        lib.close()


@pytest.fixture(scope="module")
def both():
    return run(None), run("smem")


@pytest.mark.parametrize("which", [0, 1])
def test_eigenvalues_match_lapack(both, which):
    out, eig = both[which]
    assert (out["per_system_status"] == 0).all()
    for h, x, ev in eig:
        a = x @ h @ x
        ref = np.linalg.eigvalsh(0.5 * (a + a.T))
        k = int((ev < 1e300).sum())
        assert k >= 1
        scale = max(1.0, np.abs(ref).max())
        assert np.abs(ev[:k] - ref[:k]).max() < 1e-10 * scale


def test_kernels_reach_the_same_fixed_point():
    """Converged to the fixed point (charge tolerance 1e-10), the two kernels
    agree on every output of every system, the slowly converging one included."""
    (a, _), (b, _) = run(None, tight=True), run("smem", tight=True)
    ok = (a["per_system_status"] == 0) & (b["per_system_status"] == 0)
    assert ok.sum() >= len(ok) - 1
    assert np.abs(a["energies"][ok] - b["energies"][ok]).max() < 1e-9
    offs = batch().atom_offsets
    for i in np.where(ok)[0]:
        a0, a1 = offs[i], offs[i + 1]
        assert np.abs(a["forces"][3 * a0:3 * a1] - b["forces"][3 * a0:3 * a1]).max() < 1e-7, i
        assert np.abs(a["atomic_charges"][a0:a1] - b["atomic_charges"][a0:a1]).max() < 1e-7, i


def test_kernels_agree_on_whole_computes(both):
    """Systems that converge promptly follow the same SCC path through either
    kernel; system 1164 of the workload takes over a hundred iterations and
    its trajectory depends on rounding, so it only has to land inside the
    convergence gate (energy variational, charges first order)."""
    (a, _), (b, _) = both
    fast = (a["scc_iterations"] <= 60) & (b["scc_iterations"] <= 60)
    assert fast.sum() == len(fast) - 1
    assert np.array_equal(a["scc_iterations"][fast], b["scc_iterations"][fast])
    assert np.abs(a["energies"][fast] - b["energies"][fast]).max() < 1e-9
    assert np.abs(a["energies"] - b["energies"]).max() < 1e-6
    offs = batch().atom_offsets
    for i in range(len(fast)):
        tol = 1e-8 if fast[i] else 1e-4
        a0, a1 = offs[i], offs[i + 1]
        assert np.abs(a["forces"][3 * a0:3 * a1] - b["forces"][3 * a0:3 * a1]).max() < tol
        assert np.abs(a["atomic_charges"][a0:a1] - b["atomic_charges"][a0:a1]).max() < tol


def test_warm_started_refinement_matches_the_householder_path(cuda_lib, monkeypatch):
    """The opt-in warm-started eigensolver (Ogita-Aishima refinement of the
    previous iteration's eigenvectors, k_refine.cu) gives the Householder
    path's results: same statuses and iteration counts, energies, charges and
    forces to well inside the public tolerances; it refines most channels
    after the first iterations and falls back to the Householder path for the
    rest."""
    full = W.config1(4096, seed=1)
    b = W.subset(full, [7, 100, 2048, 4000, 11, 222])
    ref = cuda_lib.compute(b)
    monkeypatch.setenv("XTBLOOM_B200_REFINE_STEPS", "5")
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=0)
    try:
        out = lib.compute(b)
        stats = lib.fetch("refine_stats", capacity=4096).reshape(256, 8)
    finally:
        lib.close()
    assert np.array_equal(out["per_system_status"], ref["per_system_status"])
    assert np.abs(out["scc_iterations"] - ref["scc_iterations"]).max() <= 1
    assert np.abs(out["energies"] - ref["energies"]).max() < 1e-8
    assert np.abs(out["atomic_charges"] - ref["atomic_charges"]).max() < 1e-6
    assert np.abs(out["forces"] - ref["forces"]).max() < 1e-6
    assert stats[:, 0].sum() > 0 and stats[:, 1:4].sum() > 0   # channels were refined
