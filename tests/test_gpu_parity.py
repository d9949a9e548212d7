"""Parity of the CUDA path with the reference (fixtures, live library, oracle stages)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import REF_LIB, TOL_E, TOL_F, TOL_Q, as_molecule
from xtbloom_b200 import abi
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run(lib, mols, **opts):
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols],
                              [m[2] for m in mols], [m[3] for m in mols])
    return b, lib.compute(b, lib.make_options(**opts) if opts else None)


def fetch(lib, name, system, cap=2_000_000):
    f = lib.lib.xtbloom_b200_debug_fetch
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_double), C.c_size_t,
                  C.POINTER(C.c_size_t)]
    out = np.zeros(cap)
    cnt = C.c_size_t()
    assert f(lib.ctx, name.encode(), system, out.ctypes.data_as(C.POINTER(C.c_double)), cap,
             C.byref(cnt)) == 0
    return out[:cnt.value].copy()


def test_reference_fixtures_in_one_batch(cuda_lib, fixtures):
    """All committed reference outputs reproduced by one ragged CUDA batch."""
    mols = [as_molecule(s) for s in fixtures]
    b, out = run(cuda_lib, mols)
    for i, s in enumerate(fixtures):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == s["status"] == 0, s["name"]
        assert abs(out["energies"][i] - s["energy"]) < TOL_E, s["name"]
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(s["forces"])).max() < TOL_F, s["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(s["charges"])).max() < TOL_Q, s["name"]
        assert abs(int(out["scc_iterations"][i]) - s["scc_iterations"]) <= 1, s["name"]


def test_tblite_goldens(cuda_lib, fixtures, tblite_goldens):
    """The pinned tblite conformance energies and forces (tolerance 5e-7)."""
    names = [c["name"] for c in tblite_goldens]
    mols = [as_molecule(next(s for s in fixtures if s["name"] == n)) for n in names]
    b, out = run(cuda_lib, mols)
    for i, c in enumerate(tblite_goldens):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert abs(out["energies"][i] - c["energy"]) < 5e-7, c["name"]
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["forces"])).max() < 5e-7, c["name"]


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference library not built")
def test_live_reference_on_random_workload_sample(cuda_lib):
    """48 random systems of the 4096-system workload against the reference library, run live."""
    rng = np.random.default_rng(7)
    big = W.config1(4096)
    idx = np.sort(rng.choice(4096, 48, replace=False))
    sample = W.subset(big, idx)
    out = cuda_lib.compute(sample)
    ref = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=0)
    r = ref.compute(sample)
    ok = r["per_system_status"] == 0
    assert np.array_equal(out["per_system_status"][ok], r["per_system_status"][ok])
    assert np.abs(out["energies"][ok] - r["energies"][ok]).max() < TOL_E
    assert np.abs(out["forces"] - r["forces"]).max() < TOL_F
    assert np.abs(out["atomic_charges"] - r["atomic_charges"]).max() < TOL_Q


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference library not built")
def test_all_64_decane_conformers_against_live_reference(cuda_lib):
    """The whole 64-conformer C10H22 batch (seed 0), every output, against the
    reference library run live, iteration counts included."""
    b = W.config0(64, seed=0)
    out = cuda_lib.compute(b)
    ref = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=0)
    r = ref.compute(b)
    assert (r["per_system_status"] == 0).all() and (out["per_system_status"] == 0).all()
    assert np.abs(out["energies"] - r["energies"]).max() < TOL_E
    assert np.abs(out["forces"] - r["forces"]).max() < TOL_F
    assert np.abs(out["atomic_charges"] - r["atomic_charges"]).max() < TOL_Q
    assert np.abs(out["scc_iterations"] - r["scc_iterations"]).max() <= 1


def test_stage_intermediates_match_oracle(cuda_lib, fixtures):
    """Integer layout and every geometry-stage intermediate against the numpy oracle."""
    from oracle import gfn2
    s = next(x for x in fixtures if x["name"] == "hetero_chain_7")
    z, x, q, u = as_molecule(s)
    run(cuda_lib, [(z, x, q, u)])
    r = gfn2.singlepoint(z, x, charge=q, uhf=u, debug=True)
    d = r.debug
    assert np.abs(fetch(cuda_lib, "cn", 0) - d["cn"]).max() < 1e-12
    assert np.abs(fetch(cuda_lib, "cn_d4", 0) - d["cn_d4"]).max() < 1e-12
    assert np.abs(fetch(cuda_lib, "overlap", 0) - d["S"].ravel()).max() < 1e-13
    assert np.abs(fetch(cuda_lib, "dipole_integrals", 0) - d["D"].ravel()).max() < 1e-12
    assert np.abs(fetch(cuda_lib, "quadrupole_integrals", 0) - d["Q"].ravel()).max() < 1e-12
    assert np.abs(fetch(cuda_lib, "h0", 0) - d["H0"].ravel()).max() < 1e-13
    assert np.abs(fetch(cuda_lib, "density", 0) - d["P"].ravel()).max() < 1e-7
    # the SCC computes the occupied levels and at least eight above them
    ev = fetch(cuda_lib, "eigenvalues", 0)
    ev = ev[ev < 1e300]
    assert len(ev) >= min(len(d["eps"]), int(np.ceil(d["nel"] / 2)) + 8)
    assert np.abs(ev - d["eps"][:len(ev)]).max() < 1e-8
    assert np.abs(fetch(cuda_lib, "qsh", 0) - d["qsh"]).max() < 1e-7
    t = fetch(cuda_lib, "energy_terms", 0)
    ref = [r.terms[k] for k in ["core", "es2", "es3", "aes2", "d4", "entropy", "rep", "atm", "pc"]]
    assert np.abs(t[:9] - np.array(ref)).max() < 1e-7
    assert t[9] == 0.0   # spin polarisation: restricted system


def test_translation_rotation_invariance(cuda_lib, fixtures):
    s = next(x for x in fixtures if x["name"] == "hetero_chain_0")
    z, x, q, u = as_molecule(s)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
    x2 = x @ R.T + np.array([3.0, -1.5, 7.25])
    b, out = run(cuda_lib, [(z, x, q, u), (z, x2, q, u)])
    assert abs(out["energies"][0] - out["energies"][1]) < 1e-9
    n = len(z)
    f1 = out["forces"][:3 * n].reshape(-1, 3)
    f2 = out["forces"][3 * n:].reshape(-1, 3)
    # rotated copies differ only by SCC convergence noise (charge tolerance 1e-6)
    assert np.abs(f1 @ R.T - f2).max() < 1e-6
    assert np.abs(f1.sum(0)).max() < 1e-9


def test_batch_equals_serial(cuda_lib, fixtures):
    mols = [as_molecule(s) for s in fixtures[:8]]
    _, batched = run(cuda_lib, mols)
    for i, m in enumerate(mols):
        _, single = run(cuda_lib, [m])
        assert abs(single["energies"][0] - batched["energies"][i]) < 1e-11


def test_finite_difference_forces(cuda_lib, fixtures):
    """Central differences (h = 1e-4 bohr) of CUDA energies match CUDA analytic forces."""
    s = next(x for x in fixtures if x["name"] == "sif5_minus")
    z, x, q, u = as_molecule(s)
    h = 1e-4
    mols = [(z, x, q, u)]
    for a in range(len(z)):
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, c] += h
            xm[a, c] -= h
            mols += [(z, xp, q, u), (z, xm, q, u)]
    b, out = run(cuda_lib, mols, ctol=1e-10, etol=1e-12)
    e = out["energies"]
    fd = -(e[1::2] - e[2::2]) / (2 * h)
    assert np.abs(fd - out["forces"][:3 * len(z)]).max() < 1e-5


def test_nonconvergence_is_isolated_with_nan_slices(cuda_lib, fixtures):
    """A system that cannot converge within max_scc_iterations gets NaN slices and status 7;
    the call itself succeeds (per-system failure isolation)."""
    mols = [as_molecule(s) for s in fixtures[:3]]
    b, out = run(cuda_lib, mols, max_iter=3)
    assert (out["per_system_status"] == abi.SCC_NOT_CONVERGED).all()
    assert np.isnan(out["energies"]).all() and np.isnan(out["forces"]).all()
    assert (out["scc_converged"] == 0).all() and (out["scc_iterations"] == 3).all()


def test_invalid_positions_modify_no_output(cuda_lib, fixtures):
    z, x, q, u = as_molecule(fixtures[0])
    x = x.copy()
    x[0, 0] = np.nan
    b = abi.ragged_from_lists([z], [x])
    outs = {"energies": np.full(1, 123.0), "forces": np.full(3 * len(z), 7.0),
            "atomic_charges": np.full(len(z), 5.0), "scc_iterations": np.full(1, -1, np.int32),
            "scc_converged": np.full(1, 9, np.uint8), "per_system_status": np.full(1, -1, np.int32)}
    with pytest.raises(abi.XtbloomError) as err:
        cuda_lib.compute(b, None, outs)
    assert err.value.status == abi.INVALID_ARGUMENT
    assert outs["energies"][0] == 123.0 and (outs["forces"] == 7.0).all()


def test_device_buffers_match_host_buffers(cuda_lib, fixtures):
    torch = pytest.importorskip("torch")
    mols = [as_molecule(s) for s in fixtures[:4]]
    b, host = run(cuda_lib, mols)
    dev = torch.device("cuda", 0)
    bd = abi.RaggedBatch(b.atom_offsets, b.atomic_numbers, torch.from_numpy(b.positions).to(dev),
                         b.molecular_charges, b.unpaired_electrons)
    B, N = b.batch_size, b.total_atoms
    outs = {"energies": torch.empty(B, dtype=torch.float64, device=dev),
            "forces": torch.empty(3 * N, dtype=torch.float64, device=dev),
            "atomic_charges": torch.empty(N, dtype=torch.float64, device=dev),
            "scc_iterations": torch.empty(B, dtype=torch.int32, device=dev),
            "scc_converged": torch.empty(B, dtype=torch.uint8, device=dev),
            "per_system_status": torch.empty(B, dtype=torch.int32, device=dev)}
    cuda_lib.compute(bd, None, outs)
    torch.cuda.synchronize()
    assert np.abs(outs["energies"].cpu().numpy() - host["energies"]).max() < 1e-12
    assert np.abs(outs["forces"].cpu().numpy() - host["forces"]).max() < 1e-11


def test_enqueue_request_completes(cuda_lib, fixtures):
    mols = [as_molecule(s) for s in fixtures[:2]]
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols])
    lib = cuda_lib.lib
    req = C.c_void_p()
    assert lib.xtbloom_request_create(cuda_lib.ctx, C.byref(req)) == 0
    B, N = b.batch_size, b.total_atoms
    outs = {"energies": np.empty(B), "forces": np.empty(3 * N), "atomic_charges": np.empty(N),
            "scc_iterations": np.empty(B, np.int32), "scc_converged": np.empty(B, np.uint8),
            "per_system_status": np.empty(B, np.int32)}
    batch = cuda_lib.make_batch(b)
    opts = cuda_lib.make_options()
    res = cuda_lib.make_result(outs)
    assert lib.xtbloom_compute_enqueue(cuda_lib.ctx, C.byref(batch), C.byref(opts), C.byref(res), req) == 0
    info = abi.RequestInfo()
    lib.xtbloom_request_info_init(C.byref(info), C.sizeof(info))
    assert lib.xtbloom_request_wait(req, C.byref(info)) == 0
    assert info.state == 2 and info.completion_status == 0
    lib.xtbloom_request_destroy(req)
    assert np.isfinite(outs["energies"]).all()


def test_calculator_interface(fixtures):
    from xtbloom_b200 import Calculator
    s = next(x for x in fixtures if x["name"] == "ketene")
    z, x, q, u = as_molecule(s)
    res = Calculator("GFN2-xTB", z, x).singlepoint()
    assert abs(res.get("energy") - s["energy"]) < TOL_E
    assert np.abs(res.get("gradient").ravel() + np.asarray(s["forces"])).max() < TOL_F
