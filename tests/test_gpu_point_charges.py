"""External point charges on the CUDA path against the reference library and the oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import REF_LIB, TOL_E, TOL_F, TOL_Q, as_molecule, as_pc
from xtbloom_b200 import abi
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu

FLAGS = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES | abi.COMPUTE_CHARGES | abi.COMPUTE_POINT_CHARGE_FORCES


def pc_batch(systems):
    b = abi.ragged_from_lists([as_molecule(s)[0] for s in systems], [as_molecule(s)[1] for s in systems],
                              [s["charge"] for s in systems], [s["uhf"] for s in systems])
    counts = [len(s.get("pc_charges", [])) for s in systems]
    b.point_charge_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    cat = lambda k, w: np.ascontiguousarray(np.concatenate([np.asarray(s.get(k, []), float).reshape(-1) for s in systems]))  # noqa: E731
    b.point_charge_positions = cat("pc_positions", 3)
    b.point_charge_values = cat("pc_charges", 1)
    b.point_charge_gammas = cat("pc_gammas", 1)
    return b


def fetch(lib, name, system, cap=100_000):
    f = lib.lib.xtbloom_b200_debug_fetch
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_double), C.c_size_t,
                  C.POINTER(C.c_size_t)]
    out = np.zeros(cap)
    cnt = C.c_size_t()
    assert f(lib.ctx, name.encode(), system, out.ctypes.data_as(C.POINTER(C.c_double)), cap,
             C.byref(cnt)) == 0
    return out[:cnt.value].copy()


def test_point_charge_fixtures_in_one_batch(cuda_lib, pc_fixtures, fixtures):
    """Every embedded fixture plus two unembedded systems (zero charges) in one ragged call."""
    plain = [s for s in fixtures if s["name"] in ("ketene", "hetero_chain_1")]
    systems = pc_fixtures + plain
    b = pc_batch(systems)
    out = cuda_lib.compute(b, cuda_lib.make_options(flags=FLAGS))
    off = b.point_charge_offsets
    for i, s in enumerate(systems):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert out["per_system_status"][i] == 0, s["name"]
        assert abs(out["energies"][i] - s["energy"]) < TOL_E, s["name"]
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(s["forces"])).max() < TOL_F, s["name"]
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(s["charges"])).max() < TOL_Q, s["name"]
        if "pc_forces" in s:
            got = out["point_charge_forces"][3 * off[i]:3 * off[i + 1]]
            assert np.abs(got - np.asarray(s["pc_forces"])).max() < TOL_F, s["name"]
        if "xtb_energy" in s:
            assert abs(out["energies"][i] - s["xtb_energy"]) < 5e-7, s["name"]


def test_charge_derivative_matches_oracle_and_finite_differences(cuda_lib, pc_fixtures):
    from oracle import gfn2
    s = next(x for x in pc_fixtures if x["name"] == "water_dimer_6pc_hardness")
    z, x, q, u = as_molecule(s)
    pp, pq, pg = as_pc(s)
    cuda_lib.compute(pc_batch([s]), cuda_lib.make_options(flags=FLAGS))
    dq = fetch(cuda_lib, "point_charge_dq", 0)
    r = gfn2.singlepoint(z, x, q, u, pc_pos=pp, pc_q=pq, pc_gam=pg)
    assert np.abs(dq - r.pc_dq).max() < 1e-8
    h = 1e-4
    var = []
    for p in range(len(pq)):
        for sgn in (1, -1):
            t = dict(s)
            qq = pq.copy()
            qq[p] += sgn * h
            t["pc_charges"] = qq.tolist()
            var.append(t)
    out = cuda_lib.compute(pc_batch(var), cuda_lib.make_options(flags=FLAGS, ctol=1e-10, etol=1e-12))
    e = out["energies"]
    assert np.abs((e[0::2] - e[1::2]) / (2 * h) - dq).max() < 1e-6


def test_config2_sample_against_live_reference(cuda_lib):
    """Four C20H42 conformers in 200 charges each (the differentiation workload's systems)."""
    if not REF_LIB.exists():
        pytest.skip("reference library not built")
    b = W.config2(4)
    out = cuda_lib.compute(b, cuda_lib.make_options(flags=FLAGS))
    ref = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=0)
    r = ref.compute(b, ref.make_options(flags=FLAGS))
    assert (out["per_system_status"] == 0).all()
    assert np.abs(out["energies"] - r["energies"]).max() < TOL_E
    assert np.abs(out["forces"] - r["forces"]).max() < TOL_F
    assert np.abs(out["point_charge_forces"] - r["point_charge_forces"]).max() < TOL_F


def test_invalid_hardness_modifies_no_output(cuda_lib, pc_fixtures):
    s = dict(next(x for x in pc_fixtures if x["name"] == "water_one_pc_gamma999"))
    s["pc_gammas"] = [0.0]
    b = pc_batch([s])
    n = len(s["numbers"])
    outs = {"energies": np.full(1, 123.0), "forces": np.full(3 * n, 7.0),
            "atomic_charges": np.full(n, 5.0), "point_charge_forces": np.full(3, 9.0),
            "scc_iterations": np.full(1, -1, np.int32), "scc_converged": np.full(1, 9, np.uint8),
            "per_system_status": np.full(1, -1, np.int32)}
    with pytest.raises(abi.XtbloomError) as err:
        cuda_lib.compute(b, cuda_lib.make_options(flags=FLAGS), outs)
    assert err.value.status == abi.INVALID_ARGUMENT
    assert outs["energies"][0] == 123.0 and (outs["point_charge_forces"] == 9.0).all()


def test_unconverged_system_gets_nan_point_charge_forces(cuda_lib, pc_fixtures):
    systems = [s for s in pc_fixtures if s["name"].startswith("water")][:2]
    out = cuda_lib.compute(pc_batch(systems), cuda_lib.make_options(flags=FLAGS, max_iter=3))
    assert (out["per_system_status"] == abi.SCC_NOT_CONVERGED).all()
    assert np.isnan(out["point_charge_forces"]).all()
