"""Golden fixtures of the GFN1-xTB path.

Two sources, both produced in the container that holds the reference checkout:
  * ``tblite`` entries: the reference's committed GFN1 conformance goldens
    (``data/conformance/gfn1/golden/*.json``: xTB 6.7.1 / tblite energies,
    forces and charges, tolerance 5e-7) for its six molecular cases, with
    their coordinates (``data/conformance/gfn1/inputs/*.coord``).
  * ``tblite_qmmm`` entries: its two GFN1 QM/MM goldens (xTB 6.7.1: a water
    dimer in six point charges, with GFN1 H/O hardnesses and with gamma = 999;
    ``inputs/*.qmmm.json``), point-charge forces included.
  * ``reference`` entries: the reference library itself (built from its
    sources by ``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) with
    model GFN1 on those six cases, on ten closed-shell hetero-alkane chains of
    the 4096-system workload (seed 1), and on twelve radicals of the 2048-radical
    GFN1 workload (seed 4; spin-polarised, two spin channels), at the default
    SCC settings and converged to the fixed point (charge tolerance 1e-10,
    energy tolerance 1e-13).
  * ``reference_pc``: the same library on the two QM/MM cases and on chains
    and radicals embedded in seeded point-charge shells (charges uniform in
    [-0.5, 0.5] e, zero net charge, 8-20 bohr from the centroid, gamma = 999
    or element-like hardness 0.5), point-charge forces included.
  * ``reference_response``: the same library with the charge response b + A q
    (b ~ N(0, 0.01) Eh/e per atom, A = (M + M^T)/2, M ~ N(0, 0.02)) on four
    conformance molecules and two radicals.

Usage:  python tests/golden/make_gfn1.py <reference checkout>  (or set XTBLOOM_REFERENCE_SRC)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from make_golden import read_coord  # noqa: E402
from xtbloom_b200 import abi, workloads as W  # noqa: E402


def entry(name, z, x, charge, uhf, nch, r, t):
    return {"name": name, "numbers": np.asarray(z).tolist(), "positions": np.asarray(x).ravel().tolist(),
            "charge": float(charge), "uhf": int(uhf), "spin_channels": int(nch),
            "status": int(r["per_system_status"][0]), "scc_iterations": int(r["scc_iterations"][0]),
            "energy": float(r["energies"][0]), "forces": r["forces"].tolist(),
            "charges": r["atomic_charges"].tolist(),
            "tight_status": int(t["per_system_status"][0]), "tight_energy": float(t["energies"][0]),
            "tight_forces": t["forces"].tolist(), "tight_charges": t["atomic_charges"].tolist()}


def main(ref: Path):
    lib = abi.Library(str(ROOT / "oracle/_ref/libxtbloom_ref.so"), backend=abi.BACKEND_CPU, cpu_threads=0)
    dflt = lib.make_options(model=abi.MODEL_GFN1)
    tight = lib.make_options(model=abi.MODEL_GFN1, ctol=1e-10, etol=1e-13)

    def run(z, x, charge, uhf, nch):
        b = abi.ragged_from_lists([z], [x], [charge], [uhf], [nch])
        return lib.compute(b, dflt), lib.compute(b, tight)

    man = json.loads((ref / "data/conformance/gfn1/manifest.json").read_text())
    tblite, refs = [], []
    for c in man["cases"]:
        if not c["input"].endswith(".coord"):
            continue
        z, x = read_coord(ref / c["input"])
        g = json.loads((ref / c["golden"]).read_text())["properties"]
        tblite.append({"name": c["id"], "numbers": z.tolist(), "positions": x.ravel().tolist(),
                       "charge": float(c["molecular_charge"]), "uhf": int(c["unpaired_electrons"]),
                       "energy": g["energy_hartree"], "forces": g["forces_hartree_per_bohr"],
                       "charges": g.get("partial_charges_e")})
        r, t = run(z, x, float(c["molecular_charge"]), int(c["unpaired_electrons"]), 1)
        refs.append(entry(c["id"], z, x, c["molecular_charge"], c["unpaired_electrons"], 1, r, t))
        print(c["id"], refs[-1]["status"], refs[-1]["energy"], g["energy_hartree"], flush=True)
    b1 = W.config1(4096, seed=1)
    for i in [0, 7, 100, 512, 1023, 2048, 3001, 3500, 4095, 1500]:
        z, x = W.molecule(b1, i)
        r, t = run(z, x, 0.0, 0, 1)
        refs.append(entry(f"hetero_chain_{i}", z, x, 0.0, 0, 1, r, t))
        print(refs[-1]["name"], refs[-1]["status"], refs[-1]["energy"], flush=True)
    b4 = W.config4(2048, seed=4)
    halo = [i for i in range(2048) if np.isin(W.molecule(b4, i)[0], (17, 35)).any()]
    plain = [i for i in range(2048) if i not in set(halo)]
    for i in plain[:6] + halo[:6]:
        z, x = W.molecule(b4, i)
        r, t = run(z, x, 0.0, 1, 2)
        refs.append(entry(f"radical_{i}", z, x, 0.0, 1, 2, r, t))
        refs[-1]["index"] = i
        print(refs[-1]["name"], refs[-1]["status"], refs[-1]["scc_iterations"], refs[-1]["energy"], flush=True)
    qmmm, pcs = [], []
    for c in man["cases"]:
        if not c["input"].endswith(".qmmm.json"):
            continue
        d = json.loads((ref / c["input"]).read_text())
        g = json.loads((ref / c["golden"]).read_text())["properties"]
        pc = d["external_point_charges"]
        item = {"name": c["id"], "numbers": d["qm"]["atomic_numbers"],
                "positions": np.asarray(d["qm"]["positions_bohr"]).ravel().tolist(),
                "charge": float(d["qm"]["molecular_charge"]), "uhf": int(d["qm"]["unpaired_electrons"]),
                "spin_channels": 1, "pc_positions": np.asarray(pc["positions_bohr"]).ravel().tolist(),
                "pc_charges": pc["charges_e"], "pc_gammas": pc["gammas_hartree"]}
        qmmm.append(dict(item, energy=g["energy_hartree"], forces=g["forces_hartree_per_bohr"],
                         charges=g.get("partial_charges_e"),
                         point_charge_forces=g["point_charge_forces_hartree_per_bohr"]))
        pcs.append(item)
    rng = np.random.default_rng(41)

    def shell(x, npc, gamma):
        c = x.mean(0)
        q = rng.uniform(-0.5, 0.5, npc)
        q -= q.mean()
        d = rng.normal(size=(npc, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        r = rng.uniform(8.0 ** 3, 20.0 ** 3, npc) ** (1 / 3)
        return (c + d * r[:, None]).ravel().tolist(), q.tolist(), [gamma] * npc

    for k, i in enumerate([7, 512, 2048, 3500]):
        z, x = W.molecule(b1, i)
        pp, pq, pg = shell(x, 60, 999.0 if k % 2 == 0 else 0.5)
        pcs.append({"name": f"hetero_chain_{i}_pc", "numbers": z.tolist(), "positions": x.ravel().tolist(),
                    "charge": 0.0, "uhf": 0, "spin_channels": 1, "pc_positions": pp, "pc_charges": pq,
                    "pc_gammas": pg})
    for i in plain[:1] + halo[:1]:
        z, x = W.molecule(b4, i)
        pp, pq, pg = shell(x, 40, 0.5)
        pcs.append({"name": f"radical_{i}_pc", "numbers": z.tolist(), "positions": x.ravel().tolist(),
                    "charge": 0.0, "uhf": 1, "spin_channels": 2, "pc_positions": pp, "pc_charges": pq,
                    "pc_gammas": pg})
    flags = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES | abi.COMPUTE_CHARGES | abi.COMPUTE_POINT_CHARGE_FORCES
    for item in pcs:
        b = abi.ragged_from_lists([np.asarray(item["numbers"], np.int32)],
                                  [np.asarray(item["positions"]).reshape(-1, 3)], [item["charge"]],
                                  [item["uhf"]], [item["spin_channels"]])
        npc = len(item["pc_charges"])
        b.point_charge_offsets = np.array([0, npc], np.int64)
        b.point_charge_positions = np.asarray(item["pc_positions"], float)
        b.point_charge_values = np.asarray(item["pc_charges"], float)
        b.point_charge_gammas = np.asarray(item["pc_gammas"], float)
        r = lib.compute(b, lib.make_options(model=abi.MODEL_GFN1, flags=flags))
        t = lib.compute(b, lib.make_options(model=abi.MODEL_GFN1, flags=flags, ctol=1e-10, etol=1e-13))
        item.update(entry(item["name"], item["numbers"], item["positions"], item["charge"], item["uhf"],
                          item["spin_channels"], r, t))
        item["point_charge_forces"] = r["point_charge_forces"].tolist()
        item["tight_point_charge_forces"] = t["point_charge_forces"].tolist()
        print(item["name"], item["status"], item["scc_iterations"], item["energy"], flush=True)
    resp = []
    for c in refs[:4] + [r_ for r_ in refs if r_["name"].startswith("radical_")][:2]:
        z = np.asarray(c["numbers"], np.int32)
        x = np.asarray(c["positions"]).reshape(-1, 3)
        n = len(z)
        shifts = rng.normal(0.0, 0.01, n)
        M = rng.normal(0.0, 0.02, (n, n))
        A = 0.5 * (M + M.T)
        b = abi.ragged_from_lists([z], [x], [c["charge"]], [c["uhf"]], [c["spin_channels"]])
        b.atomic_potential_shifts = shifts
        b.charge_response_offsets = np.array([0, n * n], np.int64)
        b.charge_response_matrix = A.ravel()
        r = lib.compute(b, dflt)
        t = lib.compute(b, tight)
        item = entry(c["name"] + "_response", z, x, c["charge"], c["uhf"], c["spin_channels"], r, t)
        item.update(shifts=shifts.tolist(), response=A.ravel().tolist())
        resp.append(item)
        print(item["name"], item["status"], item["scc_iterations"], item["energy"], flush=True)
    (HERE / "gfn1_fixtures.json").write_text(json.dumps({"tblite": tblite, "tblite_qmmm": qmmm,
                                                         "reference": refs, "reference_pc": pcs,
                                                         "reference_response": resp}))


def reference_checkout() -> Path:
    """The reference checkout: the first argument, else $XTBLOOM_REFERENCE_SRC."""
    import os
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XTBLOOM_REFERENCE_SRC")
    if not arg:
        sys.exit("usage: pass the reference checkout as the first argument "
                 "or set XTBLOOM_REFERENCE_SRC")
    return Path(arg)


if __name__ == "__main__":
    main(reference_checkout())
