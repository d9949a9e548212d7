"""Generate the golden fixtures used by the parity tests.

Two sources, both produced in the container that holds the reference checkout:
  * ``reference_fixtures.json``: energies, forces, charges and SCC iteration
    counts computed by the reference library itself (built from its sources
    by ``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) on seeded
    synthetic molecules: 6 C10H22 conformers (64-conformer workload, seed 0),
    10 hetero-alkane chains of the 4096-system workload (seed 1), and the
    coordinates of the reference's GFN2 conformance inputs.
  * ``tblite_goldens.json``: the reference's committed tblite 0.7.0 GFN2
    conformance energies/forces (data/conformance/golden/*.json), restricted
    to the molecular cases without external fields or point charges.

  * ``pc_fixtures.json``: systems embedded in external point charges, run
    through the same reference library (energies, forces, charges and
    point-charge forces), together with the reference's xTB 6.7.1 QM/MM
    goldens for the cases that come from its conformance set.

Usage:  python tests/golden/make_golden.py <reference checkout>  (or set XTBLOOM_REFERENCE_SRC)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from xtbloom_b200 import abi, workloads as W  # noqa: E402

SYM = {"h": 1, "he": 2, "c": 6, "n": 7, "o": 8, "f": 9, "ne": 10, "na": 11, "si": 14, "cl": 17,
       "zn": 30, "br": 35, "i": 53, "rn": 86}


def read_coord(path: Path):
    z, x = [], []
    for line in path.read_text().splitlines():
        s = line.split()
        if not s:
            continue
        if s[0].startswith("$"):
            if s[0] == "$end":
                break
            continue
        x.append([float(v) for v in s[:3]])
        z.append(SYM[s[3].lower()])
    return np.array(z, np.int32), np.array(x)


def molecules(ref: Path):
    mols = []
    b0 = W.config0(6)
    for i in range(6):
        z, x = W.molecule(b0, i)
        mols.append({"name": f"c10h22_conformer_{i}", "numbers": z, "positions": x, "charge": 0.0, "uhf": 0})
    b1 = W.config1(4096)
    pick = [0, 1, 7, 100, 512, 1023, 2048, 3001, 3500, 4095]
    for i in pick:
        z, x = W.molecule(b1, i)
        mols.append({"name": f"hetero_chain_{i}", "numbers": z, "positions": x, "charge": 0.0, "uhf": 0})
    man = json.loads((ref / "data/conformance/manifest.json").read_text())
    for c in man["cases"]:
        if not c["input"].endswith(".coord"):
            continue
        z, x = read_coord(ref / c["input"])
        mols.append({"name": c["id"], "numbers": z, "positions": x,
                     "charge": float(c["molecular_charge"]), "uhf": int(c["unpaired_electrons"])})
    return mols


def main(ref: Path):
    lib = abi.Library(str(ROOT / "oracle/_ref/libxtbloom_ref.so"), backend=abi.BACKEND_CPU, cpu_threads=1)
    out = []
    for m in molecules(ref):
        b = abi.ragged_from_lists([m["numbers"]], [m["positions"]], [m["charge"]], [m["uhf"]])
        r = lib.compute(b)
        out.append({"name": m["name"], "numbers": m["numbers"].tolist(),
                    "positions": np.asarray(m["positions"]).reshape(-1).tolist(),
                    "charge": m["charge"], "uhf": m["uhf"],
                    "status": int(r["per_system_status"][0]),
                    "energy": float(r["energies"][0]), "forces": r["forces"].tolist(),
                    "charges": r["atomic_charges"].tolist(),
                    "scc_iterations": int(r["scc_iterations"][0])})
    (HERE / "reference_fixtures.json").write_text(json.dumps(
        {"source": "reference library built from its sources (oracle/ref.mk), FP64, cpu_threads=1",
         "settings": {"charge_tolerance": 1e-6, "energy_tolerance": 1e-8, "max_iter": 250,
                      "temperature_K": 300.0, "mixer": "broyden 8 / 0.4"},
         "systems": out}, indent=0))
    man = json.loads((ref / "data/conformance/manifest.json").read_text())
    gold = []
    for c in man["cases"]:
        if not c["input"].endswith(".coord") or "efield" in c["id"]:
            continue
        g = json.loads((ref / c["golden"]).read_text())
        gold.append({"name": c["id"], "energy": g["properties"]["energy_hartree"],
                     "forces": g["properties"]["forces_hartree_per_bohr"],
                     "engine": g["provenance"]["engine"], "version": g["provenance"]["executable_version"].split("\n")[0]})
    (HERE / "tblite_goldens.json").write_text(json.dumps(
        {"source": "reference data/conformance/golden (tblite 0.7.0 / xTB 6.7.1), tolerance 5e-7",
         "cases": gold}, indent=0))


def pc_cases(ref: Path):
    """Point-charge embedded systems: the reference's xTB 6.7.1 QM/MM goldens, hetero
    chains with random charges (two hardness regimes) and C20H42 in 200 charges."""
    cases = []
    man = json.loads((ref / "data/conformance/manifest.json").read_text())
    for c in man["cases"]:
        g = json.loads((ref / c["golden"]).read_text())
        if "qmmm_input" not in g:
            continue
        qi = g["qmmm_input"]
        pc = qi["external_point_charges"]
        cases.append({"name": c["id"], "numbers": qi["qm"]["atomic_numbers"],
                      "positions": np.asarray(qi["qm"]["positions_bohr"]).reshape(-1).tolist(),
                      "charge": float(qi["qm"]["molecular_charge"]), "uhf": int(qi["qm"]["unpaired_electrons"]),
                      "pc_positions": np.asarray(pc["positions_bohr"]).reshape(-1).tolist(),
                      "pc_charges": list(pc["charges_e"]), "pc_gammas": list(pc["gammas_hartree"]),
                      "xtb_energy": g["properties"]["energy_hartree"],
                      "xtb_forces": g["properties"]["forces_hartree_per_bohr"],
                      "xtb_pc_forces": np.asarray(g["properties"]["point_charge_forces_hartree_per_bohr"]).reshape(-1).tolist()})
    rng = np.random.default_rng(11)
    b1 = W.config1(4096)
    for i, gam in [(7, 999.0), (100, 999.0), (512, 0.8), (3001, 0.8)]:
        z, x = W.molecule(b1, i)
        npc = 30
        c0 = x.mean(0)
        d = rng.normal(size=(npc, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        r = rng.uniform(4.0, 14.0, npc)
        q = rng.uniform(-0.5, 0.5, npc)
        q -= q.mean()
        cases.append({"name": f"hetero_chain_{i}_pc30_gamma{gam:g}", "numbers": z.tolist(),
                      "positions": x.reshape(-1).tolist(), "charge": 0.0, "uhf": 0,
                      "pc_positions": (c0 + d * r[:, None]).reshape(-1).tolist(),
                      "pc_charges": q.tolist(), "pc_gammas": [gam] * npc})
    b2 = W.config2(2)
    for i in range(2):
        z, x = W.molecule(b2, i)
        p0, p1 = int(b2.point_charge_offsets[i]), int(b2.point_charge_offsets[i + 1])
        cases.append({"name": f"c20h42_pc200_{i}", "numbers": z.tolist(), "positions": x.reshape(-1).tolist(),
                      "charge": 0.0, "uhf": 0,
                      "pc_positions": b2.point_charge_positions[3 * p0:3 * p1].tolist(),
                      "pc_charges": b2.point_charge_values[p0:p1].tolist(),
                      "pc_gammas": b2.point_charge_gammas[p0:p1].tolist()})
    return cases


def pc_batch(cases):
    b = abi.ragged_from_lists([np.asarray(c["numbers"], np.int32) for c in cases],
                              [np.asarray(c["positions"]) for c in cases],
                              [c["charge"] for c in cases], [c["uhf"] for c in cases])
    counts = [len(c["pc_charges"]) for c in cases]
    b.point_charge_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    b.point_charge_positions = np.ascontiguousarray(np.concatenate([c["pc_positions"] for c in cases]), float)
    b.point_charge_values = np.ascontiguousarray(np.concatenate([c["pc_charges"] for c in cases]), float)
    b.point_charge_gammas = np.ascontiguousarray(np.concatenate([c["pc_gammas"] for c in cases]), float)
    return b


def main_pc(ref: Path):
    lib = abi.Library(str(ROOT / "oracle/_ref/libxtbloom_ref.so"), backend=abi.BACKEND_CPU, cpu_threads=1)
    cases = pc_cases(ref)
    for c in cases:
        b = pc_batch([c])
        r = lib.compute(b, lib.make_options(flags=abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES
                                            | abi.COMPUTE_CHARGES | abi.COMPUTE_POINT_CHARGE_FORCES))
        c.update(status=int(r["per_system_status"][0]), energy=float(r["energies"][0]),
                 forces=r["forces"].tolist(), charges=r["atomic_charges"].tolist(),
                 pc_forces=r["point_charge_forces"].tolist(), scc_iterations=int(r["scc_iterations"][0]))
    (HERE / "pc_fixtures.json").write_text(json.dumps(
        {"source": "reference library built from its sources (oracle/ref.mk), FP64, cpu_threads=1; "
                   "xtb_* fields: the reference's xTB 6.7.1 QM/MM goldens (data/conformance/golden), tolerance 5e-7",
         "systems": cases}, indent=0))



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
    main_pc(reference_checkout())
