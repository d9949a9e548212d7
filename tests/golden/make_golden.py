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

Usage:  python tests/golden/make_golden.py /root/reference
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
       "zn": 30, "i": 53, "rn": 86}


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


if __name__ == "__main__":
    main(Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
