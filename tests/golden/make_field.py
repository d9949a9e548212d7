"""Golden outputs for systems in a uniform electric field, and dipole moments.

Runs the reference library (built from the reference sources by
``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) with
electric-field interaction attachments (block_version 1) on
  * the reference's ``water_efield`` conformance case (coordinates of
    ``data/conformance/inputs/water_efield.coord``, field (0.003, -0.004,
    0.005) Eh/(e bohr)); its committed tblite energy is stored beside the
    library's outputs for the pin test,
  * six of the restricted reference fixtures and two radicals of
    ``workloads.config4(2048, seed=4)`` with seeded random fields of
    |E| <= 0.01, and the same molecules without a field,
storing energies, forces, charges, dipole moments and SCC iteration counts.

Usage:  python tests/golden/make_field.py <reference checkout>  (or set XTBLOOM_REFERENCE_SRC)
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

FLAGS = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES | abi.COMPUTE_CHARGES | abi.COMPUTE_DIPOLES


def run(lib, mols, fields):
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols], [m[2] for m in mols],
                              [m[3] for m in mols], [m[4] for m in mols])
    b.efields = None if fields is None else np.asarray(fields, float)
    nb, na = b.batch_size, b.total_atoms
    out = {"energies": np.empty(nb), "forces": np.empty(3 * na), "atomic_charges": np.empty(na),
           "dipole_moments": np.empty(3 * nb), "scc_iterations": np.empty(nb, np.int32),
           "scc_converged": np.empty(nb, np.uint8), "per_system_status": np.empty(nb, np.int32)}
    return b, lib.compute(b, lib.make_options(flags=FLAGS), out)


def main(ref: Path):
    lib = abi.Library(str(ROOT / "oracle" / "_ref" / "libxtbloom_ref.so"), backend=abi.BACKEND_CPU,
                      cpu_threads=0)
    gold = json.loads((ref / "data" / "conformance" / "golden" / "water_efield.json").read_text())
    z, x = [], []
    for line in (ref / "data" / "conformance" / "inputs" / "water_efield.coord").read_text().splitlines():
        p = line.split()
        if len(p) == 4 and p[3].isalpha():
            x.append([float(v) for v in p[:3]])
            z.append({"o": 8, "h": 1}[p[3].lower()])
    fixtures = json.loads((HERE / "reference_fixtures.json").read_text())["systems"]
    uhf = json.loads((HERE / "uhf_fixtures.json").read_text())["radicals"]["systems"]
    mols = [(np.asarray(z, np.int32), np.asarray(x), 0.0, 0, 1)]
    names = ["water_efield"]
    for s in fixtures[:6]:
        mols.append((np.asarray(s["numbers"], np.int32), np.asarray(s["positions"]).reshape(-1, 3),
                     float(s["charge"]), int(s["uhf"]), 1))
        names.append(s["name"])
    full = W.config4(2048, seed=4)
    for c in uhf[:2]:
        zz, xx = W.molecule(full, c["index"])
        mols.append((zz, xx, 0.0, 1, 2))
        names.append(f"radical_{c['index']}")
    rng = np.random.default_rng(5)
    fields = [[0.003, -0.004, 0.005]] + [list(rng.uniform(-0.006, 0.006, 3)) for _ in mols[1:]]
    systems = []
    for label, fl in (("field", fields), ("no_field", None)):
        b, out = run(lib, mols, fl)
        for i, name in enumerate(names):
            a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
            systems.append({"name": name, "case": label, "field": None if fl is None else fl[i],
                            "numbers": mols[i][0].tolist(), "positions": mols[i][1].reshape(-1).tolist(),
                            "charge": mols[i][2], "uhf": mols[i][3], "spin_channels": mols[i][4],
                            "status": int(out["per_system_status"][i]),
                            "scc_iterations": int(out["scc_iterations"][i]),
                            "energy": float(out["energies"][i]),
                            "forces": out["forces"][3 * a0:3 * a1].tolist(),
                            "charges": out["atomic_charges"][a0:a1].tolist(),
                            "dipole": out["dipole_moments"][3 * i:3 * i + 3].tolist()})
    out = {"tblite_water_efield_energy": gold["properties"]["energy_hartree"], "systems": systems}
    (HERE / "field_fixtures.json").write_text(json.dumps(out))
    for s in systems:
        print(s["case"], s["name"], s["status"], s["scc_iterations"], round(s["energy"], 8), np.round(s["dipole"], 4))



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
