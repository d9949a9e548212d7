"""Golden fixtures of the GFN1-xTB path.

Two sources, both produced in the container that holds the reference checkout:
  * ``tblite`` entries: the reference's committed GFN1 conformance goldens
    (``data/conformance/gfn1/golden/*.json``: xTB 6.7.1 / tblite energies,
    forces and charges, tolerance 5e-7) for its six molecular cases, with
    their coordinates (``data/conformance/gfn1/inputs/*.coord``).
  * ``reference`` entries: the reference library itself (built from its
    sources by ``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) with
    model GFN1 on those six cases, on ten closed-shell hetero-alkane chains of
    the 4096-system workload (seed 1), and on twelve radicals of the 2048-radical
    GFN1 workload (seed 4; spin-polarised, two spin channels), at the default
    SCC settings and converged to the fixed point (charge tolerance 1e-10,
    energy tolerance 1e-13).

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
    (HERE / "gfn1_fixtures.json").write_text(json.dumps({"tblite": tblite, "reference": refs}))


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
