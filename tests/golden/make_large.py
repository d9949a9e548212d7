"""Golden outputs for large systems: water clusters of the 256-cluster workload.

Runs the reference library (built from the reference sources by
``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) on three clusters of
``workloads.config3(256, seed=3)`` -- (H2O)_N with N = 100..200 waters,
600..1200 AOs -- and stores their energies, forces, charges and SCC
iteration counts, at the default SCC settings and converged to the fixed
point (charge tolerance 1e-10, energy tolerance 1e-13).  The inputs are
regenerated from the seed by the tests.

Usage:  python tests/golden/make_large.py
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


def main():
    b = W.config3(256, seed=3)
    waters = np.diff(b.atom_offsets) // 3
    order = np.argsort(waters, kind="stable")
    picks = [int(order[0]), int(order[len(order) // 4]), int(order[-1])]
    lib = abi.Library(str(ROOT / "oracle" / "_ref" / "libxtbloom_ref.so"), backend=abi.BACKEND_CPU,
                      cpu_threads=0)
    tight = lib.make_options(ctol=1e-10, etol=1e-13)
    out = []
    for i in picks:
        r = lib.compute(W.subset(b, [i]))
        t = lib.compute(W.subset(b, [i]), tight)
        out.append({"workload": "config3(256, seed=3)", "index": i, "waters": int(waters[i]),
                    "status": int(r["per_system_status"][0]),
                    "scc_iterations": int(r["scc_iterations"][0]),
                    "energy": float(r["energies"][0]), "forces": r["forces"].tolist(),
                    "charges": r["atomic_charges"].tolist(),
                    "tight_status": int(t["per_system_status"][0]),
                    "tight_energy": float(t["energies"][0]), "tight_forces": t["forces"].tolist(),
                    "tight_charges": t["atomic_charges"].tolist()})
        print(i, waters[i], out[-1]["status"], out[-1]["scc_iterations"], out[-1]["energy"], flush=True)
    (HERE / "large_fixtures.json").write_text(json.dumps({"systems": out}))


if __name__ == "__main__":
    main()
