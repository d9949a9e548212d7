"""Golden outputs for the charge response b + A q (periodic QM/MM coupling).

Runs the reference library (built from the reference sources by
``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) on six restricted
reference fixtures and two radicals of ``workloads.config4(2048, seed=4)``
with seeded per-atom shifts b ~ N(0, 0.01) Eh/e and symmetric per-system
response blocks A = (M + M^T)/2, M ~ N(0, 0.02), storing energies, forces,
charges, SCC iteration counts and the inputs b, A.

Usage:  python tests/golden/make_response.py
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
    lib = abi.Library(str(ROOT / "oracle" / "_ref" / "libxtbloom_ref.so"), backend=abi.BACKEND_CPU,
                      cpu_threads=0)
    fixtures = json.loads((HERE / "reference_fixtures.json").read_text())["systems"]
    uhf = json.loads((HERE / "uhf_fixtures.json").read_text())["radicals"]["systems"]
    mols = [(np.asarray(s["numbers"], np.int32), np.asarray(s["positions"]).reshape(-1, 3),
             float(s["charge"]), int(s["uhf"]), 1, s["name"]) for s in fixtures[:6]]
    full = W.config4(2048, seed=4)
    for c in uhf[:2]:
        z, x = W.molecule(full, c["index"])
        mols.append((z, x, 0.0, 1, 2, f"radical_{c['index']}"))
    rng = np.random.default_rng(7)
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols], [m[2] for m in mols],
                              [m[3] for m in mols], [m[4] for m in mols])
    na = np.diff(b.atom_offsets)
    shifts = rng.normal(0.0, 0.01, b.total_atoms)
    blocks = []
    for n in na:
        M = rng.normal(0.0, 0.02, (n, n))
        blocks.append((0.5 * (M + M.T)).ravel())
    b.atomic_potential_shifts = shifts
    b.charge_response_offsets = np.concatenate([[0], np.cumsum(na * na)]).astype(np.int64)
    b.charge_response_matrix = np.concatenate(blocks)
    out = lib.compute(b)
    systems = []
    for i, m in enumerate(mols):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        systems.append({"name": m[5], "numbers": m[0].tolist(), "positions": m[1].reshape(-1).tolist(),
                        "charge": m[2], "uhf": m[3], "spin_channels": m[4],
                        "shifts": shifts[a0:a1].tolist(), "response": blocks[i].tolist(),
                        "status": int(out["per_system_status"][i]),
                        "scc_iterations": int(out["scc_iterations"][i]),
                        "energy": float(out["energies"][i]),
                        "forces": out["forces"][3 * a0:3 * a1].tolist(),
                        "charges": out["atomic_charges"][a0:a1].tolist()})
        print(m[5], systems[-1]["status"], systems[-1]["scc_iterations"], systems[-1]["energy"])
    print("result flags", lib.last_result_flags)
    (HERE / "response_fixtures.json").write_text(json.dumps({"systems": systems}))


if __name__ == "__main__":
    main()
