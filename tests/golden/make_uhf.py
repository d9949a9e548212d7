"""Golden outputs for unrestricted (two spin channel) GFN2 systems.

Runs the reference library (built from the reference sources by
``oracle/ref.mk`` into ``oracle/_ref/libxtbloom_ref.so``) with
spin_channels = 2 on
  * the OH radical of the reference's tblite UHF SCC trace
    (``data/conformance/scc-traces/oh_radical.json``; its final charges are
    stored beside the library's for the pin test), and
  * twelve doublet radicals of ``workloads.config4(2048, seed=4)`` (alkyl
    radicals C4..C45, some with Cl/Br), chosen to span the sizes and to
    include halogens,
and stores energies, forces, charges and SCC iteration counts, at the
default SCC settings and converged to the fixed point (charge tolerance
1e-10, energy tolerance 1e-13: ``tight_*``).  The radical inputs are
regenerated from the seed by the tests.

Usage:  python tests/golden/make_uhf.py <reference checkout>  (or set XTBLOOM_REFERENCE_SRC)
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


def run(lib, b):
    r = lib.compute(b)
    t = lib.compute(b, lib.make_options(ctol=1e-10, etol=1e-13))
    return {"status": int(r["per_system_status"][0]), "scc_iterations": int(r["scc_iterations"][0]),
            "energy": float(r["energies"][0]), "forces": r["forces"].tolist(),
            "charges": r["atomic_charges"].tolist(),
            "tight_status": int(t["per_system_status"][0]), "tight_energy": float(t["energies"][0]),
            "tight_forces": t["forces"].tolist(), "tight_charges": t["atomic_charges"].tolist()}


def main(ref: Path):
    lib = abi.Library(str(ROOT / "oracle" / "_ref" / "libxtbloom_ref.so"), backend=abi.BACKEND_CPU,
                      cpu_threads=0)
    trace = json.loads((ref / "data" / "conformance" / "scc-traces" / "oh_radical.json").read_text())
    inp = trace["input"]
    z = np.asarray(inp["atomic_numbers"], np.int32)
    x = np.asarray(inp["positions"], float).reshape(-1, 3)
    oh = abi.ragged_from_lists([z], [x], [inp["molecular_charge"]], [inp["unpaired_electrons"]],
                               [inp["spin_channels"]])
    out = {"oh_radical": dict(run(lib, oh), numbers=z.tolist(), positions=x.reshape(-1).tolist(),
                              tblite_final_charges=trace["iterations"][-1]["raw_qat"][0],
                              tblite_iterations=int(trace["terminal"]["iterations"]))}
    b = W.config4(2048, seed=4)
    n = np.diff(b.atom_offsets)
    halo = [i for i in range(b.batch_size)
            if np.isin(W.molecule(b, i)[0], [17, 35]).any()]
    order = np.argsort(n, kind="stable")
    picks = [int(order[0]), int(order[1]), int(order[len(order) // 3]), int(order[len(order) // 2]),
             int(order[-2]), int(order[-1])] + halo[:6]
    rad = []
    for i in picks:
        r = run(lib, W.subset(b, [i]))
        r["index"] = i
        rad.append(r)
        print(i, n[i], r["status"], r["scc_iterations"], r["energy"], flush=True)
    out["radicals"] = {"workload": "config4(2048, seed=4)", "systems": rad}
    (HERE / "uhf_fixtures.json").write_text(json.dumps(out))



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
