"""Generate the packed parameter tables used by the library and the oracle.

The GFN2-xTB element/shell parameters (tblite 0.7.0 export), the Stewart
STO-nG expansion tables, the D4 reference tables (dftd4) and the two mctc-lib
radius tables are read from the reference checkout's published data files
(``data/parameters/gfn2.json``, ``tblite_sto.hpp``, ``d4.hpp``,
``tblite_spin.hpp``) and from the
two small radius tables in ``src/model/gfn2/h0.cpp`` and
``src/model/gfn2/coordination.cpp``.  Nothing is typed in by hand: every
number is parsed from those files and written to ``params.npz`` beside this
script.  The data are LGPL-3.0-or-later (tblite, dftd4) and Apache-2.0
(mctc-lib); see ``LICENSES.md`` in this directory.

Usage:  python -m xtbloom_b200.data.generate_params /path/to/reference
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def _numbers(text: str) -> list[float]:
    return [float(x) for x in re.findall(NUM, text)]


def _block(text: str, name: str) -> str:
    """Body of ``... name{{ ... }};`` in a generated C++ header."""
    start = text.index(name + "{{")
    end = text.index("}};", start)
    return text[start + len(name) + 2:end]


def _std_array_block(text: str, name: str) -> str:
    start = text.index(name)
    brace = text.index("{{", start)
    end = text.index("}};", brace)
    return text[brace + 2:end]


def gfn2_tables(ref: Path) -> dict[str, np.ndarray]:
    d = json.loads((ref / "data/parameters/gfn2.json").read_text())
    els = d["elements"]
    assert [e["atomic_number"] for e in els] == list(range(1, 87))
    nz = 86
    max_sh = 3
    out: dict[str, np.ndarray] = {}
    nsh = np.zeros(nz, np.int32)
    shl = np.full((nz, max_sh), -1, np.int32)
    shn = np.zeros((nz, max_sh), np.int32)
    shng = np.zeros((nz, max_sh), np.int32)
    f = {k: np.zeros((nz, max_sh)) for k in (
        "level", "kcn", "shpoly", "slater", "refocc", "hubbard_scale")}
    keymap = {"level": "level", "kcn": "coordination_number_scale",
              "shpoly": "shell_polynomial", "slater": "slater",
              "refocc": "reference_occupation", "hubbard_scale": "shell_hubbard_scale"}
    for zi, e in enumerate(els):
        nsh[zi] = len(e["shells"])
        for si, s in enumerate(e["shells"]):
            assert s["index"] == si
            shl[zi, si] = s["angular_momentum"]
            shn[zi, si] = s["principal_quantum_number"]
            shng[zi, si] = s["ngauss"]
            for k, j in keymap.items():
                f[k][zi, si] = s[j]
    out["gfn2_nshell"] = nsh
    out["gfn2_shell_l"] = shl
    out["gfn2_shell_n"] = shn
    out["gfn2_shell_ngauss"] = shng
    for k, v in f.items():
        out["gfn2_shell_" + k] = v
    for k in ("gam", "gam3", "arep", "zeff", "en", "mprad", "mpvcn", "dkernel", "qkernel"):
        out["gfn2_" + k] = np.array([e[k] for e in els], float)
    h = d["hamiltonian"]
    assert h["coordination_number"] == "dexp" and not h["pair_scale_overrides"]
    sps = np.zeros((3, 3))
    for item in h["shell_pair_scale"]:
        a, b = item["angular_momenta"]
        sps[a, b] = sps[b, a] = item["value"]
    out["gfn2_shell_pair_scale"] = sps
    out["gfn2_globals"] = np.array([
        h["wexp"], h["enscale"], h["kpol"], h["pair_scale_default"],
        d["repulsion"]["kexp"], d["repulsion"]["klight"],
        d["thirdorder"]["s"], d["thirdorder"]["p"], d["thirdorder"]["d"],
        d["multipole"]["dmp3"], d["multipole"]["dmp5"], d["multipole"]["kexp"],
        d["multipole"]["shift"], d["multipole"]["rmax"],
        d["dispersion"]["a1"], d["dispersion"]["a2"], d["dispersion"]["s6"],
        d["dispersion"]["s8"], d["dispersion"]["s9"], d["charge"]["gexp"],
    ])
    assert d["charge"]["average"] == "arithmetic"
    assert d["dispersion"]["self_consistent"] and not d["dispersion"]["smooth"]
    return out


GLOBAL_NAMES = ["wexp", "enscale", "kpol", "pair_scale_default", "rep_kexp",
                "rep_klight", "es3_s", "es3_p", "es3_d", "mp_dmp3", "mp_dmp5",
                "mp_kexp", "mp_shift", "mp_rmax", "d4_a1", "d4_a2", "d4_s6",
                "d4_s8", "d4_s9", "es2_gexp"]


def sto_tables(ref: Path) -> dict[str, np.ndarray]:
    t = (ref / "data/parameters/tblite_sto.hpp").read_text()
    out = {}
    for ng in (3, 4, 6):
        a = np.array(_numbers(_block(t, f"kAlpha{ng}")))
        c = np.array(_numbers(_block(t, f"kCoeff{ng}")))
        out[f"sto_alpha{ng}"] = a.reshape(15, ng)
        out[f"sto_coeff{ng}"] = c.reshape(15, ng)
    for name in ("kAlpha6s", "kCoeff6s", "kAlpha6p", "kCoeff6p"):
        v = np.array(_numbers(_block(t, name)))
        assert v.size == 6
        out["sto_" + name[1:].lower()] = v
    return out


def radius_tables(ref: Path) -> dict[str, np.ndarray]:
    h0 = (ref / "src/model/gfn2/h0.cpp").read_text()
    cn = (ref / "src/model/gfn2/coordination.cpp").read_text()
    ar = np.array(_numbers(_block(h0, "kAtomicRadiiAngstrom")))
    cr = np.array(_numbers(_block(cn, "kCovalentRadiiAngstrom")))
    assert ar.size == 86 and cr.size == 86
    return {"atomic_radii_angstrom": ar, "covalent_radii_angstrom": cr}


def d4_tables(ref: Path) -> dict[str, np.ndarray]:
    t = (ref / "data/parameters/d4.hpp").read_text()
    el = re.findall(r"D4ElementData\{([^}]*)\}", _block(t, "kElements"))
    rf = re.findall(r"D4ReferenceData\{([^}]*)\}", _block(t, "kReferences"))
    el = np.array([_numbers(x) for x in el])
    rf = np.array([_numbers(x) for x in rf])
    c6 = np.array(_numbers(_block(t, "kReferenceC6")))
    assert el.shape == (86, 7) and rf.shape == (262, 3) and c6.size == 262 * 262
    return {
        "d4_ref_offset": el[:, 0].astype(np.int32),
        "d4_ref_count": el[:, 1].astype(np.int32),
        "d4_rcov": el[:, 2], "d4_en": el[:, 3], "d4_zeff": el[:, 4],
        "d4_eta": el[:, 5], "d4_r4r2": el[:, 6],
        "d4_ref_cn": rf[:, 0], "d4_ref_q": rf[:, 1],
        "d4_ref_ngauss": rf[:, 2].astype(np.int32),
        "d4_ref_c6": c6.reshape(262, 262),
    }


def spin_tables(ref: Path) -> dict[str, np.ndarray]:
    """Element spin constants W_ll' (ss, sp, pp, sd, pd, dd; Hartree) of tblite,
    parsed from ``data/parameters/tblite_spin.hpp``."""
    text = (ref / "data" / "parameters" / "tblite_spin.hpp").read_text()
    start = text.index("kSpinConstants{{")
    body = text[start + len("kSpinConstants{{"):text.index("}};", start)]
    vals = np.array(_numbers(body), float)
    return {"spin_constants": vals.reshape(86, 6)}


def generate(ref: Path, out: Path) -> None:
    tables: dict[str, np.ndarray] = {}
    tables.update(gfn2_tables(ref))
    tables.update(sto_tables(ref))
    tables.update(radius_tables(ref))
    tables.update(d4_tables(ref))
    tables.update(spin_tables(ref))
    np.savez_compressed(out, **tables)


if __name__ == "__main__":
    reference = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    generate(reference, Path(__file__).with_name("params.npz"))
