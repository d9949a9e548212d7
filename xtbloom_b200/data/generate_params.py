"""Generate the packed parameter tables used by the library and the oracle.

The GFN2-xTB and GFN1-xTB element/shell parameters (tblite exports), the
Stewart STO-nG expansion tables (and the legacy STO-6G 4s/4p rows of GFN1),
the D4 reference tables (dftd4), the D3 reference tables (simple-dftd3) and
the two mctc-lib radius tables are read from the reference checkout's
published data files (``data/parameters/gfn2.json``, ``gfn1.json``,
``gfn1_d3.json``, ``gfn1_legacy_sto.hpp``, ``tblite_sto.hpp``, ``d4.hpp``,
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


def gfn1_tables(ref: Path) -> dict[str, np.ndarray]:
    """GFN1-xTB element, shell and global parameters (tblite export,
    ``data/parameters/gfn1.json``); shell levels and CN scales stay in eV."""
    d = json.loads((ref / "data/parameters/gfn1.json").read_text())
    els = d["elements"]
    assert [e["atomic_number"] for e in els] == list(range(1, 87))
    nz, max_sh = 86, 3
    out: dict[str, np.ndarray] = {}
    nsh = np.zeros(nz, np.int32)
    ints = {k: np.full((nz, max_sh), -1 if k == "l" else 0, np.int32) for k in ("l", "n", "ngauss", "valence")}
    f = {k: np.zeros((nz, max_sh)) for k in ("level", "kcn", "shpoly", "slater", "refocc", "hubbard_scale")}
    keymap = {"level": "level", "kcn": "coordination_number_scale", "shpoly": "shell_polynomial",
              "slater": "slater", "refocc": "reference_occupation", "hubbard_scale": "shell_hubbard_scale"}
    for zi, e in enumerate(els):
        nsh[zi] = len(e["shells"])
        assert nsh[zi] <= max_sh
        for si, sh in enumerate(e["shells"]):
            assert sh["index"] == si
            ints["l"][zi, si] = sh["angular_momentum"]
            ints["n"][zi, si] = sh["principal_quantum_number"]
            ints["ngauss"][zi, si] = sh["ngauss"]
            ints["valence"][zi, si] = 1 if sh["is_valence"] else 0
            for k, j in keymap.items():
                f[k][zi, si] = sh[j]
    out["gfn1_nshell"] = nsh
    for k, v in ints.items():
        out["gfn1_shell_" + k] = v
    for k, v in f.items():
        out["gfn1_shell_" + k] = v
    for k, j in (("gam", "gam"), ("gam3", "gam3"), ("arep", "arep"), ("zeff", "zeff"), ("en", "en"),
                 ("xbond", "xbond"), ("atomic_radius", "atomic_radius_bohr"),
                 ("covalent_radius", "covalent_radius_bohr")):
        out["gfn1_" + k] = np.array([e[j] for e in els], float)
    h = d["hamiltonian"]
    assert h["coordination_number"] == "exp"
    sps = np.zeros((3, 3))
    for item in h["shell_pair_scale"]:
        a, b = item["angular_momenta"]
        sps[a, b] = sps[b, a] = item["value"]
    out["gfn1_shell_pair_scale"] = sps
    kpair = np.full((nz, nz), h["pair_scale_default"])
    for item in h["pair_scale_overrides"]:
        a, b = item["atomic_numbers"]
        kpair[a - 1, b - 1] = kpair[b - 1, a - 1] = item["value"]
    out["gfn1_kpair"] = kpair
    cn = d["coordination_number"]
    assert cn["model"] == "exp" and d["charge"]["average"] == "harmonic"
    assert d["thirdorder"]["mode"] == "atom" and d["dispersion"]["model"] == "d3"
    out["gfn1_globals"] = np.array([
        h["kpol"], h["enscale"], d["repulsion"]["kexp"], d["repulsion"]["klight"],
        d["dispersion"]["a1"], d["dispersion"]["a2"], d["dispersion"]["s6"], d["dispersion"]["s8"],
        d["dispersion"]["s9"], d["halogen"]["damping"], d["halogen"]["radius_scale"],
        cn["steepness"], cn["cutoff_bohr"], d["charge"]["gexp"],
    ])
    return out


GFN1_GLOBAL_NAMES = ["kpol", "enscale", "rep_kexp", "rep_klight", "d3_a1", "d3_a2", "d3_s6",
                     "d3_s8", "d3_s9", "xb_damping", "xb_radius_scale", "cn_steepness",
                     "cn_cutoff", "es2_gexp"]


def gfn1_sto_tables(ref: Path) -> dict[str, np.ndarray]:
    """The legacy STO-6G 4s/4p rows GFN1 uses (``gfn1_legacy_sto.hpp``)."""
    t = (ref / "data/parameters/gfn1_legacy_sto.hpp").read_text()
    out = {}
    for name, key in (("kLegacyAlpha6_4sp", "alpha"), ("kLegacyCoeff6_4s", "coeff_s"),
                      ("kLegacyCoeff6_4p", "coeff_p")):
        v = np.array(_numbers(_std_array_block(t, name)))
        assert v.size == 6
        out["gfn1_sto6_4sp_" + key] = v
    return out


def d3_tables(ref: Path) -> dict[str, np.ndarray]:
    """DFT-D3 reference data of GFN1 (simple-dftd3 export, ``gfn1_d3.json``):
    per element the reference CNs; the reference C6 of every pair of
    references, expanded into one symmetric table over all 237 references."""
    d = json.loads((ref / "data/parameters/gfn1_d3.json").read_text())
    els = d["elements"]
    cnt = np.array([e["reference_count"] for e in els], np.int32)
    off = np.array([e["reference_offset"] for e in els], np.int32)
    nref = int(cnt.sum())
    c6 = np.array(d["c6"], float)
    table = np.zeros((nref, nref))
    for z2 in range(1, 87):
        for z1 in range(1, z2 + 1):
            pr = d["pair_records"][(z1 - 1) + z2 * (z2 - 1) // 2]
            assert pr["first_reference_count"] == cnt[z1 - 1] and pr["second_reference_count"] == cnt[z2 - 1]
            for i in range(cnt[z1 - 1]):
                for j in range(cnt[z2 - 1]):
                    v = c6[pr["c6_offset"] + j * cnt[z1 - 1] + i]
                    table[off[z1 - 1] + i, off[z2 - 1] + j] = v
                    table[off[z2 - 1] + j, off[z1 - 1] + i] = v
    return {"d3_ref_count": cnt, "d3_ref_offset": off,
            "d3_ref_cn": np.array(d["coordination_numbers"], float),
            "d3_r4r2": np.array(d["r4r2"], float), "d3_ref_c6": table}


def generate(ref: Path, out: Path) -> None:
    tables: dict[str, np.ndarray] = {}
    tables.update(gfn2_tables(ref))
    tables.update(sto_tables(ref))
    tables.update(radius_tables(ref))
    tables.update(d4_tables(ref))
    tables.update(spin_tables(ref))
    tables.update(gfn1_tables(ref))
    tables.update(gfn1_sto_tables(ref))
    tables.update(d3_tables(ref))
    np.savez_compressed(out, **tables)



def reference_checkout() -> Path:
    """The reference checkout: the first argument, else $XTBLOOM_REFERENCE_SRC."""
    import os
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XTBLOOM_REFERENCE_SRC")
    if not arg:
        sys.exit("usage: pass the reference checkout as the first argument "
                 "or set XTBLOOM_REFERENCE_SRC")
    return Path(arg)

if __name__ == "__main__":
    reference = reference_checkout()
    generate(reference, Path(__file__).with_name("params.npz"))
