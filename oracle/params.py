"""Parameter access for the CPU oracle (test infrastructure only).

The oracle reads the same generated tables as the library
(``xtbloom_b200/data/params.npz``), which are parsed from the reference's
published data files by ``xtbloom_b200/data/generate_params.py``.
"""
from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np

PARAMS_PATH = Path(__file__).resolve().parents[1] / "xtbloom_b200" / "data" / "params.npz"

GLOBAL_NAMES = ["wexp", "enscale", "kpol", "pair_scale_default", "rep_kexp",
                "rep_klight", "es3_s", "es3_p", "es3_d", "mp_dmp3", "mp_dmp5",
                "mp_kexp", "mp_shift", "mp_rmax", "d4_a1", "d4_a2", "d4_s6",
                "d4_s8", "d4_s9", "es2_gexp"]

# Unit conversions the reference keeps verbatim for parity
# (src/model/gfn2/h0.cpp:20-21, src/model/gfn2/coordination.cpp:30).
EV_TO_HARTREE = 1.0 / 27.21138505
ANGSTROM_TO_BOHR = 1.8897261246204404
KELVIN_TO_HARTREE = 3.166808578545117e-6


@lru_cache(maxsize=1)
def load() -> dict:
    raw = np.load(PARAMS_PATH)
    p = {k: raw[k] for k in raw.files}
    p["g"] = dict(zip(GLOBAL_NAMES, p["gfn2_globals"].tolist()))
    return p
