"""Large systems: water clusters of 600-1200 AOs against the reference library.

Exercises the eigensolver paths for matrices that do not fit one CTA's shared
memory (global-memory Householder prefix, back-transform and inverse
iteration at n up to 1200), in one ragged batch.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, TOL_E, TOL_F, TOL_Q
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_water_clusters_match_reference(cuda_lib):
    cases = json.loads((GOLDEN / "large_fixtures.json").read_text())["systems"]
    full = W.config3(256, seed=3)
    b = W.subset(full, [c["index"] for c in cases])
    out = cuda_lib.compute(b)
    for i, c in enumerate(cases):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert a1 - a0 == 3 * c["waters"]
        assert out["per_system_status"][i] == c["status"] == 0
        assert abs(out["energies"][i] - c["energy"]) < TOL_E, (i, out["energies"][i], c["energy"])
        assert np.abs(out["forces"][3 * a0:3 * a1] - np.asarray(c["forces"])).max() < TOL_F
        assert np.abs(out["atomic_charges"][a0:a1] - np.asarray(c["charges"])).max() < TOL_Q
        assert abs(int(out["scc_iterations"][i]) - c["scc_iterations"]) <= 1
