"""Shared fixtures; the ``gpu`` marker selects tests that need a B200."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"
REF_LIB = ROOT / "oracle" / "_ref" / "libxtbloom_ref.so"

# Public tolerances of the path (energy, force, charge).
TOL_E = 1e-6
TOL_F = 1e-5
TOL_Q = 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")


@pytest.fixture(scope="session")
def fixtures():
    return json.loads((GOLDEN / "reference_fixtures.json").read_text())["systems"]


@pytest.fixture(scope="session")
def pc_fixtures():
    return json.loads((GOLDEN / "pc_fixtures.json").read_text())["systems"]


def as_pc(sys_):
    return (np.asarray(sys_["pc_positions"], float).reshape(-1, 3), np.asarray(sys_["pc_charges"], float),
            np.asarray(sys_["pc_gammas"], float))


@pytest.fixture(scope="session")
def tblite_goldens():
    return json.loads((GOLDEN / "tblite_goldens.json").read_text())["cases"]


@pytest.fixture(scope="session")
def cuda_lib():
    from xtbloom_b200 import abi, library_path
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=0)
    yield lib
    lib.close()


def as_molecule(sys_):
    return (np.asarray(sys_["numbers"], np.int32), np.asarray(sys_["positions"], float).reshape(-1, 3),
            float(sys_["charge"]), int(sys_["uhf"]))
