"""Drop-in check: the reference's own Python package over this library.

The reference's ``xtbloom`` package (python/xtbloom, loaded unchanged from the
reference checkout) binds its native core through ``XTBLOOM_LIBRARY``
(python/xtbloom/library.py:346-383).  Pointed at this project's
``libxtbloom_b200.so`` it must load it, find every symbol group it probes
(the request ABI, compute options v3), and run its own tests
(python/tests/test_library.py, test_interface.py, test_batch.py) with the
same outcome as over the reference library itself -- except that a compute
needs a B200: on a machine without one, every compute test must fail with
the library's BACKEND_UNAVAILABLE status (there is no CPU fallback), and
nothing else may fail.

The package reads its version from installed distribution metadata, so the
test gives it a minimal ``xtbloom`` metadata directory on the path; the
reference tree itself is only read.  Skipped when the reference checkout is
absent ($XTBLOOM_REFERENCE_SRC, else the build's default location).
"""
from __future__ import annotations

import os
import subprocess
import sys
import xml.etree.ElementTree as ET
from pathlib import Path

import pytest

from conftest import REF_LIB, ROOT

sys.path.insert(0, str(ROOT))
from __graft_entry__ import REFERENCE  # noqa: E402

PKG = REFERENCE / "python"
TESTS = ["test_library.py", "test_interface.py", "test_batch.py"]
OURS = ROOT / "xtbloom_b200" / "libxtbloom_b200.so"

pytestmark = pytest.mark.skipif(not (PKG / "xtbloom" / "library.py").exists() or not OURS.exists(),
                                reason="reference checkout or built library absent")


def metadata_dir(tmp: Path) -> Path:
    d = tmp / "meta" / "xtbloom-0.0.0.dist-info"
    d.mkdir(parents=True)
    (d / "METADATA").write_text("Metadata-Version: 2.1\nName: xtbloom\nVersion: 0.0.0\n")
    return tmp / "meta"


def run_reference_tests(lib: Path, tmp: Path, tag: str) -> dict:
    """Outcome per test id: None (passed or skipped) or the failure message."""
    xml = tmp / f"{tag}.xml"
    env = dict(os.environ, XTBLOOM_LIBRARY=str(lib),
               PYTHONPATH=os.pathsep.join([str(metadata_dir(tmp / tag)), str(PKG)]))
    subprocess.run([sys.executable, "-m", "pytest", "-p", "no:cacheprovider", "-q",
                    f"--junitxml={xml}", *[str(PKG / "tests" / t) for t in TESTS]],
                   env=env, cwd=tmp, capture_output=True, timeout=900)
    out = {}
    for tc in ET.parse(xml).iter("testcase"):
        bad = tc.find("failure") if tc.find("failure") is not None else tc.find("error")
        out[f'{tc.get("classname")}::{tc.get("name")}'] = None if bad is None else (bad.get("message") or "")
    return out


def test_reference_package_loads_this_library(tmp_path):
    code = ("import xtbloom.library as L, sys\n"
            "h = L.load_library()\n"
            "print(h._name)\n"
            "print(L.request_api_available(h), L.compute_options_v3_available(h))\n")
    env = dict(os.environ, XTBLOOM_LIBRARY=str(OURS),
               PYTHONPATH=os.pathsep.join([str(metadata_dir(tmp_path)), str(PKG)]))
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    name, flags = r.stdout.strip().splitlines()[-2:]
    assert Path(name).resolve() == OURS.resolve()
    assert flags == "True True"


@pytest.mark.skipif(not REF_LIB.exists(), reason="reference library not built")
def test_reference_python_tests_run_unchanged_against_this_library(tmp_path):
    ref = run_reference_tests(REF_LIB, tmp_path, "ref")
    ours = run_reference_tests(OURS, tmp_path, "ours")
    assert set(ours) == set(ref) and len(ours) >= 60
    gpu_needed = {k for k, v in ours.items() if v is not None and "backend unavailable" in v}
    # everything that passes over the reference library passes here, unless it computes
    regressions = {k: v for k, v in ours.items()
                   if v is not None and ref[k] is None and k not in gpu_needed}
    assert not regressions, regressions
    passed = [k for k, v in ours.items() if v is None]
    assert len(passed) >= 30
    # a compute without a device reports the library's status, never a CPU result
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if not has_gpu:
        assert len(gpu_needed) >= 25
