"""xtbloom_b200: batched GFN2-xTB single points on NVIDIA B200 (sm_100a).

The compute path is the in-tree CUDA library ``libxtbloom_b200.so`` behind the
versioned caller-buffer C ABI declared in ``include/xtbloom.h``.  This package
is the Python host side: a ctypes binding (``abi``), a ``Calculator`` /
``BatchCalculator`` mirroring the reference's Python interface, and seeded
synthetic workloads.
"""
from __future__ import annotations

from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIBRARY_PATH = PACKAGE_DIR / "libxtbloom_b200.so"


def library_path() -> str:
    """Path of the in-tree CUDA library; raises if it has not been built."""
    if not LIBRARY_PATH.exists():
        raise RuntimeError(
            f"{LIBRARY_PATH} is missing: build it with `python -m xtbloom_b200.build` "
            "(there is no CPU fallback)")
    return str(LIBRARY_PATH)


from .interface import BatchCalculator, Calculator, Result  # noqa: E402

__all__ = ["Calculator", "BatchCalculator", "Result", "library_path", "LIBRARY_PATH"]
