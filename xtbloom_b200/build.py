"""Build the sm_100a CUDA library ``libxtbloom_b200.so`` in-tree.

Steps: (1) turn ``data/params.npz`` into ``csrc/generated/params.inc``
(plain C arrays compiled into the library), (2) compile every ``csrc/*.cu``
and ``csrc/*.cpp`` with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
and link one shared library with the CUDA runtime linked statically.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
GEN = CSRC / "generated"
OBJ = PKG / "_build"
LIB = PKG / "libxtbloom_b200.so"
ROOT = PKG.parent
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-I", str(ROOT / "include"), "-I", str(CSRC)]


def _array(name: str, arr: np.ndarray, ctype: str) -> str:
    flat = np.asarray(arr).ravel()
    if ctype == "double":
        body = ",".join(repr(float(x)) for x in flat)
    else:
        body = ",".join(str(int(x)) for x in flat)
    return f"static const {ctype} {name}[{flat.size}] = {{{body}}};\n"


def generate_params_header() -> Path:
    GEN.mkdir(parents=True, exist_ok=True)
    out = GEN / "params.inc"
    src = PKG / "data" / "params.npz"
    if out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    p = np.load(src)
    parts = ["/* Generated from xtbloom_b200/data/params.npz by build.py; do not edit. */\n"]
    for k in p.files:
        a = p[k]
        ctype = "int" if a.dtype.kind in "iu" else "double"
        parts.append(_array("kP_" + k, a, ctype))
    out.write_text("".join(parts))
    return out


def _compile(src: Path) -> Path:
    OBJ.mkdir(exist_ok=True)
    obj = OBJ / (src.name + ".o")
    deps = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [GEN / "params.inc"] \
        + list((ROOT / "include").glob("*.h"))
    newest = max(d.stat().st_mtime for d in deps + [src])
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd += ["-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed for {src.name}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    generate_params_header()
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
               "-Xlinker", "--exclude-libs,ALL", "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
