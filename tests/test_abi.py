"""The C-ABI library loads, exports every declared entry point, and validates on the host."""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT
from xtbloom_b200 import abi, library_path

HEADER = ROOT / "include" / "xtbloom.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"XTBLOOM_API[^;(]*?\b(xtbloom_\w+)\s*\(", text, re.S)))


def test_header_declares_the_reference_abi():
    names = declared_symbols()
    for name in abi.ABI_SYMBOLS:
        assert name in names, name


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(library_path())
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_struct_layouts_match_the_reference_abi():
    assert C.sizeof(abi.Batch) == 456
    assert abi.Batch.total_interactions.offset == 352
    assert C.sizeof(abi.ComputeOptions) == 80
    assert C.sizeof(abi.BatchResult) == 280
    assert C.sizeof(abi.ContextOptions) == 32


def test_initialisers_set_reference_defaults():
    lib = abi.bind(library_path())
    o = abi.ComputeOptions()
    assert lib.xtbloom_compute_options_init(C.byref(o), C.sizeof(o)) == abi.SUCCESS
    assert o.struct_size == 80 and o.api_version == 1
    assert o.model == abi.MODEL_GFN2 and o.flags == (abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES)
    assert o.max_scc_iterations == 250 and o.charge_tolerance == 1e-6 and o.energy_tolerance == 1e-8
    assert abs(o.electronic_temperature - 300 * abi.KELVIN_TO_HARTREE) < 1e-18
    assert o.scc_mixer_history == 8 and o.scc_mixer_damping == 0.4
    c = abi.ContextOptions()
    assert lib.xtbloom_context_options_init(C.byref(c), C.sizeof(c)) == abi.SUCCESS
    assert c.device_id == -1 and c.backend == abi.BACKEND_AUTO
    # a too-small structure is rejected
    assert lib.xtbloom_compute_options_init(C.byref(o), 8) == abi.INVALID_ARGUMENT


def test_initialisers_record_the_callers_size():
    """A newer caller's larger structure keeps its size; nothing past the known
    layout is written; sizes above uint32_t are refused (src/api.cpp:66-80)."""
    lib = abi.bind(library_path())
    buf = (C.c_uint8 * 128)(*([0xAB] * 128))
    assert lib.xtbloom_compute_options_init(C.cast(buf, C.POINTER(abi.ComputeOptions)), 96) == abi.SUCCESS
    o = abi.ComputeOptions.from_buffer(buf)
    assert o.struct_size == 96 and o.api_version == 1
    assert bytes(buf[80:128]) == b"\xab" * 48
    big = C.c_size_t(1 << 32).value
    assert lib.xtbloom_compute_options_init(C.byref(abi.ComputeOptions()), big) == abi.INVALID_ARGUMENT
    assert b"uint32_t" in lib.xtbloom_get_last_error()


def test_status_strings_and_version():
    lib = abi.bind(library_path())
    assert lib.xtbloom_status_string(abi.SCC_NOT_CONVERGED) == b"SCC not converged"
    assert lib.xtbloom_version_string().startswith(b"0.1")


def test_cpu_backend_is_refused_without_fallback():
    """The CPU backend is unavailable by design: there is no CPU fallback."""
    lib = abi.bind(library_path())
    o = abi.ContextOptions()
    lib.xtbloom_context_options_init(C.byref(o), C.sizeof(o))
    o.backend = abi.BACKEND_CPU
    ctx = C.c_void_p()
    assert lib.xtbloom_context_create(C.byref(o), C.byref(ctx)) == abi.BACKEND_UNAVAILABLE
    assert not ctx.value


def test_compute_rejects_null_context():
    lib = abi.bind(library_path())
    b = abi.Batch()
    lib.xtbloom_batch_init(C.byref(b), C.sizeof(b))
    o = abi.ComputeOptions()
    lib.xtbloom_compute_options_init(C.byref(o), C.sizeof(o))
    r = abi.BatchResult()
    lib.xtbloom_batch_result_init(C.byref(r), C.sizeof(r))
    assert lib.xtbloom_compute(None, C.byref(b), C.byref(o), C.byref(r)) == abi.INVALID_ARGUMENT
    assert b"context" in lib.xtbloom_get_last_error()


def test_ragged_packing_is_exact():
    from xtbloom_b200 import workloads as W
    b = W.config0(4)
    assert b.atom_offsets.tolist() == [0, 32, 64, 96, 128]
    assert b.atomic_numbers.dtype == np.int32 and b.positions.dtype == np.float64
    b1 = W.config1(64)
    n_ao = [int(np.sum(np.where(W.molecule(b1, i)[0] == 1, 1, 4))) for i in range(64)]
    assert min(n_ao) >= 20 and max(n_ao) <= 242
