"""Result arenas and their DLPack export, on host arenas (no GPU needed).

Mirrors the reference's tests/result_owner_test.cpp: managed-tensor fields
read back byte by byte, independent repeated exports, exports that outlive the
producer's reference, and every failure path leaving the output NULL.  Import
through torch.from_dlpack and numpy.from_dlpack checks the capsule protocol.
"""
from __future__ import annotations

import ctypes as C
import gc

import numpy as np
import pytest
import torch

from xtbloom_b200 import abi, dlpack, library_path


@pytest.fixture(scope="module")
def lib():
    return dlpack.bind(abi.bind(library_path()))


def view(shape, offset=0, code=2, bits=64, lanes=1, **kw):
    arr = (C.c_int64 * max(len(shape), 1))(*shape)
    v = dlpack.DLPackView(C.sizeof(dlpack.DLPackView), 1, offset, code, bits, lanes, len(shape), 0,
                          C.cast(arr, C.POINTER(C.c_int64)))
    for k, val in kw.items():
        setattr(v, k, val)
    v._keep = arr
    return v


def export(lib, arena, v, version=1):
    out = C.c_void_p(0x1234)
    st = lib.xtbloom_result_owner_export_dltensor(arena.handle, C.byref(v), version, C.byref(out))
    return st, out.value


def delete(ptr, versioned):
    dlpack._call_deleter(ptr, versioned)


def test_view_layout_matches_the_reference_abi():
    assert C.sizeof(dlpack.DLPackView) == 48
    assert dlpack.DLPackView.shape.offset == 40
    assert C.sizeof(dlpack.ResultOwnerOptions) == 32
    assert C.sizeof(dlpack.DLTensor) == 48
    assert C.sizeof(dlpack.DLManagedTensor) == 64
    assert C.sizeof(dlpack.DLManagedTensorVersioned) == 80


def test_host_arena_versioned_and_legacy_export(lib):
    arena = dlpack.ResultArena(lib, 4096)
    assert arena.size_bytes == 4096 and arena.memory_space == abi.MEMORY_HOST and arena.data
    st, p = export(lib, arena, view((8, 8), offset=64))
    assert st == abi.SUCCESS and p
    m = C.cast(p, C.POINTER(dlpack.DLManagedTensorVersioned)).contents
    assert (m.major, m.minor, m.flags) == (1, 0, 0)
    t = m.dl_tensor
    assert t.ndim == 2 and (t.device.device_type, t.device.device_id) == (1, 0)
    assert (t.dtype.code, t.dtype.bits, t.dtype.lanes) == (2, 64, 1)
    assert t.byte_offset == 0 and t.data == arena.data + 64      # offset folded into data
    assert (t.shape[0], t.shape[1]) == (8, 8) and not t.strides
    st, p2 = export(lib, arena, view((8, 8), offset=64))
    assert st == abi.SUCCESS and p2 and p2 != p                    # fresh single-use tensor
    st, legacy = export(lib, arena, view((8, 8), offset=64), version=0)
    assert st == abi.SUCCESS and legacy
    lt = C.cast(legacy, C.POINTER(dlpack.DLManagedTensor)).contents
    assert lt.dl_tensor.ndim == 2 and lt.dl_tensor.device.device_type == 1 and lt.manager_ctx
    # the exports hold their own arena references past the producer's release
    np.frombuffer((C.c_double * 8).from_address(arena.data + 64), np.float64)[:] = 7.5
    arena.close()
    assert C.cast(t.data, C.POINTER(C.c_double))[3] == 7.5
    delete(p, True)
    delete(p2, True)
    delete(legacy, False)


def test_export_failures_leave_output_null(lib):
    arena = dlpack.ResultArena(lib, 512)
    bad = [view((8, 64)),                                 # 4096 bytes > 512 arena
           view((16,), code=3),                           # unknown dtype code
           view((16,), code=1, bits=16), view((16,), code=1, bits=32), view((16,), code=1, bits=64),
           view((16,), code=4, bits=16), view((16,), code=6, bits=8),
           view((16,), lanes=2),
           view((16,), offset=4),                         # breaks float64 alignment
           view((-1,)),
           view((16,), offset=512 + 8),
           view((16,), reserved=1),
           view((16,), struct_size=16),
           view((16,), api_version=2),
           view((1,) * 9)]
    for v in bad:
        st, p = export(lib, arena, v)
        assert st == abi.INVALID_ARGUMENT and p is None
    st, p = export(lib, arena, view((8, 8)), version=7)
    assert st == abi.INVALID_ARGUMENT and p is None
    # an empty view is valid and publishes NULL data with the copied extents
    st, p = export(lib, arena, view((0, 3)))
    assert st == abi.SUCCESS and p
    t = C.cast(p, C.POINTER(dlpack.DLManagedTensorVersioned)).contents.dl_tensor
    assert not t.data and (t.shape[0], t.shape[1]) == (0, 3)
    delete(p, True)
    # a zero-dimensional view exports one element
    st, p = export(lib, arena, view((), offset=8))
    assert st == abi.SUCCESS and p
    delete(p, True)
    arena.close()


def test_owner_creation_failures(lib):
    o = dlpack.ResultOwnerOptions()
    assert lib.xtbloom_result_owner_options_init(C.byref(o), 27) == abi.INVALID_ARGUMENT
    assert lib.xtbloom_result_owner_options_init(C.byref(o), C.sizeof(o)) == abi.SUCCESS
    assert o.memory_space == abi.MEMORY_HOST and o.device_id == -1
    for field, value in [("size_bytes", 0), ("reserved", 1), ("device_id", 0), ("memory_space", 9)]:
        x = dlpack.ResultOwnerOptions.from_buffer_copy(o)
        x.size_bytes = 64
        setattr(x, field, value)
        h = C.c_void_p(0x99)
        assert lib.xtbloom_result_owner_create(C.byref(x), C.byref(h)) == abi.INVALID_ARGUMENT
        assert not h.value
    # retain/release accounting; a NULL release is a no-op
    a = dlpack.ResultArena(lib, 64)
    lib.xtbloom_result_owner_retain(a.handle)
    lib.xtbloom_result_owner_release(a.handle)
    lib.xtbloom_result_owner_release(None)
    a.close()
    a.close()


def test_torch_and_numpy_import_through_the_capsule(lib):
    arena = dlpack.ResultArena(lib, 1024)
    host = np.frombuffer((C.c_char * 1024).from_address(arena.data), np.uint8)
    host[:] = 0
    np.frombuffer(host.data, np.float64)[4:16] = np.arange(12.0)
    sl = arena.slice(32, (3, 4), np.float64)
    assert sl.__dlpack_device__() == (1, 0)
    t = torch.from_dlpack(sl)
    a = np.from_dlpack(sl)
    assert t.shape == (3, 4) and t.dtype == torch.float64
    assert np.array_equal(t.numpy(), np.arange(12.0).reshape(3, 4)) and np.array_equal(a, t.numpy())
    ints = torch.from_dlpack(arena.slice(0, (32,), np.int32))
    assert ints.dtype == torch.int32 and int(ints[0]) == 0
    arena.close()                       # the imported tensors keep the arena alive
    t[0, 0] = 42.0                      # zero-copy: both imports see the write
    assert a[0, 0] == 42.0
    # legacy capsule, and an unconsumed capsule freed by its destructor
    cap = sl.__dlpack__()
    del cap
    legacy = torch.utils.dlpack.from_dlpack(sl.__dlpack__())
    assert legacy[2, 3] == 11.0
    del t, a, ints, legacy
    gc.collect()
    sl.close()
    with pytest.raises(ValueError):
        sl.export(True)
