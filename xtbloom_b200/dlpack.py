"""DLPack producer over library-owned result arenas.

A result arena (``xtbloom_result_owner_t``) is a reference-counted host or
CUDA allocation that a compute writes its result buffers into and that
outlives the context.  A compact row-major slice of it exports through
``xtbloom_result_owner_export_dltensor`` as a DLPack 1.0 managed tensor; this
module wraps that tensor in the ``dltensor`` / ``dltensor_versioned``
PyCapsule of the Python DLPack protocol, so ``torch.from_dlpack`` and
``numpy.from_dlpack`` import the finished result without a copy.

Follows the reference's producer (python/xtbloom/_dlpack.py:834-1230,
``_ResultArena`` and ``DLPackResultBuffer``): every ``__dlpack__`` call makes a
fresh single-use capsule that holds its own arena reference; an importer that
consumes the capsule renames it ``used_dltensor[_versioned]`` and calls the
native deleter itself, and an unconsumed capsule forwards to the same deleter
when it is collected, so nothing leaks and nothing is freed twice.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

DEVICE_CPU, DEVICE_CUDA = 1, 2
CAPSULE = b"dltensor"
CAPSULE_VERSIONED = b"dltensor_versioned"

# DLDataType code/bits of the dtypes the C ABI exports
_DTYPES = {np.dtype(np.int8): (0, 8), np.dtype(np.int16): (0, 16), np.dtype(np.int32): (0, 32),
           np.dtype(np.int64): (0, 64), np.dtype(np.uint8): (1, 8),
           np.dtype(np.float32): (2, 32), np.dtype(np.float64): (2, 64)}


class ResultOwnerOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                ("memory_space", C.c_int32), ("device_id", C.c_int32),
                ("size_bytes", C.c_uint64), ("reserved", C.c_uint32)]


class DLPackView(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                ("byte_offset", C.c_uint64), ("dtype_code", C.c_int32),
                ("dtype_bits", C.c_int32), ("dtype_lanes", C.c_int32), ("ndim", C.c_int32),
                ("reserved", C.c_uint32), ("shape", C.POINTER(C.c_int64))]


# DLPack 1.0 managed-tensor layout (public dlpack.h), for reading exports back
class DLDevice(C.Structure):
    _fields_ = [("device_type", C.c_int32), ("device_id", C.c_int32)]


class DLDataType(C.Structure):
    _fields_ = [("code", C.c_uint8), ("bits", C.c_uint8), ("lanes", C.c_uint16)]


class DLTensor(C.Structure):
    _fields_ = [("data", C.c_void_p), ("device", DLDevice), ("ndim", C.c_int32),
                ("dtype", DLDataType), ("shape", C.POINTER(C.c_int64)),
                ("strides", C.POINTER(C.c_int64)), ("byte_offset", C.c_uint64)]


DELETER = C.CFUNCTYPE(None, C.c_void_p)


class DLManagedTensor(C.Structure):
    _fields_ = [("dl_tensor", DLTensor), ("manager_ctx", C.c_void_p), ("deleter", DELETER)]


class DLManagedTensorVersioned(C.Structure):
    _fields_ = [("major", C.c_uint32), ("minor", C.c_uint32), ("manager_ctx", C.c_void_p),
                ("deleter", DELETER), ("flags", C.c_uint64), ("dl_tensor", DLTensor)]


def bind(lib: C.CDLL) -> C.CDLL:
    """Declare the result-owner prototypes on a loaded library."""
    P = C.POINTER
    lib.xtbloom_result_owner_options_init.restype = C.c_int32
    lib.xtbloom_result_owner_options_init.argtypes = [P(ResultOwnerOptions), C.c_size_t]
    lib.xtbloom_result_owner_create.restype = C.c_int32
    lib.xtbloom_result_owner_create.argtypes = [P(ResultOwnerOptions), P(C.c_void_p)]
    lib.xtbloom_result_owner_buffer.restype = C.c_int32
    lib.xtbloom_result_owner_buffer.argtypes = [C.c_void_p, P(abi.Buffer)]
    lib.xtbloom_result_owner_retain.restype = None
    lib.xtbloom_result_owner_retain.argtypes = [C.c_void_p]
    lib.xtbloom_result_owner_release.restype = None
    lib.xtbloom_result_owner_release.argtypes = [C.c_void_p]
    lib.xtbloom_result_owner_export_dltensor.restype = C.c_int32
    lib.xtbloom_result_owner_export_dltensor.argtypes = [C.c_void_p, P(DLPackView), C.c_int,
                                                         P(C.c_void_p)]
    return lib


# CPython capsule calls on raw addresses: the destructor runs while the capsule
# is being deallocated, when building a py_object for it would resurrect it.
_api = C.PyDLL(None)
_api.PyCapsule_New.restype = C.py_object
_api.PyCapsule_New.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
_api.PyCapsule_GetName.restype = C.c_char_p
_api.PyCapsule_GetName.argtypes = [C.c_void_p]
_api.PyCapsule_GetPointer.restype = C.c_void_p
_api.PyCapsule_GetPointer.argtypes = [C.c_void_p, C.c_char_p]


def _call_deleter(managed: int, versioned: bool) -> None:
    kind = DLManagedTensorVersioned if versioned else DLManagedTensor
    fn = C.cast(managed, C.POINTER(kind)).contents.deleter
    if fn:
        fn(managed)


def _make_destructor(versioned: bool):
    name = CAPSULE_VERSIONED if versioned else CAPSULE

    @C.CFUNCTYPE(None, C.c_void_p)
    def destructor(capsule: int) -> None:
        if _api.PyCapsule_GetName(capsule) != name:
            return          # consumed: the importer owns the managed tensor now
        managed = _api.PyCapsule_GetPointer(capsule, name)
        if managed:
            _call_deleter(managed, versioned)
    return destructor


# alive for the whole process: a capsule can outlive every Python object here
_DESTRUCTORS = {False: _make_destructor(False), True: _make_destructor(True)}


class ResultArena:
    """One reference to a native result arena (host or CUDA device memory)."""

    def __init__(self, lib: C.CDLL, size_bytes: int, memory_space: int = abi.MEMORY_HOST,
                 device_id: int = -1):
        self.lib = bind(lib)
        o = ResultOwnerOptions()
        self._check(lib.xtbloom_result_owner_options_init(C.byref(o), C.sizeof(o)))
        o.memory_space, o.device_id, o.size_bytes = memory_space, device_id, size_bytes
        h = C.c_void_p()
        self._check(lib.xtbloom_result_owner_create(C.byref(o), C.byref(h)))
        self.handle = h.value
        b = abi.Buffer()
        self._check(lib.xtbloom_result_owner_buffer(self.handle, C.byref(b)))
        self.data, self.size_bytes, self.memory_space = b.data, b.size_bytes, b.memory_space
        self.device_id = device_id if memory_space == abi.MEMORY_CUDA else 0

    def _check(self, status: int) -> None:
        if status != abi.SUCCESS:
            raise abi.XtbloomError(status, self.lib.xtbloom_get_last_error().decode())

    def buffer(self, byte_offset: int, size_bytes: int) -> abi.Buffer:
        """An output buffer over [byte_offset, byte_offset + size_bytes)."""
        if byte_offset < 0 or size_bytes < 0 or byte_offset + size_bytes > self.size_bytes:
            raise ValueError("buffer exceeds the arena")
        return abi.Buffer(self.data + byte_offset, size_bytes, self.memory_space, 0)

    def slice(self, byte_offset: int, shape, dtype) -> DLPackResultBuffer:
        return DLPackResultBuffer(self, byte_offset, tuple(int(s) for s in shape), np.dtype(dtype))

    def close(self) -> None:
        """Drop this reference; exported tensors keep the arena alive."""
        if self.handle:
            self.lib.xtbloom_result_owner_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DLPackResultBuffer:
    """A DLPack producer over one compact slice of a result arena.  It holds its
    own arena reference, so it stays exportable after the arena object closes."""

    def __init__(self, arena: ResultArena, byte_offset: int, shape: tuple, dtype: np.dtype):
        if dtype not in _DTYPES:
            raise TypeError(f"dtype {dtype} has no DLPack export")
        if not arena.handle:
            raise ValueError("result arena is closed")
        self.arena, self.byte_offset, self.shape, self.dtype = arena, byte_offset, shape, dtype
        arena.lib.xtbloom_result_owner_retain(arena.handle)
        self.handle = arena.handle

    def close(self) -> None:
        if self.handle:
            self.arena.lib.xtbloom_result_owner_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __dlpack_device__(self) -> tuple[int, int]:
        cuda = self.arena.memory_space == abi.MEMORY_CUDA
        return (DEVICE_CUDA if cuda else DEVICE_CPU, self.arena.device_id)

    def export(self, versioned: bool) -> int:
        """The raw managed-tensor pointer of one export (the caller owns it)."""
        if not self.handle:
            raise ValueError("result slice is closed")
        code, bits = _DTYPES[self.dtype]
        shape = (C.c_int64 * max(len(self.shape), 1))(*self.shape)
        v = DLPackView(C.sizeof(DLPackView), 1, self.byte_offset, code, bits, 1, len(self.shape), 0,
                       C.cast(shape, C.POINTER(C.c_int64)))
        out = C.c_void_p()
        self.arena._check(self.arena.lib.xtbloom_result_owner_export_dltensor(
            self.handle, C.byref(v), 1 if versioned else 0, C.byref(out)))
        return out.value

    def __dlpack__(self, stream=None, max_version=None, copy=None, dl_device=None):
        if copy is True:
            raise BufferError("copy=True is not supported by result arenas")
        if dl_device is not None and tuple(dl_device) != self.__dlpack_device__():
            raise BufferError(f"slice lives on {self.__dlpack_device__()}, not {dl_device}")
        # compute results are complete on the context stream when the call returns,
        # so no stream synchronisation is owed to the consumer
        versioned = max_version is not None and tuple(max_version) >= (1, 0)
        managed = self.export(versioned)
        name = CAPSULE_VERSIONED if versioned else CAPSULE
        try:
            return _api.PyCapsule_New(managed, name, C.cast(_DESTRUCTORS[versioned], C.c_void_p))
        except BaseException:
            _call_deleter(managed, versioned)
            raise
