"""ctypes mirror of the versioned caller-buffer C ABI (``include/xtbloom/xtbloom.h``).

The layouts follow the reference's public header byte for byte
(include/xtbloom/xtbloom.h:284-700 in the reference project) so that the
same descriptors drive either this package's CUDA library or any other
library exporting the ``xtbloom_*`` symbols.  All structures start with
``struct_size`` / ``api_version`` and are initialised through the library's
own ``*_init`` functions, exactly as the reference bindings do
(python/xtbloom/library.py:164-250).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

API_VERSION = 1
KELVIN_TO_HARTREE = 3.166808578545117e-6

# status codes (xtbloom.h:65-78)
SUCCESS, INVALID_ARGUMENT, BACKEND_UNAVAILABLE, NOT_SUPPORTED = 0, 1, 2, 3
ALLOCATION_FAILED, NOT_IMPLEMENTED, INTERNAL_ERROR = 4, 5, 6
SCC_NOT_CONVERGED, EIGENSOLVER_FAILED = 7, 8
# request states (xtbloom.h:80-90)
REQUEST_IDLE, REQUEST_PENDING, REQUEST_COMPLETE = 0, 1, 2
# determinism policies (xtbloom.h:127-134)
DETERMINISM_DEFAULT, DETERMINISM_REPRODUCIBLE = 0, 1
STATUS_NAMES = {0: "SUCCESS", 1: "INVALID_ARGUMENT", 2: "BACKEND_UNAVAILABLE",
                3: "NOT_SUPPORTED", 4: "ALLOCATION_FAILED", 5: "NOT_IMPLEMENTED",
                6: "INTERNAL_ERROR", 7: "SCC_NOT_CONVERGED", 8: "EIGENSOLVER_FAILED"}

BACKEND_AUTO, BACKEND_CPU, BACKEND_CUDA = 0, 1, 2
MEMORY_HOST, MEMORY_CUDA = 0, 1
MODEL_GFN1, MODEL_GFN2 = 1, 2
START_FRESH, START_WARM = 1, 2
MIXER_BROYDEN = 1
COMPUTE_ENERGY, COMPUTE_FORCES, COMPUTE_CHARGES = 1, 2, 4
COMPUTE_POINT_CHARGE_FORCES, COMPUTE_DIPOLES = 8, 16


class ContextOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                ("backend", C.c_int32), ("device_id", C.c_int32),
                ("cpu_threads", C.c_int32), ("reserved", C.c_uint32),
                ("stream", C.c_void_p)]


class ConstBuffer(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size_bytes", C.c_size_t),
                ("memory_space", C.c_int32), ("reserved", C.c_uint32)]


class Buffer(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size_bytes", C.c_size_t),
                ("memory_space", C.c_int32), ("reserved", C.c_uint32)]


BATCH_BUFFERS = ["atom_offsets", "atomic_numbers", "positions", "molecular_charges",
                 "unpaired_electrons", "point_charge_offsets", "point_charge_positions",
                 "point_charge_values", "point_charge_gammas", "atomic_potential_shifts",
                 "charge_response_offsets", "charge_response_matrix", "spin_channels"]


class Batch(C.Structure):
    _fields_ = ([("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                 ("batch_size", C.c_int64), ("total_atoms", C.c_int64),
                 ("total_point_charges", C.c_int64),
                 ("total_charge_response_elements", C.c_int64)]
                + [(n, ConstBuffer) for n in BATCH_BUFFERS]
                + [("total_interactions", C.c_int64),
                   ("interaction_descriptors", ConstBuffer),
                   ("interaction_payload", ConstBuffer),
                   ("cell_matrices", ConstBuffer), ("periodic_axes", ConstBuffer)])


class ComputeOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                ("model", C.c_int32), ("flags", C.c_uint32),
                ("max_scc_iterations", C.c_int32), ("reserved", C.c_uint32),
                ("charge_tolerance", C.c_double), ("energy_tolerance", C.c_double),
                ("electronic_temperature", C.c_double),
                ("scc_start_mode", C.c_int32), ("reserved_v2", C.c_uint32),
                ("scc_mixer", C.c_int32), ("scc_mixer_history", C.c_int32),
                ("scc_mixer_damping", C.c_double), ("determinism", C.c_int32),
                ("reserved_v3", C.c_uint32)]


RESULT_BUFFERS = ["energies", "forces", "atomic_charges", "point_charge_forces",
                  "scc_iterations", "scc_converged", "per_system_status",
                  "dipole_moments", "quadrupole_moments", "wiberg_orders", "spin_populations"]


class BatchResult(C.Structure):
    _fields_ = ([("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                 ("flags", C.c_uint32), ("reserved", C.c_uint32)]
                + [(n, Buffer) for n in RESULT_BUFFERS])


class RequestInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                ("state", C.c_int32), ("completion_status", C.c_int32),
                ("result_flags", C.c_uint32), ("reserved", C.c_uint32)]


class WorkspaceQuery(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("api_version", C.c_uint32),
                ("compute_flags", C.c_uint32), ("reserved", C.c_uint32),
                ("host_required_bytes", C.c_uint64), ("host_required_alignment", C.c_uint32),
                ("device_required_bytes", C.c_uint64), ("device_required_alignment", C.c_uint32),
                ("reserved_v2", C.c_uint32)]


# Sizes asserted by the reference header on LP64 (xtbloom.h:322-400).
assert C.sizeof(ContextOptions) == 32
assert C.sizeof(ConstBuffer) == 24
assert Batch.total_interactions.offset == 352
assert C.sizeof(Batch) == 456
assert C.sizeof(ComputeOptions) == 80
assert C.sizeof(BatchResult) == 280

ABI_SYMBOLS = [
    "xtbloom_version_string", "xtbloom_status_string", "xtbloom_get_last_error",
    "xtbloom_context_options_init", "xtbloom_batch_init", "xtbloom_compute_options_init",
    "xtbloom_batch_result_init", "xtbloom_workspace_query_init", "xtbloom_request_info_init",
    "xtbloom_context_create", "xtbloom_context_destroy", "xtbloom_context_get_backend",
    "xtbloom_context_get_device_id", "xtbloom_request_create", "xtbloom_request_query",
    "xtbloom_request_wait", "xtbloom_request_get_error", "xtbloom_request_destroy",
    "xtbloom_compute", "xtbloom_compute_enqueue", "xtbloom_plan_create", "xtbloom_plan_destroy",
    "xtbloom_plan_query_workspace", "xtbloom_plan_compute", "xtbloom_plan_compute_enqueue",
]


PRECISION_FP64 = 0
PRECISION_MIXED = 1


def bind(path: str) -> C.CDLL:
    """Load a library exporting the xtbloom ABI and declare its prototypes."""
    lib = C.CDLL(path)
    P = C.POINTER
    st = C.c_int32
    lib.xtbloom_version_string.restype = C.c_char_p
    lib.xtbloom_status_string.restype = C.c_char_p
    lib.xtbloom_status_string.argtypes = [st]
    lib.xtbloom_get_last_error.restype = C.c_char_p
    for name, typ in [("xtbloom_context_options_init", ContextOptions),
                      ("xtbloom_batch_init", Batch),
                      ("xtbloom_compute_options_init", ComputeOptions),
                      ("xtbloom_batch_result_init", BatchResult),
                      ("xtbloom_request_info_init", RequestInfo),
                      ("xtbloom_workspace_query_init", WorkspaceQuery)]:
        fn = getattr(lib, name)
        fn.restype = st
        fn.argtypes = [P(typ), C.c_size_t]
    lib.xtbloom_context_create.restype = st
    lib.xtbloom_context_create.argtypes = [P(ContextOptions), P(C.c_void_p)]
    lib.xtbloom_context_destroy.restype = None
    lib.xtbloom_context_destroy.argtypes = [C.c_void_p]
    lib.xtbloom_context_get_backend.restype = st
    lib.xtbloom_context_get_backend.argtypes = [C.c_void_p]
    lib.xtbloom_context_get_device_id.restype = C.c_int32
    lib.xtbloom_context_get_device_id.argtypes = [C.c_void_p]
    lib.xtbloom_compute.restype = st
    lib.xtbloom_compute.argtypes = [C.c_void_p, P(Batch), P(ComputeOptions), P(BatchResult)]
    lib.xtbloom_compute_enqueue.restype = st
    lib.xtbloom_compute_enqueue.argtypes = [C.c_void_p, P(Batch), P(ComputeOptions),
                                            P(BatchResult), C.c_void_p]
    lib.xtbloom_request_create.restype = st
    lib.xtbloom_request_create.argtypes = [C.c_void_p, P(C.c_void_p)]
    lib.xtbloom_request_wait.restype = st
    lib.xtbloom_request_wait.argtypes = [C.c_void_p, P(RequestInfo)]
    lib.xtbloom_request_query.restype = st
    lib.xtbloom_request_query.argtypes = [C.c_void_p, P(RequestInfo)]
    lib.xtbloom_request_get_error.restype = C.c_char_p
    lib.xtbloom_request_get_error.argtypes = [C.c_void_p]
    lib.xtbloom_request_destroy.restype = None
    lib.xtbloom_request_destroy.argtypes = [C.c_void_p]
    lib.xtbloom_plan_create.restype = st
    lib.xtbloom_plan_create.argtypes = [C.c_void_p, P(Batch), P(ComputeOptions), P(C.c_void_p)]
    lib.xtbloom_plan_destroy.restype = None
    lib.xtbloom_plan_destroy.argtypes = [C.c_void_p]
    lib.xtbloom_plan_query_workspace.restype = st
    lib.xtbloom_plan_query_workspace.argtypes = [C.c_void_p, P(WorkspaceQuery)]
    lib.xtbloom_plan_compute.restype = st
    lib.xtbloom_plan_compute.argtypes = [C.c_void_p, P(Batch), P(ComputeOptions), P(BatchResult)]
    lib.xtbloom_plan_compute_enqueue.restype = st
    lib.xtbloom_plan_compute_enqueue.argtypes = [C.c_void_p, P(Batch), P(ComputeOptions),
                                                 P(BatchResult), C.c_void_p]
    return lib


class XtbloomError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


INTERACTION_ELECTRIC_FIELD = 0x0101


class Interaction(C.Structure):
    _fields_ = [("type", C.c_int32), ("flags", C.c_uint32), ("system_index", C.c_int64),
                ("payload_offset", C.c_uint64), ("payload_size", C.c_uint64)]


def pack_efields(efields):
    """Descriptors and payload of electric-field attachments (block_version 1:
    int32 version, int32 reserved, three doubles) for every row without NaN."""
    rows = [i for i, e in enumerate(np.asarray(efields, float)) if np.all(np.isfinite(e))]
    desc = (Interaction * max(len(rows), 1))()
    payload = np.zeros(32 * max(len(rows), 1), np.uint8)
    for k, i in enumerate(rows):
        desc[k] = Interaction(INTERACTION_ELECTRIC_FIELD, 0, i, 32 * k, 32)
        block = np.zeros(4, np.float64)
        block[1:] = np.asarray(efields, float)[i]
        raw = block.view(np.uint8).copy()
        raw[0:4] = np.frombuffer(np.int32(1).tobytes(), np.uint8)
        raw[4:8] = 0
        payload[32 * k:32 * k + 32] = raw
    return desc, payload, len(rows)


def _cbuf(arr) -> ConstBuffer:
    if arr is None:
        return ConstBuffer(None, 0, MEMORY_HOST, 0)
    if hasattr(arr, "data_ptr"):          # torch tensor
        space = MEMORY_CUDA if arr.is_cuda else MEMORY_HOST
        return ConstBuffer(arr.data_ptr(), arr.numel() * arr.element_size(), space, 0)
    return ConstBuffer(arr.ctypes.data, arr.nbytes, MEMORY_HOST, 0)


def _obuf(arr) -> Buffer:
    if arr is None:
        return Buffer(None, 0, MEMORY_HOST, 0)
    if isinstance(arr, Buffer):           # e.g. a slice of a result arena
        return arr
    if hasattr(arr, "data_ptr"):
        space = MEMORY_CUDA if arr.is_cuda else MEMORY_HOST
        return Buffer(arr.data_ptr(), arr.numel() * arr.element_size(), space, 0)
    return Buffer(arr.ctypes.data, arr.nbytes, MEMORY_HOST, 0)


@dataclass
class RaggedBatch:
    """Host (numpy) or device (torch) arrays of one ragged batch."""
    atom_offsets: object
    atomic_numbers: object
    positions: object
    molecular_charges: object
    unpaired_electrons: object
    spin_channels: object = None
    point_charge_offsets: object = None
    point_charge_positions: object = None
    point_charge_values: object = None
    point_charge_gammas: object = None
    # per system uniform electric field (Hartree / (e bohr)), shape (B, 3); a row
    # of NaN (or None for the whole batch) means no attachment
    efields: object = None
    # charge response b + A q: per-atom shifts b, per-system symmetric
    # atoms x atoms blocks A (row-major, packed) at charge_response_offsets
    atomic_potential_shifts: object = None
    charge_response_offsets: object = None
    charge_response_matrix: object = None

    @property
    def batch_size(self) -> int:
        return int(len(self.atom_offsets) - 1)

    @property
    def total_atoms(self) -> int:
        return int(len(self.atomic_numbers))


class Library:
    """Thin owner of one loaded ABI library and one context."""

    def __init__(self, path: str, backend: int = BACKEND_AUTO, device_id: int = 0,
                 cpu_threads: int = 0, stream: int | None = None):
        self.lib = bind(path)
        self.path = path
        opts = ContextOptions()
        self._check(self.lib.xtbloom_context_options_init(C.byref(opts), C.sizeof(opts)))
        opts.backend = backend
        opts.device_id = device_id
        opts.cpu_threads = cpu_threads
        opts.stream = stream
        ctx = C.c_void_p()
        self._check(self.lib.xtbloom_context_create(C.byref(opts), C.byref(ctx)))
        self.ctx = ctx

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.xtbloom_context_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int):
        if status != SUCCESS:
            msg = self.lib.xtbloom_get_last_error()
            raise XtbloomError(status, msg.decode() if msg else "")

    def set_execution(self, precision: int = PRECISION_FP64, switch_residual: float = 0.0,
                      capture_graphs: bool = False):
        """Select the execution form of later computes (CUDA contexts only):
        FP64 throughout, or split-precision GEMMs until the precision switch."""
        f = self.lib.xtbloom_b200_context_set_execution
        f.restype = C.c_int32
        f.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_int32]
        self._check(f(self.ctx, int(precision), float(switch_residual), 1 if capture_graphs else 0))

    def fetch(self, name: str, system: int = -1, capacity: int = 1 << 16) -> np.ndarray:
        """Diagnostics export of the most recent compute (xtbloom_b200_debug_fetch)."""
        f = self.lib.xtbloom_b200_debug_fetch
        f.restype = C.c_int32
        f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_double), C.c_size_t,
                      C.POINTER(C.c_size_t)]
        out = np.zeros(capacity)
        cnt = C.c_size_t()
        self._check(f(self.ctx, name.encode(), system, out.ctypes.data_as(C.POINTER(C.c_double)),
                      capacity, C.byref(cnt)))
        return out[:cnt.value].copy()

    def make_batch(self, b: RaggedBatch) -> Batch:
        batch = Batch()
        self._check(self.lib.xtbloom_batch_init(C.byref(batch), C.sizeof(batch)))
        batch.batch_size = b.batch_size
        batch.total_atoms = b.total_atoms
        for name in ("atom_offsets", "atomic_numbers", "positions", "molecular_charges",
                     "unpaired_electrons", "spin_channels"):
            setattr(batch, name, _cbuf(getattr(b, name)))
        if b.point_charge_offsets is not None:
            batch.total_point_charges = int(len(b.point_charge_values))
            for name in ("point_charge_offsets", "point_charge_positions",
                         "point_charge_values", "point_charge_gammas"):
                setattr(batch, name, _cbuf(getattr(b, name)))
        if b.charge_response_matrix is not None:
            batch.total_charge_response_elements = int(len(b.charge_response_matrix))
            for name in ("atomic_potential_shifts", "charge_response_offsets", "charge_response_matrix"):
                setattr(batch, name, _cbuf(getattr(b, name)))
        if b.efields is not None:
            desc, payload, k = pack_efields(b.efields)
            if k:
                batch.total_interactions = k
                batch.interaction_descriptors = ConstBuffer(C.addressof(desc), C.sizeof(Interaction) * k,
                                                            MEMORY_HOST, 0)
                batch.interaction_payload = ConstBuffer(payload.ctypes.data, payload.nbytes, MEMORY_HOST, 0)
                batch._keep = (desc, payload)   # the buffers must outlive the call
        return batch

    def make_options(self, model=MODEL_GFN2, flags=COMPUTE_ENERGY | COMPUTE_FORCES | COMPUTE_CHARGES,
                     max_iter=250, ctol=1e-6, etol=1e-8, kt=300.0 * KELVIN_TO_HARTREE,
                     start=START_FRESH, history=8, damping=0.4) -> ComputeOptions:
        opts = ComputeOptions()
        self._check(self.lib.xtbloom_compute_options_init(C.byref(opts), C.sizeof(opts)))
        opts.model = model
        opts.flags = flags
        opts.max_scc_iterations = max_iter
        opts.charge_tolerance = ctol
        opts.energy_tolerance = etol
        opts.electronic_temperature = kt
        opts.scc_start_mode = start
        opts.scc_mixer = MIXER_BROYDEN
        opts.scc_mixer_history = history
        opts.scc_mixer_damping = damping
        return opts

    def make_result(self, outs: dict) -> BatchResult:
        res = BatchResult()
        self._check(self.lib.xtbloom_batch_result_init(C.byref(res), C.sizeof(res)))
        for name, arr in outs.items():
            setattr(res, name, _obuf(arr))
        return res

    def compute(self, b: RaggedBatch, options: ComputeOptions | None = None,
                outputs: dict | None = None) -> dict:
        """One blocking ``xtbloom_compute`` with host output buffers."""
        options = options or self.make_options()
        nb, na = b.batch_size, b.total_atoms
        if outputs is None:
            outputs = {"energies": np.empty(nb), "forces": np.empty(3 * na),
                       "atomic_charges": np.empty(na),
                       "scc_iterations": np.empty(nb, np.int32),
                       "scc_converged": np.empty(nb, np.uint8),
                       "per_system_status": np.empty(nb, np.int32)}
            if b.point_charge_offsets is not None and options.flags & COMPUTE_POINT_CHARGE_FORCES:
                outputs["point_charge_forces"] = np.empty(3 * len(b.point_charge_values))
        batch = self.make_batch(b)
        res = self.make_result({k: v for k, v in outputs.items() if k in RESULT_BUFFERS})
        self._check(self.lib.xtbloom_compute(self.ctx, C.byref(batch), C.byref(options), C.byref(res)))
        self.last_result_flags = res.flags
        return outputs


def host_outputs(b: RaggedBatch, fill: float = np.nan) -> dict:
    """Host output buffers of one batch (energies, forces, charges, diagnostics)."""
    nb, na = b.batch_size, b.total_atoms
    return {"energies": np.full(nb, fill), "forces": np.full(3 * na, fill),
            "atomic_charges": np.full(na, fill),
            "scc_iterations": np.full(nb, -7, np.int32), "scc_converged": np.full(nb, 7, np.uint8),
            "per_system_status": np.full(nb, -7, np.int32)}


class Plan:
    """A fixed-topology plan (xtbloom_plan_*) of a Library's context."""

    def __init__(self, lib: Library, b: RaggedBatch, options: ComputeOptions | None = None):
        self.lib = lib
        self.options = options or lib.make_options()
        self._batch = lib.make_batch(b)
        h = C.c_void_p()
        lib._check(lib.lib.xtbloom_plan_create(lib.ctx, C.byref(self._batch), C.byref(self.options),
                                               C.byref(h)))
        self.handle = h

    def workspace(self) -> WorkspaceQuery:
        q = WorkspaceQuery()
        self.lib._check(self.lib.lib.xtbloom_workspace_query_init(C.byref(q), C.sizeof(q)))
        q.compute_flags = self.options.flags
        self.lib._check(self.lib.lib.xtbloom_plan_query_workspace(self.handle, C.byref(q)))
        return q

    def compute(self, b: RaggedBatch, outputs: dict | None = None,
                options: ComputeOptions | None = None) -> dict:
        outputs = outputs if outputs is not None else host_outputs(b)
        batch = self.lib.make_batch(b)
        res = self.lib.make_result({k: v for k, v in outputs.items() if k in RESULT_BUFFERS})
        self.lib._check(self.lib.lib.xtbloom_plan_compute(self.handle, C.byref(batch),
                                                          C.byref(options or self.options),
                                                          C.byref(res)))
        return outputs

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lib.xtbloom_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ragged_from_lists(numbers_list, positions_list, charges=None, uhf=None,
                      spin_channels=None) -> RaggedBatch:
    """Pack per-molecule arrays into the ABI's ragged host layout.  spin_channels
    (1 restricted, 2 unrestricted per molecule) is omitted when None."""
    counts = [len(z) for z in numbers_list]
    offs = np.zeros(len(counts) + 1, np.int64)
    offs[1:] = np.cumsum(counts)
    nb = len(counts)
    return RaggedBatch(
        atom_offsets=offs,
        atomic_numbers=np.ascontiguousarray(np.concatenate(numbers_list).astype(np.int32)),
        positions=np.ascontiguousarray(np.concatenate([np.asarray(p, float).reshape(-1) for p in positions_list])),
        molecular_charges=np.asarray(charges if charges is not None else np.zeros(nb), float),
        unpaired_electrons=np.asarray(uhf if uhf is not None else np.zeros(nb), np.int32),
        spin_channels=None if spin_channels is None else np.ascontiguousarray(np.asarray(spin_channels, np.int32)),
    )
