"""Python calculators over the CUDA library, mirroring the reference interface.

``Calculator(method, numbers, positions, charge, uhf, ...).singlepoint()`` and
``BatchCalculator`` follow the names, argument meanings and error behaviour of
the reference's ``xtbloom.interface`` (python/xtbloom/interface.py:1792-2100):
electronic temperature in kelvin, tolerances in atomic units, results through
``Result.get(name)``.  Failures surface as ``abi.XtbloomError`` carrying the
library status.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import abi

_METHODS = {"gfn2-xtb": abi.MODEL_GFN2, "gfn2": abi.MODEL_GFN2,
            "gfn1-xtb": abi.MODEL_GFN1, "gfn1": abi.MODEL_GFN1}

_SYMBOLS = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10,
            "Na": 11, "Mg": 12, "Al": 13, "Si": 14, "P": 15, "S": 16, "Cl": 17, "Ar": 18,
            "K": 19, "Ca": 20, "Br": 35, "I": 53}

_CONTEXTS: dict = {}


def _library(device_id: int | None) -> abi.Library:
    key = -1 if device_id is None else int(device_id)
    if key not in _CONTEXTS:
        from . import library_path
        _CONTEXTS[key] = abi.Library(library_path(), backend=abi.BACKEND_CUDA,
                                     device_id=key)
    return _CONTEXTS[key]


def _resolve_method(method: str) -> int:
    try:
        return _METHODS[method.lower()]
    except KeyError as exc:
        raise ValueError(f"unknown method {method!r}") from exc


def _numbers(numbers) -> np.ndarray:
    arr = list(numbers)
    if arr and isinstance(arr[0], str):
        arr = [_SYMBOLS[s] for s in arr]
    return np.asarray(arr, dtype=np.int32)


class Result:
    """Dictionary-like container of one calculation's outputs."""

    def __init__(self, values: dict):
        self._values = values

    def get(self, name: str):
        if name not in self._values:
            raise KeyError(f"result has no property {name!r}")
        return self._values[name]

    def __contains__(self, name: str) -> bool:
        return name in self._values

    def keys(self):
        return self._values.keys()


class _Settings:
    def __init__(self, model, max_scc_iterations, charge_tolerance, energy_tolerance,
                 electronic_temperature, scc_mixer_history, scc_mixer_damping):
        self.model = model
        self.max_scc_iterations = int(max_scc_iterations)
        self.charge_tolerance = float(charge_tolerance)
        self.energy_tolerance = float(energy_tolerance)
        self.electronic_temperature = float(electronic_temperature)
        self.scc_mixer_history = int(scc_mixer_history)
        self.scc_mixer_damping = float(scc_mixer_damping)

    def set(self, attribute: str, value) -> None:
        if not hasattr(self, attribute) or attribute == "model":
            raise ValueError(f"unknown setting {attribute!r}")
        setattr(self, attribute, type(getattr(self, attribute))(value))

    def options(self, lib: abi.Library, flags: int) -> abi.ComputeOptions:
        return lib.make_options(model=self.model, flags=flags, max_iter=self.max_scc_iterations,
                                ctol=self.charge_tolerance, etol=self.energy_tolerance,
                                kt=self.electronic_temperature * abi.KELVIN_TO_HARTREE,
                                history=self.scc_mixer_history, damping=self.scc_mixer_damping)


class BatchCalculator:
    """Ragged batch of molecules evaluated in one ``xtbloom_compute`` call.

    ``device_ids`` (an addition with no reference counterpart) spreads one
    batch over several GPUs of the node: the systems are partitioned by
    predicted cost (``sharding.plan_shards``), each GPU's context computes
    its shard concurrently, and the results come back in system order.  The
    iteration counts of each call weight the next call's partition."""

    def __init__(self, method: str, numbers: Sequence, positions: Sequence,
                 charges: Sequence[float] | None = None, uhf: Sequence[int] | None = None, *,
                 device_id: int | None = None, device_ids: Sequence[int] | None = None,
                 max_scc_iterations: int = 250,
                 charge_tolerance: float = 1.0e-6, energy_tolerance: float = 1.0e-8,
                 electronic_temperature: float = 300.0, scc_mixer_history: int = 8,
                 scc_mixer_damping: float = 0.4):
        self._model = _resolve_method(method)
        self._numbers = [_numbers(z) for z in numbers]
        self._positions = [np.asarray(p, dtype=float).reshape(-1, 3) for p in positions]
        if len(self._numbers) != len(self._positions):
            raise ValueError("numbers and positions describe different batch sizes")
        for z, p in zip(self._numbers, self._positions):
            if len(z) != len(p):
                raise ValueError("positions must have one row per atom")
        nb = len(self._numbers)
        self._charges = np.zeros(nb) if charges is None else np.asarray(charges, float)
        self._uhf = np.zeros(nb, np.int32) if uhf is None else np.asarray(uhf, np.int32)
        self._settings = _Settings(self._model, max_scc_iterations, charge_tolerance,
                                   energy_tolerance, electronic_temperature, scc_mixer_history,
                                   scc_mixer_damping)
        self._device_id = device_id
        if device_ids is not None:
            device_ids = [int(d) for d in device_ids]
            if not device_ids or len(set(device_ids)) != len(device_ids):
                raise ValueError("device_ids must name distinct devices")
            if device_id is not None:
                raise ValueError("give device_id or device_ids, not both")
        self._device_ids = device_ids
        self._last_iterations = None

    def set(self, attribute: str, value) -> None:
        self._settings.set(attribute, value)

    def update(self, positions: Sequence) -> None:
        new = [np.asarray(p, dtype=float).reshape(-1, 3) for p in positions]
        if [len(p) for p in new] != [len(p) for p in self._positions]:
            raise ValueError("update may change coordinates only")
        self._positions = new

    def _compute(self, batch: abi.RaggedBatch, flags: int) -> dict:
        if self._device_ids is None or len(self._device_ids) == 1:
            dev = self._device_id if self._device_ids is None else self._device_ids[0]
            lib = _library(dev)
            return lib.compute(batch, self._settings.options(lib, flags))
        from . import sharding
        libs = [_library(d) for d in self._device_ids]
        cost = sharding.predicted_cost(batch, self._model, self._last_iterations)
        fns = [lambda b, lib=lib: lib.compute(b, self._settings.options(lib, flags)) for lib in libs]
        return sharding.threaded_compute(batch, fns, cost)

    def singlepoint(self) -> Result:
        batch = abi.ragged_from_lists(self._numbers, self._positions, self._charges, self._uhf)
        flags = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES | abi.COMPUTE_CHARGES
        out = self._compute(batch, flags)
        self._last_iterations = np.asarray(out["scc_iterations"]).copy()
        forces = out["forces"].reshape(-1, 3)
        offs = batch.atom_offsets
        split = lambda a: [a[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
        return Result({
            "energies": out["energies"],
            "forces": split(forces),
            "gradients": [-f for f in split(forces)],
            "charges": split(out["atomic_charges"]),
            "scc_iterations": out["scc_iterations"],
            "scc_converged": out["scc_converged"].astype(bool),
            "status": out["per_system_status"],
        })


class Calculator(BatchCalculator):
    """Single-molecule calculator (tblite-like API)."""

    def __init__(self, method: str, numbers, positions, charge: float = 0.0,
                 uhf: int | None = None, **kwargs):
        super().__init__(method, [numbers], [positions], [charge], [uhf or 0], **kwargs)

    def update(self, positions=None) -> None:
        if positions is not None:
            super().update([positions])

    def singlepoint(self) -> Result:
        res = super().singlepoint()
        status = int(res.get("status")[0])
        if status != abi.SUCCESS:
            raise abi.XtbloomError(status, "the system did not converge")
        return Result({
            "energy": float(res.get("energies")[0]),
            "forces": res.get("forces")[0],
            "gradient": res.get("gradients")[0],
            "charges": res.get("charges")[0],
            "scc_iterations": int(res.get("scc_iterations")[0]),
        })
