"""GFN2 energies as a differentiable torch function over the CUDA library.

``gfn2_energy(numbers, atom_offsets, positions, pc_offsets, pc_positions,
pc_charges, pc_gammas)`` returns one energy per system (Hartree) and is
differentiable with respect to the QM positions, the point-charge positions
and the point-charge values.  The forward pass is one ``xtbloom_compute``
call with the tensors passed as device buffers; the backward pass uses the
analytic adjoints the library returns with it: dE/dR = -forces,
dE/dR_pc = -point_charge_forces and dE/dQ_pc = sum_s q_s K_sp (the
point-charge potential derivative, read through ``xtbloom_b200_debug_fetch``).
Systems that fail (status != 0) have NaN energies and NaN gradients.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi

_LIB: abi.Library | None = None


def _library() -> abi.Library:
    global _LIB
    if _LIB is None:
        from . import library_path
        _LIB = abi.Library(library_path(), backend=abi.BACKEND_CUDA,
                           device_id=torch.cuda.current_device())
    return _LIB


def _charge_derivatives(lib: abi.Library, npc: int) -> np.ndarray:
    f = lib.lib.xtbloom_b200_debug_fetch
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_double), C.c_size_t,
                  C.POINTER(C.c_size_t)]
    out = np.zeros(max(npc, 1))
    cnt = C.c_size_t()
    st = f(lib.ctx, b"point_charge_dq", -1, out.ctypes.data_as(C.POINTER(C.c_double)), out.size,
           C.byref(cnt))
    if st != 0:
        raise abi.XtbloomError(st, lib.lib.xtbloom_get_last_error().decode())
    return out[:cnt.value]


class _GFN2Energy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, pc_positions, pc_charges, static):
        numbers, atom_offsets, charges, uhf, pc_offsets, pc_gammas, options = static
        lib = _library()
        dev = positions.device
        B = atom_offsets.numel() - 1
        N = positions.shape[0]
        have_pc = pc_charges is not None and pc_charges.numel() > 0
        batch = abi.RaggedBatch(atom_offsets, numbers, positions.detach().contiguous().reshape(-1),
                                charges, uhf)
        flags = abi.COMPUTE_ENERGY | abi.COMPUTE_FORCES
        if have_pc:
            batch.point_charge_offsets = pc_offsets
            batch.point_charge_positions = pc_positions.detach().contiguous().reshape(-1)
            batch.point_charge_values = pc_charges.detach().contiguous()
            batch.point_charge_gammas = pc_gammas
            flags |= abi.COMPUTE_POINT_CHARGE_FORCES
        f64 = dict(dtype=torch.float64, device=dev)
        outs = {"energies": torch.empty(B, **f64), "forces": torch.empty(3 * N, **f64),
                "scc_iterations": torch.empty(B, dtype=torch.int32, device=dev),
                "scc_converged": torch.empty(B, dtype=torch.uint8, device=dev),
                "per_system_status": torch.empty(B, dtype=torch.int32, device=dev)}
        P = pc_charges.numel() if have_pc else 0
        if have_pc:
            outs["point_charge_forces"] = torch.empty(3 * P, **f64)
        lib.compute(batch, lib.make_options(flags=flags, **options), outs)
        torch.cuda.current_stream(dev).synchronize()
        dEdR = -outs["forces"].reshape(N, 3)
        if have_pc:
            dEdRp = -outs["point_charge_forces"].reshape(P, 3)
            dEdQ = torch.as_tensor(_charge_derivatives(lib, P), **f64)
            # charges of failed systems carry NaN derivatives like their forces
            dEdQ = torch.where(torch.isnan(dEdRp[:, 0]), torch.full_like(dEdQ, float("nan")), dEdQ)
            pc_sys = torch.repeat_interleave(torch.arange(B, device=dev),
                                             (pc_offsets[1:] - pc_offsets[:-1]).to(dev))
        else:
            dEdRp = dEdQ = pc_sys = None
        at_sys = torch.repeat_interleave(torch.arange(B, device=dev), (atom_offsets[1:] - atom_offsets[:-1]).to(dev))
        ctx.save_for_backward(dEdR, at_sys, *( [dEdRp, dEdQ, pc_sys] if have_pc else []))
        ctx.have_pc = have_pc
        return outs["energies"]

    @staticmethod
    def backward(ctx, g):
        saved = ctx.saved_tensors
        dEdR, at_sys = saved[0], saved[1]
        g_pos = g[at_sys][:, None] * dEdR
        g_pcpos = g_pcq = None
        if ctx.have_pc:
            dEdRp, dEdQ, pc_sys = saved[2], saved[3], saved[4]
            g_pcpos = g[pc_sys][:, None] * dEdRp
            g_pcq = g[pc_sys] * dEdQ
        return g_pos, g_pcpos, g_pcq, None


def gfn2_energy(numbers: torch.Tensor, atom_offsets: torch.Tensor, positions: torch.Tensor,
                pc_offsets: torch.Tensor | None = None, pc_positions: torch.Tensor | None = None,
                pc_charges: torch.Tensor | None = None, pc_gammas: torch.Tensor | None = None,
                molecular_charges: torch.Tensor | None = None,
                unpaired_electrons: torch.Tensor | None = None, **options) -> torch.Tensor:
    """Energies [B] of a ragged batch; positions [N, 3] (bohr, float64, CUDA).

    numbers int32 [N], atom_offsets int64 [B+1]; point charges optional:
    pc_offsets int64 [B+1], pc_positions [P, 3], pc_charges [P], pc_gammas [P].
    ``options`` are forwarded to ``abi.Library.make_options`` (max_iter, ctol,
    etol, kt, history, damping)."""
    if not positions.is_cuda:
        raise ValueError("positions must be a CUDA tensor (there is no CPU path)")
    dev = positions.device
    B = atom_offsets.numel() - 1
    numbers = numbers.to(dev, torch.int32).contiguous()
    atom_offsets = atom_offsets.to(dev, torch.int64).contiguous()
    charges = (molecular_charges if molecular_charges is not None
               else torch.zeros(B, dtype=torch.float64)).to(dev, torch.float64).contiguous()
    uhf = (unpaired_electrons if unpaired_electrons is not None
           else torch.zeros(B, dtype=torch.int32)).to(dev, torch.int32).contiguous()
    if pc_charges is not None:
        pc_offsets = pc_offsets.to(dev, torch.int64).contiguous()
        pc_gammas = pc_gammas.to(dev, torch.float64).contiguous()
    static = (numbers, atom_offsets, charges, uhf, pc_offsets, pc_gammas, options)
    return _GFN2Energy.apply(positions, pc_positions, pc_charges, static)
