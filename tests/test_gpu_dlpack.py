"""A compute writes into a CUDA result arena; the results import into torch
through DLPack without a copy and equal the committed reference outputs."""
from __future__ import annotations

import gc

import numpy as np
import pytest
import torch

from conftest import TOL_E, TOL_F, TOL_Q, as_molecule
from xtbloom_b200 import abi, dlpack

pytestmark = pytest.mark.gpu


def test_cuda_arena_results_import_into_torch(cuda_lib, fixtures):
    mols = [as_molecule(s) for s in fixtures]
    b = abi.ragged_from_lists([m[0] for m in mols], [m[1] for m in mols],
                              [m[2] for m in mols], [m[3] for m in mols])
    nb, na = b.batch_size, b.total_atoms
    # energies | forces | charges | status | iterations | converged flags
    off_e, off_f = 0, 8 * nb
    off_q = off_f + 8 * 3 * na
    off_s = off_q + 8 * na
    off_i = off_s + 4 * nb
    off_c = off_i + 4 * nb
    size = off_c + nb
    arena = dlpack.ResultArena(cuda_lib.lib, size, abi.MEMORY_CUDA, 0)
    assert arena.memory_space == abi.MEMORY_CUDA
    cuda_lib.compute(b, outputs={"energies": arena.buffer(off_e, 8 * nb),
                                 "forces": arena.buffer(off_f, 8 * 3 * na),
                                 "atomic_charges": arena.buffer(off_q, 8 * na),
                                 "per_system_status": arena.buffer(off_s, 4 * nb),
                                 "scc_iterations": arena.buffer(off_i, 4 * nb),
                                 "scc_converged": arena.buffer(off_c, nb)})
    e = torch.from_dlpack(arena.slice(off_e, (nb,), np.float64))
    f = torch.from_dlpack(arena.slice(off_f, (na, 3), np.float64))
    q = torch.from_dlpack(arena.slice(off_q, (na,), np.float64))
    s = torch.from_dlpack(arena.slice(off_s, (nb,), np.int32))
    conv = torch.from_dlpack(arena.slice(off_c, (nb,), np.uint8))
    arena.close()               # the imported tensors hold the arena
    assert e.is_cuda and e.device.index == 0 and f.shape == (na, 3) and s.dtype == torch.int32
    assert e.data_ptr() == arena.data + off_e      # zero copy
    e, f, q, s, conv = (x.cpu().numpy() for x in (e, f, q, s, conv))
    assert (conv == 1).all()
    for i, sys_ in enumerate(fixtures):
        a0, a1 = b.atom_offsets[i], b.atom_offsets[i + 1]
        assert s[i] == sys_["status"] == 0, sys_["name"]
        assert abs(e[i] - sys_["energy"]) < TOL_E, sys_["name"]
        assert np.abs(f[a0:a1].reshape(-1) - np.asarray(sys_["forces"])).max() < TOL_F, sys_["name"]
        assert np.abs(q[a0:a1] - np.asarray(sys_["charges"])).max() < TOL_Q, sys_["name"]
    gc.collect()
    torch.cuda.synchronize()
