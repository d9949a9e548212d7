"""The differentiable energy (torch.autograd.Function over the CUDA library)."""
from __future__ import annotations

import numpy as np
import pytest

from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def tensors(b, dev):
    t = lambda a, dt: torch.as_tensor(np.asarray(a), dtype=dt, device=dev)  # noqa: E731
    return dict(numbers=t(b.atomic_numbers, torch.int32), atom_offsets=t(b.atom_offsets, torch.int64),
                positions=t(b.positions, torch.float64).reshape(-1, 3),
                pc_offsets=t(b.point_charge_offsets, torch.int64),
                pc_positions=t(b.point_charge_positions, torch.float64).reshape(-1, 3),
                pc_charges=t(b.point_charge_values, torch.float64),
                pc_gammas=t(b.point_charge_gammas, torch.float64))


def test_gradients_match_the_oracle():
    from oracle import gfn2
    from xtbloom_b200.autograd import gfn2_energy
    dev = torch.device("cuda", 0)
    b = W.config2(2, npc=40)
    a = tensors(b, dev)
    for k in ("positions", "pc_positions", "pc_charges"):
        a[k].requires_grad_(True)
    e = gfn2_energy(**a)
    w = torch.tensor([1.0, -0.5], dtype=torch.float64, device=dev)   # per-system weights
    (e * w).sum().backward()
    for i in range(2):
        z, x = W.molecule(b, i)
        p0, p1 = int(b.point_charge_offsets[i]), int(b.point_charge_offsets[i + 1])
        r = gfn2.singlepoint(z, x, pc_pos=b.point_charge_positions[3 * p0:3 * p1],
                             pc_q=b.point_charge_values[p0:p1], pc_gam=b.point_charge_gammas[p0:p1])
        a0, a1 = int(b.atom_offsets[i]), int(b.atom_offsets[i + 1])
        assert abs(e[i].item() - r.energy) < 1e-6
        wi = w[i].item()
        assert np.abs(a["positions"].grad[a0:a1].cpu().numpy() - wi * r.gradient).max() < 1e-5
        assert np.abs(a["pc_positions"].grad[p0:p1].cpu().numpy() - wi * r.pc_gradient).max() < 1e-5
        assert np.abs(a["pc_charges"].grad[p0:p1].cpu().numpy() - wi * r.pc_dq).max() < 1e-5


def test_directional_finite_differences():
    """Central differences (h = 1e-4) along random directions of positions, point-charge
    positions and point-charge values agree with the autograd directional derivative."""
    from xtbloom_b200.autograd import gfn2_energy
    dev = torch.device("cuda", 0)
    b = W.config2(1, npc=30)
    a = tensors(b, dev)
    tight = dict(ctol=1e-10, etol=1e-12)
    g = torch.Generator(device="cpu").manual_seed(5)
    for k in ("positions", "pc_positions", "pc_charges"):
        x = a[k].clone().requires_grad_(True)
        args = dict(a)
        args[k] = x
        gfn2_energy(**args, **tight).sum().backward()
        u = torch.randn(x.shape, generator=g, dtype=torch.float64).to(dev)
        u /= u.norm()
        h = 1e-4
        args[k] = (x + h * u).detach()
        ep = gfn2_energy(**args, **tight).item()
        args[k] = (x - h * u).detach()
        em = gfn2_energy(**args, **tight).item()
        assert abs((ep - em) / (2 * h) - (x.grad * u).sum().item()) < 1e-6, k
