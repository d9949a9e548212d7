"""Seeded synthetic molecular workloads (alkane chains, hetero chains, water clusters).

The chain builder follows the idea of the reference's benchmark alkane
builder (benchmarks/natoms_scaling.py:804-890): a tetrahedral zig-zag
backbone grown from internal coordinates with random backbone dihedrals,
saturated with hydrogens, then jittered.  Bond lengths, dihedral
distributions, jitter and seeds are the ones the benchmark configurations
state: C-C 2.91, C-H 2.06, C-O 2.70, C-N 2.77, C-Cl 3.33, C-Br 3.65 bohr;
dihedrals uniform in {60, 180, 300} degrees plus N(0, 10 degrees); Gaussian
position jitter 0.03 bohr.  N-H bonds (not stated) use 1.91 bohr.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import RaggedBatch, ragged_from_lists

TETRA = math.acos(-1.0 / 3.0)          # 109.47 degrees
BOND = {("C", "C"): 2.91, ("C", "H"): 2.06, ("C", "O"): 2.70, ("C", "N"): 2.77,
        ("N", "H"): 1.91, ("C", "Cl"): 3.33, ("C", "Br"): 3.65}
Z = {"H": 1, "C": 6, "N": 7, "O": 8, "Cl": 17, "Br": 35}


def _bond(a: str, b: str) -> float:
    return BOND.get((a, b)) or BOND[(b, a)]


def _place(a, b, c, bond, angle, dihedral):
    """NeRF: position of d given a-b-c, |cd| = bond, angle bcd, dihedral abcd."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(angle), bond * math.sin(angle) * math.cos(dihedral),
                   bond * math.sin(angle) * math.sin(dihedral)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def _perp(u):
    t = np.array([1.0, 0.0, 0.0]) if abs(u[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(u, t)
    e1 /= np.linalg.norm(e1)
    return e1, np.cross(u, e1)


def chain(backbone: list[str], rng: np.random.Generator, jitter: float = 0.03,
          remove_h_at: int | None = None, halogens: dict | None = None):
    """Build one saturated chain.  backbone: heavy-atom symbols ('C','O','N').

    remove_h_at: index of a carbon that loses one hydrogen (radical).
    halogens: {carbon index: [symbols]} replacing hydrogens on that carbon."""
    n = len(backbone)
    pos = [np.zeros(3)]
    if n > 1:
        pos.append(np.array([_bond(backbone[0], backbone[1]), 0.0, 0.0]))
    if n > 2:
        b = _bond(backbone[1], backbone[2])
        ang = math.pi - TETRA
        pos.append(pos[1] + b * np.array([math.cos(ang), math.sin(ang), 0.0]))
    for k in range(3, n):
        dih = math.radians(rng.choice([60.0, 180.0, 300.0]) + rng.normal(0.0, 10.0))
        pos.append(_place(pos[k - 3], pos[k - 2], pos[k - 1], _bond(backbone[k - 1], backbone[k]), TETRA, dih))
    symbols = list(backbone)
    coords = list(pos)
    halogens = halogens or {}
    for i, el in enumerate(backbone):
        nbrs = [j for j in (i - 1, i + 1) if 0 <= j < n]
        valence = {"C": 4, "N": 3, "O": 2}[el]
        nh = valence - len(nbrs)
        subs = list(halogens.get(i, []))
        if remove_h_at == i:
            nh -= 1
        if nh <= 0:
            continue
        u = [(pos[j] - pos[i]) / np.linalg.norm(pos[j] - pos[i]) for j in nbrs]
        if len(u) == 0:
            dirs = [np.array([1.0, 0, 0]), np.array([-1 / 3, math.sqrt(8) / 3, 0]),
                    np.array([-1 / 3, -math.sqrt(2) / 3, math.sqrt(6) / 3]),
                    np.array([-1 / 3, -math.sqrt(2) / 3, -math.sqrt(6) / 3])]
        elif len(u) == 1:
            e1, e2 = _perp(u[0])
            phi0 = rng.uniform(0, 2 * math.pi)
            dirs = [math.cos(TETRA) * u[0] + math.sin(TETRA) * (math.cos(phi0 + k * 2 * math.pi / 3) * e1
                                                                 + math.sin(phi0 + k * 2 * math.pi / 3) * e2)
                    for k in range(3)]
        else:
            bis = -(u[0] + u[1])
            bis /= np.linalg.norm(bis)
            nrm = np.cross(u[0], u[1])
            nrm /= np.linalg.norm(nrm)
            half = 0.5 * TETRA
            dirs = [math.cos(half) * bis + math.sin(half) * nrm, math.cos(half) * bis - math.sin(half) * nrm]
        for k in range(nh):
            sym = subs.pop(0) if subs else "H"
            symbols.append(sym)
            coords.append(pos[i] + _bond(el, sym) * dirs[k])
    xyz = np.array(coords) + rng.normal(0.0, jitter, (len(coords), 3))
    return np.array([Z[s] for s in symbols], np.int32), xyz


def alkane(c: int, rng) -> tuple[np.ndarray, np.ndarray]:
    return chain(["C"] * c, rng)


def hetero_alkane(c: int, rng, fraction: float = 0.10):
    """C_cH_(2c+2) with a fraction of interior CH2 replaced by O or NH (no two adjacent)."""
    bb = ["C"] * c
    for i in range(1, c - 1):
        if rng.random() < fraction and bb[i - 1] == "C":
            bb[i] = "O" if rng.random() < 0.5 else "N"
    return chain(bb, rng)


def config0(count: int = 64, seed: int = 0):
    """64 C10H22 conformers (32 atoms, 62 AOs), seed 0."""
    rng = np.random.default_rng(seed)
    mols = [alkane(10, rng) for _ in range(count)]
    return ragged_from_lists([m[0] for m in mols], [m[1] for m in mols])


def config1(count: int = 4096, seed: int = 1):
    """Ragged batch of hetero chains, C count uniform in 3..40, seed 1."""
    rng = np.random.default_rng(seed)
    mols = [hetero_alkane(int(rng.integers(3, 41)), rng) for _ in range(count)]
    return ragged_from_lists([m[0] for m in mols], [m[1] for m in mols])


def water_cluster(nw: int, rng) -> tuple[np.ndarray, np.ndarray]:
    """(H2O)_nw: oxygens on a 5.4 bohr cubic lattice inside a sphere, jitter 0.2,
    O-H 1.81 bohr, H-O-H 104.5 degrees, uniform random orientation."""
    k = int(math.ceil((nw * 6 / math.pi) ** (1 / 3))) + 2
    g = np.arange(-k, k + 1) * 5.4
    pts = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
    pts = pts[np.argsort(np.linalg.norm(pts, axis=1), kind="stable")][:nw]
    numbers, coords = [], []
    half = math.radians(104.5) / 2
    for o in pts:
        o = o + rng.normal(0.0, 0.2, 3)
        qv = rng.normal(size=4)
        qv /= np.linalg.norm(qv)
        w, x, y, z = qv
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        h1 = R @ np.array([1.81 * math.sin(half), 0.0, 1.81 * math.cos(half)])
        h2 = R @ np.array([-1.81 * math.sin(half), 0.0, 1.81 * math.cos(half)])
        numbers += [8, 1, 1]
        coords += [o, o + h1, o + h2]
    return np.array(numbers, np.int32), np.array(coords)


def config3(count: int = 256, seed: int = 3):
    rng = np.random.default_rng(seed)
    mols = [water_cluster(int(rng.integers(100, 201)), rng) for _ in range(count)]
    return ragged_from_lists([m[0] for m in mols], [m[1] for m in mols])


def config2(count: int = 1024, seed: int = 2, npc: int = 200):
    """C20H42 conformers each embedded in 200 point charges (8-20 bohr shell)."""
    rng = np.random.default_rng(seed)
    mols = [alkane(20, rng) for _ in range(count)]
    b = ragged_from_lists([m[0] for m in mols], [m[1] for m in mols])
    pcp, pcq = [], []
    for _, xyz in mols:
        c = xyz.mean(0)
        q = rng.uniform(-0.5, 0.5, npc)
        q -= q.mean()
        d = rng.normal(size=(npc, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        r = (rng.uniform(8.0 ** 3, 20.0 ** 3, npc)) ** (1 / 3)
        pcp.append(c + d * r[:, None])
        pcq.append(q)
    b.point_charge_offsets = np.arange(count + 1, dtype=np.int64) * npc
    b.point_charge_positions = np.ascontiguousarray(np.concatenate(pcp).reshape(-1))
    b.point_charge_values = np.ascontiguousarray(np.concatenate(pcq))
    b.point_charge_gammas = np.full(count * npc, 999.0)
    return b


def config4(count: int = 2048, seed: int = 4):
    """Open-shell radicals (doublets, two spin channels): alkane chains C_nH_(2n+2)
    with n uniform in 4..45 and one H removed at a uniform random carbon; 15 % of
    them carry 1-3 H -> Cl or Br substitutions (C-Cl 3.33, C-Br 3.65 bohr), seed 4."""
    rng = np.random.default_rng(seed)
    mols = []
    for _ in range(count):
        c = int(rng.integers(4, 46))
        rm = int(rng.integers(0, c))
        hal: dict = {}
        if rng.random() < 0.15:
            for _ in range(int(rng.integers(1, 4))):
                hal.setdefault(int(rng.integers(0, c)), []).append("Cl" if rng.random() < 0.5 else "Br")
        mols.append(chain(["C"] * c, rng, remove_h_at=rm, halogens=hal))
    return ragged_from_lists([m[0] for m in mols], [m[1] for m in mols], np.zeros(count),
                             np.ones(count, np.int32), np.full(count, 2, np.int32))


def subset(b: RaggedBatch, idx) -> RaggedBatch:
    idx = list(idx)
    nums, poss = [], []
    for i in idx:
        a0, a1 = int(b.atom_offsets[i]), int(b.atom_offsets[i + 1])
        nums.append(b.atomic_numbers[a0:a1])
        poss.append(b.positions[3 * a0:3 * a1])
    sc = None if b.spin_channels is None else np.asarray(b.spin_channels)[idx]
    return ragged_from_lists(nums, poss, b.molecular_charges[idx], b.unpaired_electrons[idx], sc)


def molecule(b: RaggedBatch, i: int):
    a0, a1 = int(b.atom_offsets[i]), int(b.atom_offsets[i + 1])
    return np.asarray(b.atomic_numbers[a0:a1]), np.asarray(b.positions[3 * a0:3 * a1]).reshape(-1, 3)
