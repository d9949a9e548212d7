"""CPU restatement of the reference's GFN2-xTB single point -- TEST ORACLE.

This module is test infrastructure: only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg may import it, and only as the checker.
It restates, in numpy, the FP64 algorithm of the reference CPU backend for
one molecule: basis expansion, coordination numbers, overlap and multipole
integrals, H0, ES2/ES3/AES2 electrostatics, self-consistent D4 with ATM,
repulsion, the generalized eigenproblem with Fermi smearing, Mulliken
populations, Johnson modified-Broyden mixing, the SCC energy functional and
the analytic gradient.  Each function cites the reference file:line it
follows (paths relative to the reference project root).

Parity pin: total energies and forces are checked against the reference
library compiled from its own sources (``oracle/ref.mk``) and against the
reference's committed tblite conformance goldens (see ``tests/test_oracle.py``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import eigh
from scipy.special import erf

from . import params as PR

SQRT3 = math.sqrt(3.0)
SQRT_PI3 = 5.5683279968317061          # pi^(3/2), common/integrals.cpp:30
INTEGRAL_CUTOFF = 25.0                 # common/integrals.hpp:26
DFACT = [1.0, 1.0, 3.0, 15.0, 105.0]   # common/sto.cpp:15

# Cartesian exponents in tblite order (common/integrals.cpp:48-51).
CART = {0: [(0, 0, 0)],
        1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
        2: [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]}
# Multipole operator powers [x,y,z,xx,xy,yy,xz,yz,zz] (common/integrals.cpp:54-64).
MPOW = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (0, 2, 0),
        (1, 0, 1), (0, 1, 1), (0, 0, 2)]
# Cartesian -> real spherical transforms (common/integrals.cpp:74-120).
TRANS = {
    0: np.array([[1.0]]),
    1: np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0]]),
    2: np.array([[0.0, SQRT3, 0.0, 0.0, 0.0, 0.0],
                 [0.0, 0.0, 0.0, 0.0, SQRT3, 0.0],
                 [-0.5, 0.0, 0.0, -0.5, 0.0, 1.0],
                 [0.0, 0.0, SQRT3, 0.0, 0.0, 0.0],
                 [0.5 * SQRT3, 0.0, 0.0, -0.5 * SQRT3, 0.0, 0.0]]),
}


# --------------------------------------------------------------------------
# Basis (model/gfn2/basis.cpp:66, common/sto.cpp:20-123)
# --------------------------------------------------------------------------
def sto_table(n: int, l: int, ng: int, p: dict):
    """STO-nG base exponents/coefficients (common/sto.cpp:20-67)."""
    if n == 6 and ng == 6:
        return (p["sto_alpha6s"], p["sto_coeff6s"]) if l == 0 else (p["sto_alpha6p"], p["sto_coeff6p"])
    typ = {0: n - 1, 1: n + 3, 2: n + 6, 3: n + 8, 4: n + 9}[l]
    return p[f"sto_alpha{ng}"][typ], p[f"sto_coeff{ng}"][typ]


def expand_sto(n: int, l: int, ng: int, zeta: float, p: dict):
    """Scaled, Cartesian-normalised primitives (common/sto.cpp:69-92)."""
    a0, c0 = sto_table(n, l, ng, p)
    alpha = np.asarray(a0, float) * zeta * zeta
    norm = (2.0 / math.pi * alpha) ** 0.75 * np.sqrt(4.0 * alpha) ** l / math.sqrt(DFACT[l])
    return alpha, np.asarray(c0, float) * norm


def orthogonalize_to_first(a1, c1, a, c):
    """Gram-Schmidt of a shell against the first shell of equal l (common/sto.cpp:94-121)."""
    s = np.sum(c1[:, None] * c[None, :] * (math.pi / (a1[:, None] + a[None, :])) ** 1.5)
    a = np.concatenate([a, a1])
    c = np.concatenate([c, -s * c1])
    nrm = np.sum(c[:, None] * c[None, :] * (math.pi / (a[:, None] + a[None, :])) ** 1.5)
    return a, c / math.sqrt(nrm)


@dataclass
class Basis:
    numbers: np.ndarray
    sh_atom: np.ndarray
    sh_l: np.ndarray
    sh_ao: np.ndarray          # first AO of each shell
    sh_zeta: np.ndarray
    prims: list                # (alpha, coeff) per shell
    ao_atom: np.ndarray
    ao_shell: np.ndarray
    nao: int
    atom_sh: np.ndarray        # first shell of each atom (len N+1)
    sh_local: np.ndarray       # element-local shell index
    refocc: np.ndarray         # reference shell occupations


def make_basis(numbers: np.ndarray) -> Basis:
    p = PR.load()
    sh_atom, sh_l, sh_ao, sh_zeta, prims, sh_local, refocc = [], [], [], [], [], [], []
    atom_sh = [0]
    ao = 0
    for a, z in enumerate(numbers):
        zi = int(z) - 1
        first = {}
        for s in range(int(p["gfn2_nshell"][zi])):
            l = int(p["gfn2_shell_l"][zi, s])
            n = int(p["gfn2_shell_n"][zi, s])
            ng = int(p["gfn2_shell_ngauss"][zi, s])
            zeta = float(p["gfn2_shell_slater"][zi, s])
            alpha, coeff = expand_sto(n, l, ng, zeta, p)
            if l in first:
                a1, c1 = prims[first[l]]
                alpha, coeff = orthogonalize_to_first(a1, c1, alpha, coeff)
            else:
                first[l] = len(prims)
            sh_atom.append(a)
            sh_l.append(l)
            sh_ao.append(ao)
            sh_zeta.append(zeta)
            prims.append((alpha, coeff))
            sh_local.append(s)
            refocc.append(float(p["gfn2_shell_refocc"][zi, s]))
            ao += 2 * l + 1
        atom_sh.append(len(sh_atom))
    sh_l = np.array(sh_l)
    sh_ao = np.array(sh_ao)
    ao_atom = np.concatenate([[sh_atom[i]] * (2 * l + 1) for i, l in enumerate(sh_l)]).astype(int)
    ao_shell = np.concatenate([[i] * (2 * l + 1) for i, l in enumerate(sh_l)]).astype(int)
    return Basis(np.asarray(numbers), np.array(sh_atom), sh_l, sh_ao, np.array(sh_zeta), prims,
                 ao_atom, ao_shell, ao, np.array(atom_sh), np.array(sh_local), np.array(refocc))


# --------------------------------------------------------------------------
# Coordination number, GFN2 double exponential (model/gfn2/coordination.cpp:120-138,197-320)
# --------------------------------------------------------------------------
def _logistic(x):
    return 0.5 * (1.0 + np.tanh(0.5 * x))


def cn_dexp(numbers, pos, with_deriv=False):
    p = PR.load()
    rc = (4.0 / 3.0) * PR.ANGSTROM_TO_BOHR * p["covalent_radii_angstrom"][numbers - 1]
    n = len(numbers)
    cn = np.zeros(n)
    dcn = np.zeros((n, n)) if with_deriv else None   # d count_ij / d r_ij
    for i in range(n):
        for j in range(i):
            d = pos[i] - pos[j]
            r = math.sqrt(d @ d)
            if r * r > 25.0 ** 2:
                continue
            rad = rc[i] + rc[j]
            f1 = _logistic(10.0 * (rad / r - 1.0))
            f2 = _logistic(20.0 * ((rad + 2.0) / r - 1.0))
            cn[i] += f1 * f2
            cn[j] += f1 * f2
            if with_deriv:
                dv = -(10.0 * rad * f1 * (1 - f1) * f2 + 20.0 * (rad + 2.0) * f2 * (1 - f2) * f1) / (r * r)
                dcn[i, j] = dcn[j, i] = dv
    return cn, dcn


def cn_vjp(pos, dcn, adj, grad):
    """add_coordination_gradient_cpu (model/gfn2/coordination.cpp:257-320)."""
    n = len(pos)
    for i in range(n):
        for j in range(i):
            if dcn[i, j] == 0.0:
                continue
            d = pos[i] - pos[j]
            r = math.sqrt(d @ d)
            g = (adj[i] + adj[j]) * dcn[i, j] / r * d
            grad[i] += g
            grad[j] -= g


# --------------------------------------------------------------------------
# Overlap / multipole integrals (common/integrals.cpp:356-690)
# --------------------------------------------------------------------------
def _axis_table(pa, pb, inv2p, amax, bmax):
    """1-D Obara-Saika overlap recurrence (common/integrals.cpp:362-388).

    pa, pb, inv2p broadcast arrays; returns T[a][b] lists of arrays."""
    T = [[None] * (bmax + 1) for _ in range(amax + 1)]
    one = np.ones_like(pa)
    T[0][0] = one
    for a in range(1, amax + 1):
        T[a][0] = pa * T[a - 1][0]
        if a > 1:
            T[a][0] = T[a][0] + (a - 1) * inv2p * T[a - 2][0]
    for b in range(1, bmax + 1):
        T[0][b] = pb * T[0][b - 1]
        if b > 1:
            T[0][b] = T[0][b] + (b - 1) * inv2p * T[0][b - 2]
        for a in range(1, amax + 1):
            T[a][b] = pa * T[a - 1][b] + b * inv2p * T[a - 1][b - 1]
            if a > 1:
                T[a][b] = T[a][b] + (a - 1) * inv2p * T[a - 2][b]
    return T


def _traceless(m):
    """Raw second moments [xx,xy,yy,xz,yz,zz] -> tblite traceless form (common/integrals.cpp:425-438)."""
    tr = 0.5 * (m[0] + m[2] + m[5])
    return np.array([1.5 * m[0] - tr, 1.5 * m[1], 1.5 * m[2] - tr, 1.5 * m[3], 1.5 * m[4], 1.5 * m[5] - tr])


def shell_pair(lb, lk, ab, cb, ak, ck, v, grad=False):
    """Local bra/ket block about the ket centre (common/integrals.cpp:498-652).

    v = R_ket - R_bra.  Returns S[sb,sk], M[9,sb,sk] (dipole + traceless
    quadrupole, operator origin at the ket atom) and, with grad, their
    derivatives with respect to R_ket: dS[3,sb,sk], dM[3,9,sb,sk]."""
    r2 = float(v @ v)
    AK = ak[:, None]
    AB = ab[None, :]
    asum = AK + AB
    inv = 1.0 / asum
    est = AK * AB * r2 * inv
    keep = est <= INTEGRAL_CUTOFF
    pref = np.where(keep, np.exp(-np.where(keep, est, 0.0)) * SQRT_PI3 * inv ** 1.5
                    * ck[:, None] * cb[None, :], 0.0)
    inv2p = 0.5 * inv
    amax = lk + (3 if grad else 2)
    tabs = []
    for c in range(3):
        pa = -v[c] * AB * inv
        pb = v[c] * AK * inv
        tabs.append(_axis_table(pa, pb, inv2p, amax, lb))
    cb_ = CART[lb]
    ck_ = CART[lk]
    nb, nk = len(cb_), len(ck_)
    S = np.zeros((nb, nk))
    M = np.zeros((9, nb, nk))
    dS = np.zeros((3, nb, nk))
    dM = np.zeros((3, 9, nb, nk))
    for ib, bp in enumerate(cb_):
        for ik, kp in enumerate(ck_):
            one = [tabs[c][kp[c]][bp[c]] for c in range(3)]
            S[ib, ik] = np.sum(pref * one[0] * one[1] * one[2])
            if grad:
                for c in range(3):
                    a = kp[c]
                    d1 = 2.0 * AK * tabs[c][a + 1][bp[c]]
                    if a > 0:
                        d1 = d1 - a * tabs[c][a - 1][bp[c]]
                    o = [one[(c + 1) % 3], one[(c + 2) % 3]]
                    dS[c, ib, ik] = np.sum(pref * d1 * o[0] * o[1])
            for m, mp in enumerate(MPOW):
                od = [tabs[c][kp[c] + mp[c]][bp[c]] for c in range(3)]
                M[m, ib, ik] = np.sum(pref * od[0] * od[1] * od[2])
                if grad:
                    for c in range(3):
                        e = kp[c] + mp[c]
                        d1 = 2.0 * AK * tabs[c][e + 1][bp[c]]
                        if e > 0:
                            d1 = d1 - e * tabs[c][e - 1][bp[c]]
                        dM[c, m, ib, ik] = np.sum(pref * d1 * od[(c + 1) % 3] * od[(c + 2) % 3])
    TB, TK = TRANS[lb], TRANS[lk]
    Ss = TB @ S @ TK.T
    Ms = np.einsum("ij,mjk,lk->mil", TB, M, TK)
    Ms[3:] = _traceless(Ms[3:])
    if not grad:
        return Ss, Ms
    dSs = np.einsum("ij,cjk,lk->cil", TB, dS, TK)
    dMs = np.einsum("ij,cmjk,lk->cmil", TB, dM, TK)
    for c in range(3):
        dMs[c, 3:] = _traceless(dMs[c, 3:])
    return Ss, Ms, dSs, dMs


def shift_reverse(v, S, D, Q):
    """Reverse (ket-row) element with the operator origin moved to the bra atom
    (common/integrals.cpp:824-850)."""
    Dr = D + v[:, None, None] * S
    sh = np.array([2 * v[0] * D[0] + v[0] * v[0] * S,
                   v[0] * D[1] + v[1] * D[0] + v[0] * v[1] * S,
                   2 * v[1] * D[1] + v[1] * v[1] * S,
                   v[0] * D[2] + v[2] * D[0] + v[0] * v[2] * S,
                   v[1] * D[2] + v[2] * D[1] + v[1] * v[2] * S,
                   2 * v[2] * D[2] + v[2] * v[2] * S])
    tr = 0.5 * (sh[0] + sh[2] + sh[5])
    Qr = Q + 1.5 * sh
    Qr[0] -= tr
    Qr[2] -= tr
    Qr[5] -= tr
    return Dr, Qr


def integrals(basis: Basis, pos):
    """S, D[3], Q[6] full matrices (evaluate_overlap_cpu / evaluate_multipole_cpu,
    common/integrals.cpp:700-865).  D[c][mu][nu] = <mu|(r-R_nu)_c|nu>."""
    n = basis.nao
    S = np.zeros((n, n))
    D = np.zeros((3, n, n))
    Q = np.zeros((6, n, n))
    nat = len(basis.numbers)
    for A in range(nat):                    # ket atom
        for B in range(A + 1):              # bra atom
            v = pos[A] - pos[B]
            for ks in range(basis.atom_sh[A], basis.atom_sh[A + 1]):
                for bs in range(basis.atom_sh[B], basis.atom_sh[B + 1]):
                    if A == B and bs > ks:
                        continue
                    lb, lk = basis.sh_l[bs], basis.sh_l[ks]
                    ab, cb = basis.prims[bs]
                    ak, ck = basis.prims[ks]
                    Ss, Ms = shell_pair(lb, lk, ab, cb, ak, ck, v)
                    ib = slice(basis.sh_ao[bs], basis.sh_ao[bs] + 2 * lb + 1)
                    ik = slice(basis.sh_ao[ks], basis.sh_ao[ks] + 2 * lk + 1)
                    S[ib, ik] = Ss
                    S[ik, ib] = Ss.T
                    Dl, Ql = Ms[:3], Ms[3:]
                    if bs == ks:
                        # same shell, same centre: exactly symmetric block
                        Dl = 0.5 * (Dl + np.swapaxes(Dl, 1, 2))
                        Ql = 0.5 * (Ql + np.swapaxes(Ql, 1, 2))
                        D[:, ib, ik] = Dl
                        Q[:, ib, ik] = Ql
                        continue
                    D[:, ib, ik] = Dl
                    Q[:, ib, ik] = Ql
                    Dr, Qr = shift_reverse(v, Ss, Dl, Ql)
                    D[:, ik, ib] = np.swapaxes(Dr, 1, 2)
                    Q[:, ik, ib] = np.swapaxes(Qr, 1, 2)
    return S, D, Q


def integral_vjp(basis: Basis, pos, aS, aD, aQ, grad):
    """dE/dR from adjoints of S, D, Q (add_overlap_gradient_cpu and
    add_multipole_gradient_cpu with add_multipole_shift_pullback,
    common/integrals.cpp:440-496, 867-1145)."""
    nat = len(basis.numbers)
    for A in range(nat):
        for B in range(A):
            v = pos[A] - pos[B]
            g = np.zeros(3)
            for ks in range(basis.atom_sh[A], basis.atom_sh[A + 1]):
                for bs in range(basis.atom_sh[B], basis.atom_sh[B + 1]):
                    lb, lk = basis.sh_l[bs], basis.sh_l[ks]
                    ab, cb = basis.prims[bs]
                    ak, ck = basis.prims[ks]
                    Ss, Ms, dSs, dMs = shell_pair(lb, lk, ab, cb, ak, ck, v, grad=True)
                    ib = slice(basis.sh_ao[bs], basis.sh_ao[bs] + 2 * lb + 1)
                    ik = slice(basis.sh_ao[ks], basis.sh_ao[ks] + 2 * lk + 1)
                    # forward (bra row, ket col) adjoints; reverse (ket row, bra col)
                    sA = aS[ib, ik] + aS[ik, ib].T
                    fD = aD[:, ib, ik]
                    rD = np.swapaxes(aD[:, ik, ib], 1, 2)
                    fQ = aQ[:, ib, ik]
                    rQ = np.swapaxes(aQ[:, ik, ib], 1, 2)
                    Dl = Ms[:3]
                    # pullback of the origin shift (reverse elements)
                    dsum = rQ[0] + rQ[2] + rQ[5]
                    raw = np.array([1.5 * rQ[0] - 0.5 * dsum, 1.5 * rQ[1], 1.5 * rQ[2] - 0.5 * dsum,
                                    1.5 * rQ[3], 1.5 * rQ[4], 1.5 * rQ[5] - 0.5 * dsum])
                    x, y, z = v
                    axx, axy, ayy, axz, ayz, azz = raw
                    sadj = sA + rD[0] * x + rD[1] * y + rD[2] * z \
                        + axx * x * x + axy * x * y + ayy * y * y + axz * x * z + ayz * y * z + azz * z * z
                    dadj = fD + rD
                    dadj = dadj + np.array([2 * axx * x + axy * y + axz * z,
                                            axy * x + 2 * ayy * y + ayz * z,
                                            axz * x + ayz * y + 2 * azz * z])
                    qadj = fQ + rQ
                    dx, dy, dz = Dl
                    vadj = np.array([
                        np.sum(rD[0] * Ss + axx * (2 * dx + 2 * x * Ss) + axy * (dy + y * Ss) + axz * (dz + z * Ss)),
                        np.sum(rD[1] * Ss + axy * (dx + x * Ss) + ayy * (2 * dy + 2 * y * Ss) + ayz * (dz + z * Ss)),
                        np.sum(rD[2] * Ss + axz * (dx + x * Ss) + ayz * (dy + y * Ss) + azz * (2 * dz + 2 * z * Ss)),
                    ])
                    for c in range(3):
                        g[c] += vadj[c] + np.sum(sadj * dSs[c]) + np.sum(dadj * dMs[c, :3]) \
                            + np.sum(qadj * dMs[c, 3:])
            grad[A] += g
            grad[B] -= g


# --------------------------------------------------------------------------
# H0 (model/gfn2/h0.cpp:248-597)
# --------------------------------------------------------------------------
@dataclass
class H0Data:
    level: np.ndarray
    kcn: np.ndarray
    shpoly: np.ndarray
    rad: np.ndarray
    pair_scale: np.ndarray   # shell x shell


def make_h0(basis: Basis) -> H0Data:
    p = PR.load()
    g = p["g"]
    z = basis.numbers[basis.sh_atom] - 1
    loc = basis.sh_local
    level = p["gfn2_shell_level"][z, loc] * PR.EV_TO_HARTREE
    kcn = p["gfn2_shell_kcn"][z, loc] * PR.EV_TO_HARTREE
    shpoly = p["gfn2_shell_shpoly"][z, loc]
    rad = p["atomic_radii_angstrom"][basis.numbers - 1] * PR.ANGSTROM_TO_BOHR
    zeta = basis.sh_zeta
    en = p["gfn2_en"][z]
    zs = (2.0 * np.sqrt(zeta[:, None] * zeta[None, :]) / (zeta[:, None] + zeta[None, :])) ** g["wexp"]
    es = 1.0 + g["enscale"] * (en[:, None] - en[None, :]) ** 2
    ss = p["gfn2_shell_pair_scale"][basis.sh_l[:, None], basis.sh_l[None, :]]
    return H0Data(level, kcn, shpoly, rad, zs * es * ss * g["pair_scale_default"])


def _h0_factors(basis, h0: H0Data, pos, cn):
    """Per shell pair factor 0.5*(h_i+h_j)*spatial_scale and its radial derivative."""
    ns = len(basis.sh_l)
    lev = h0.level - h0.kcn * cn[basis.sh_atom]
    fac = np.zeros((ns, ns))
    spat = np.ones((ns, ns))
    dspat = np.zeros((ns, ns))
    for i in range(ns):
        A = basis.sh_atom[i]
        for j in range(ns):
            B = basis.sh_atom[j]
            if A != B:
                d = pos[A] - pos[B]
                r = math.sqrt(d @ d)
                rr = math.sqrt(r / (h0.rad[A] + h0.rad[B]))
                p1 = 1.0 + h0.shpoly[i] * rr
                p2 = 1.0 + h0.shpoly[j] * rr
                spat[i, j] = h0.pair_scale[i, j] * p1 * p2
                dspat[i, j] = h0.pair_scale[i, j] * (h0.shpoly[i] * p2 + h0.shpoly[j] * p1) * rr / (2.0 * r)
            fac[i, j] = 0.5 * (lev[i] + lev[j]) * spat[i, j]
    return lev, fac, spat, dspat


def _expand(basis, x):
    """Shell x shell -> AO x AO."""
    return x[np.ix_(basis.ao_shell, basis.ao_shell)]


def h0_matrix(basis, h0: H0Data, pos, cn, S):
    _, fac, _, _ = _h0_factors(basis, h0, pos, cn)
    return S * _expand(basis, fac)


def h0_vjp(basis, h0: H0Data, pos, cn, S, P, aS, acn, grad):
    """add_h0_vjp_cpu (model/gfn2/h0.cpp:469-597)."""
    lev, fac, spat, dspat = _h0_factors(basis, h0, pos, cn)
    aS += P * _expand(basis, fac)
    ns = len(basis.sh_l)
    # block weights sum_{mu in i, nu in j} P S
    PS = P * S
    bw = np.zeros((ns, ns))
    np.add.at(bw, (basis.ao_shell[:, None], basis.ao_shell[None, :]), PS)
    lw = 0.5 * bw * spat
    for i in range(ns):
        for j in range(ns):
            acn[basis.sh_atom[i]] -= h0.kcn[i] * lw[i, j]
            acn[basis.sh_atom[j]] -= h0.kcn[j] * lw[i, j]
            A, B = basis.sh_atom[i], basis.sh_atom[j]
            if A != B:
                d = pos[A] - pos[B]
                r = math.sqrt(d @ d)
                rad = bw[i, j] * 0.5 * (lev[i] + lev[j]) * dspat[i, j]
                g = rad / r * d
                grad[A] += g
                grad[B] -= g


# --------------------------------------------------------------------------
# ES2 / ES3 (model/gfn2/es2.cpp:205-300,1040-1110; model/gfn2/es3.cpp:190-230)
# --------------------------------------------------------------------------
def shell_hardness(basis):
    p = PR.load()
    z = basis.numbers[basis.sh_atom] - 1
    return p["gfn2_gam"][z] * p["gfn2_shell_hubbard_scale"][z, basis.sh_local]


def shell_gamma3(basis):
    p = PR.load()
    g = p["g"]
    z = basis.numbers[basis.sh_atom] - 1
    sc = np.array([g["es3_s"], g["es3_p"], g["es3_d"]])[basis.sh_l]
    return p["gfn2_gam3"][z] * sc


def es2_gamma(basis, pos):
    eta = shell_hardness(basis)
    avg = 0.5 * (eta[:, None] + eta[None, :])
    at = basis.sh_atom
    d = pos[at][:, None, :] - pos[at][None, :, :]
    r2 = np.sum(d * d, axis=-1)
    same = at[:, None] == at[None, :]
    gam = np.where(same, avg, 1.0 / np.sqrt(r2 + 1.0 / avg ** 2))
    return gam


def es2_grad(basis, pos, gam, qsh, grad):
    at = basis.sh_atom
    n = len(basis.numbers)
    w = np.zeros((n, n))
    g3 = qsh[:, None] * qsh[None, :] * gam ** 3
    np.add.at(w, (at[:, None], at[None, :]), g3)
    for A in range(n):
        for B in range(A):
            d = pos[A] - pos[B]
            g = -w[A, B] * d
            grad[A] += g
            grad[B] -= g


# --------------------------------------------------------------------------
# AES2 (model/gfn2/aes2.cpp:356-713, 891-1000)
# --------------------------------------------------------------------------
QSCALE = np.array([1.0, 2.0, 1.0, 2.0, 2.0, 1.0])


@dataclass
class AES2:
    dk: np.ndarray
    qk: np.ndarray
    mrad: np.ndarray
    dmrad: np.ndarray
    pairs: list   # (f, s, disp, k3, k5, avg_rad)


def aes2_setup(numbers, pos, cn):
    p = PR.load()
    g = p["g"]
    z = numbers - 1
    r0 = p["gfn2_mprad"][z]
    vcn = p["gfn2_mpvcn"][z]
    arg = g["mp_kexp"] * (cn - vcn - g["mp_shift"])
    frac = _logistic(arg)
    mrad = r0 + (g["mp_rmax"] - r0) * frac
    dmrad = (g["mp_rmax"] - r0) * g["mp_kexp"] * frac * (1 - frac)
    pairs = []
    n = len(numbers)
    for s in range(n):
        for f in range(s):
            d = pos[f] - pos[s]
            r = math.sqrt(d @ d)
            R = 0.5 * (mrad[f] + mrad[s])
            sc = R / r
            k3 = 1.0 / r ** 3 / (1.0 + 6.0 * sc ** 3)
            k5 = 1.0 / r ** 5 / (1.0 + 6.0 * sc ** 4)
            pairs.append((f, s, d, k3, k5, R))
    return AES2(p["gfn2_dkernel"][z], p["gfn2_qkernel"][z], mrad, dmrad, pairs)


def _sq(d, k5):
    return np.array([d[0] * d[0], 2 * d[0] * d[1], d[1] * d[1], 2 * d[0] * d[2], 2 * d[1] * d[2], d[2] * d[2]]) * k5


def aes2_potential(a: AES2, q, dip, qp):
    n = len(q)
    vat = np.zeros(n)
    vd = 2.0 * a.dk[:, None] * dip
    vq = 2.0 * a.qk[:, None] * QSCALE[None, :] * qp
    for f, s, d, k3, k5, _ in a.pairs:
        sd = d * k3
        sq = _sq(d, k5)
        iso = (d @ d) * k5
        vat[f] += sd @ dip[s] + sq @ qp[s]
        vat[s] += -(sd @ dip[f]) + sq @ qp[f]
        vd[f] += -q[s] * sd + iso * dip[s] - 3 * k5 * d * (d @ dip[s])
        vd[s] += q[f] * sd + iso * dip[f] - 3 * k5 * d * (d @ dip[f])
        vq[f] += q[s] * sq
        vq[s] += q[f] * sq
    return vat, vd, vq


def aes2_energy(a: AES2, q, dip, qp):
    e = np.sum(a.dk * np.sum(dip * dip, 1)) + np.sum(a.qk * np.sum(QSCALE * qp * qp, 1))
    for f, s, d, k3, k5, _ in a.pairs:
        sq = _sq(d, k5)
        e += k3 * (d @ (q[f] * dip[s] - q[s] * dip[f]))
        e += k5 * ((d @ d) * (dip[f] @ dip[s]) - 3 * (d @ dip[f]) * (d @ dip[s]))
        e += q[f] * (sq @ qp[s]) + q[s] * (sq @ qp[f])
    return e


def aes2_vjp(a: AES2, q, dip, qp, grad, acn):
    """pair_vjp (model/gfn2/aes2.cpp:596-713)."""
    for f, s, d, k3, k5, R in a.pairs:
        r = math.sqrt(d @ d)
        sc = R / r
        f3 = 1.0 / (1.0 + 6.0 * sc ** 3)
        f5 = 1.0 / (1.0 + 6.0 * sc ** 4)
        cdv = q[f] * dip[s] - q[s] * dip[f]
        pf, ps = d @ dip[f], d @ dip[s]
        dd = dip[f] @ dip[s]
        cdn = d @ cdv
        r2 = d @ d
        ddn = r2 * dd - 3 * pf * ps
        T = q[f] * qp[s] + q[s] * qp[f]
        tv = np.array([T[0] * d[0] + T[1] * d[1] + T[3] * d[2],
                       T[1] * d[0] + T[2] * d[1] + T[4] * d[2],
                       T[3] * d[0] + T[4] * d[1] + T[5] * d[2]])
        cqn = d @ tv
        k3d = -3.0 * f3 * k3 / r
        k5d = -(1.0 + 4.0 * f5) * k5 / r
        k3r = -3.0 * (1.0 - f3) * k3 / R
        k5r = -4.0 * (1.0 - f5) * k5 / R
        k5n = ddn + cqn
        erd = k3r * cdn + k5r * k5n
        ddd = 2 * dd * d - 3 * (pf * dip[s] + ps * dip[f])
        g = k3 * cdv + k3d * cdn * d / r + k5 * (ddd + 2 * tv) + k5d * k5n * d / r
        grad[f] += g
        grad[s] -= g
        acn[f] += 0.5 * erd * a.dmrad[f]
        acn[s] += 0.5 * erd * a.dmrad[s]


# --------------------------------------------------------------------------
# D4 (model/gfn2/d4.cpp:49-60,283-470,560-1364)
# --------------------------------------------------------------------------
@dataclass
class D4:
    numbers: np.ndarray
    cn: np.ndarray
    pairs: list          # (f, s, disp, damp, ddamp, r0, count_deriv)
    zw: np.ndarray = None


def d4_setup(numbers, pos):
    p = PR.load()
    g = p["g"]
    z = numbers - 1
    n = len(numbers)
    cn = np.zeros(n)
    pairs = []
    for s in range(1, n):
        for f in range(s):
            d = pos[f] - pos[s]
            r2 = d @ d
            rcov = p["d4_rcov"][z[f]] + p["d4_rcov"][z[s]]
            den = abs(p["d4_en"][z[f]] - p["d4_en"][z[s]])
            enf = 4.10451 * math.exp(-(den + 19.08857) ** 2 / (2.0 * 11.28174 * 11.28174))
            cderiv = 0.0
            if r2 <= 30.0 ** 2:
                r = math.sqrt(r2)
                x = 7.5 * (r - rcov) / rcov
                c = 0.5 * enf * (1.0 + math.erf(-x))
                cn[f] += c
                cn[s] += c
                cderiv = -enf * 7.5 * math.exp(-x * x) / math.sqrt(math.pi) / rcov
            rrij = 3.0 * p["d4_r4r2"][z[f]] * p["d4_r4r2"][z[s]]
            r0 = g["d4_a1"] * math.sqrt(rrij) + g["d4_a2"]
            damp = ddamp = 0.0
            if r2 <= 50.0 ** 2:
                r4 = r2 * r2
                r6 = r4 * r2
                t6 = 1.0 / (r6 + r0 ** 6)
                t8 = 1.0 / (r4 * r4 + r0 ** 8)
                damp = g["d4_s6"] * t6 + g["d4_s8"] * rrij * t8
                ddamp = g["d4_s6"] * (-6.0 * r4 * t6 * t6) + g["d4_s8"] * rrij * (-8.0 * r6 * t8 * t8)
            pairs.append((f, s, d, damp, ddamp, r0, cderiv))
    return D4(numbers, cn, pairs)


def d4_weights(numbers, cn, q):
    """prepare_weight_slice (model/gfn2/d4.cpp:298-366): w, dw/dcn, dw/dq per atom."""
    p = PR.load()
    out = []
    for a, zz in enumerate(numbers):
        zi = zz - 1
        off, cnt = int(p["d4_ref_offset"][zi]), int(p["d4_ref_count"][zi])
        rcn = p["d4_ref_cn"][off:off + cnt]
        rq = p["d4_ref_q"][off:off + cnt]
        ng = p["d4_ref_ngauss"][off:off + cnt]
        num = np.zeros(cnt)
        dnum = np.zeros(cnt)
        for r in range(cnt):
            for gg in range(1, ng[r] + 1):
                fct = gg * 6.0
                dl = cn[a] - rcn[r]
                val = math.exp(-fct * dl * dl)
                num[r] += val
                dnum[r] += 2.0 * fct * (rcn[r] - cn[a]) * val
        norm, dnorm = num.sum(), dnum.sum()
        inv = 1.0 / norm if abs(norm) > 1.4916681462400413e-154 else 0.0
        if inv == 0.0:
            cw = np.where(np.abs(rcn.max() - rcn) < 1e-12, 1.0, 0.0)
            dcw = np.zeros(cnt)
        else:
            cw = num * inv
            dcw = inv * (dnum - num * dnorm * inv)
        qmod = q[a] + p["d4_zeff"][zi]
        cst = p["d4_eta"][zi] * 2.0
        qref = rq + p["d4_zeff"][zi]
        if qmod < 0.0:
            scl = np.full(cnt, math.exp(3.0))
            dscl = np.zeros(cnt)
        else:
            inner = np.exp(cst * (1.0 - qref / qmod))
            scl = np.exp(3.0 * (1.0 - inner))
            dscl = -3.0 * cst * inner * scl * qref / (qmod * qmod)
        out.append((off, cnt, cw * scl, dcw * scl, cw * dscl))
    return out


def _pair_c6(wa, wb, c6ref):
    oa, ca, w1, dcn1, dq1 = wa
    ob, cb, w2, dcn2, dq2 = wb
    R = c6ref[oa:oa + ca, ob:ob + cb]
    return (w1 @ R @ w2, dcn1 @ R @ w2, w1 @ R @ dcn2, dq1 @ R @ w2, w1 @ R @ dq2)


def d4_two_body(d4: D4, q, grad=None):
    """Energy, atom potential (and at fixed q the gradient) of the D4 two-body term."""
    p = PR.load()
    c6ref = p["d4_ref_c6"]
    W = d4_weights(d4.numbers, d4.cn, q)
    n = len(q)
    e = 0.0
    vat = np.zeros(n)
    acn = np.zeros(n)
    for f, s, d, damp, ddamp, r0, _ in d4.pairs:
        if damp == 0.0:
            continue
        c6, dcf, dcs, dqf, dqs = _pair_c6(W[f], W[s], c6ref)
        e -= c6 * damp
        vat[f] -= dqf * damp
        vat[s] -= dqs * damp
        if grad is not None:
            g = -c6 * ddamp * d
            grad[f] += g
            grad[s] -= g
            acn[f] -= dcf * damp
            acn[s] -= dcs * damp
    if grad is not None:
        d4_cn_vjp(d4, acn, grad)
    return e, vat


def d4_cn_vjp(d4: D4, acn, grad):
    for f, s, d, _, _, _, cd in d4.pairs:
        if cd == 0.0:
            continue
        r = math.sqrt(d @ d)
        g = cd * (acn[f] + acn[s]) / r * d
        grad[f] += g
        grad[s] -= g


def d4_atm(d4: D4, grad=None):
    """evaluate_d4_atm_cpu / add_d4_atm_gradient_cpu (model/gfn2/d4.cpp:1120-1362)."""
    p = PR.load()
    g = p["g"]
    c6ref = p["d4_ref_c6"]
    n = len(d4.numbers)
    W = d4_weights(d4.numbers, d4.cn, np.zeros(n))
    pi = {}
    for f, s, d, _, _, r0, _ in d4.pairs:
        pi[(f, s)] = (d, r0)
    c6c = {}

    def c6(a, b):
        key = (a, b)
        if key not in c6c:
            c6c[key] = _pair_c6(W[a], W[b], c6ref)
        return c6c[key]

    e = 0.0
    acn = np.zeros(n)
    cut2 = 25.0 ** 2
    ex3 = 16.0 / 3.0
    for i in range(2, n):
        for j in range(1, i):
            vij, r0ij = pi[(j, i)]
            r2ij = vij @ vij
            if r2ij > cut2:
                continue
            cij = c6(i, j)
            for k in range(j):
                vik, r0ik = pi[(k, i)]
                vjk, r0jk = pi[(k, j)]
                r2ik = vik @ vik
                r2jk = vjk @ vjk
                if r2ik > cut2 or r2jk > cut2:
                    continue
                cik = c6(i, k)
                cjk = c6(j, k)
                r2p = r2ij * r2ik * r2jk
                r1p = math.sqrt(r2p)
                r3p = r2p * r1p
                r5p = r3p * r2p
                ratio = r0ij * r0ik * r0jk / r1p
                rpow = ratio ** ex3
                damp = 1.0 / (1.0 + 6.0 * rpow)
                ang = 0.375 * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik) * (-r2ij + r2jk + r2ik) / r5p + 1.0 / r3p
                prod = cij[0] * cik[0] * cjk[0]
                c9 = -g["d4_s9"] * math.sqrt(abs(prod))
                e -= ang * damp * c9
                if grad is None:
                    continue
                ddmp = -2.0 * 16.0 * rpow * damp * damp

                def dg(t, o1, o2, vec):
                    dang = -0.375 * (t ** 3 + t * t * (o1 + o2) + t * (3 * o1 * o1 + 2 * o1 * o2 + 3 * o2 * o2)
                                     - 5.0 * (o1 - o2) ** 2 * (o1 + o2)) / r5p
                    return c9 * (-dang * damp + ang * ddmp) / t * vec

                gij = dg(r2ij, r2jk, r2ik, vij)
                gik = dg(r2ik, r2jk, r2ij, vik)
                gjk = dg(r2jk, r2ik, r2ij, vjk)
                grad[i] -= gij + gik
                grad[j] += gij - gjk
                grad[k] += gik + gjk
                de = ang * damp * c9
                acn[i] -= 0.5 * de * (cij[1] / cij[0] + cik[1] / cik[0])
                acn[j] -= 0.5 * de * (cij[2] / cij[0] + cjk[1] / cjk[0])
                acn[k] -= 0.5 * de * (cik[2] / cik[0] + cjk[2] / cjk[0])
    if grad is not None:
        d4_cn_vjp(d4, acn, grad)
    return e


# --------------------------------------------------------------------------
# Repulsion (model/gfn2/repulsion.cpp:93-176)
# --------------------------------------------------------------------------
def repulsion(numbers, pos, grad=None):
    p = PR.load()
    g = p["g"]
    z = numbers - 1
    sa = np.sqrt(p["gfn2_arep"][z])
    ze = p["gfn2_zeff"][z]
    light = numbers <= 2
    e = 0.0
    for i in range(len(numbers)):
        for j in range(i):
            d = pos[i] - pos[j]
            r2 = d @ d
            if r2 > 25.0 ** 2:
                continue
            r = math.sqrt(r2)
            lp = light[i] and light[j]
            k = g["rep_klight"] if lp else g["rep_kexp"]
            rp = r if lp else r * math.sqrt(r)
            pa = sa[i] * sa[j]
            pe = ze[i] * ze[j] * math.exp(-pa * rp) / r
            e += pe
            if grad is not None:
                fs = (pa * k * rp + 1.0) * pe / r2
                grad[i] -= fs * d
                grad[j] += fs * d
    return e


# --------------------------------------------------------------------------
# Occupations (model/gfn2/eigensolver.cpp:1026-1219)
# --------------------------------------------------------------------------
def fermi(eps, nel, kt):
    """Fermi-Dirac occupations of one spin channel, chemical potential, entropy."""
    n = len(eps)
    if nel <= 0.0:
        return np.zeros(n), 0.0, 0.0
    if nel >= n:
        return np.ones(n), eps[-1] + 50 * kt, 0.0
    holes = nel > 0.5 * n
    ref = eps[-1] if holes else eps[0]
    e = eps - ref
    target = n - nel if holes else nel

    def qty(mu):
        x = (e - mu) / kt
        f = 0.5 * (1.0 - np.tanh(0.5 * x))
        return np.sum(1.0 - f) if holes else np.sum(f)

    margin = max(64.0, -math.log(target / n) + 8.0) * kt + 64 * np.finfo(float).eps * max(1.0, e[-1] - e[0])
    lo, hi = e[0] - margin, e[-1] + margin
    for _ in range(400):
        mid = lo + 0.5 * (hi - lo)
        qv = qty(mid)
        if mid == lo or mid == hi:
            break
        if (not holes and qv < target) or (holes and qv > target):
            lo = mid
        else:
            hi = mid
    mu = lo + 0.5 * (hi - lo)
    x = (e - mu) / kt
    f = 0.5 * (1.0 - np.tanh(0.5 * x))
    fm = f[(f > 0) & (f < 1)]
    s = -np.sum(fm * np.log(fm) + (1 - fm) * np.log(1 - fm))
    return f, ref + mu, s


# --------------------------------------------------------------------------
# Broyden mixer (common/scc_mixer.cpp:559-740)
# --------------------------------------------------------------------------
class Broyden:
    def __init__(self, x0, memory=8, damping=0.4):
        self.cur = np.array(x0, float)
        self.prev = np.zeros_like(self.cur)
        self.prev_res = np.zeros_like(self.cur)
        self.memory = memory
        self.damp = damping
        self.it = 0
        self.df = {}
        self.u = {}
        self.om = {}

    def step(self, raw):
        res = raw - self.cur
        nrm = math.sqrt(res @ res)
        rms = nrm / math.sqrt(len(res))
        it_new = self.it + 1
        if it_new == 1:
            mixed = self.cur + self.damp * res
        else:
            df = res - self.prev_res
            inv = 1.0 / max(math.sqrt(df @ df), np.finfo(float).eps)
            df = df * inv
            u = self.damp * df + inv * (self.cur - self.prev)
            om = max(1.0, 0.01 / nrm) if nrm > 0.01 / 100000.0 else 100000.0
            hc = min(self.memory, self.it)
            first = self.it - hc + 1
            new_slot = (self.it - 1) % self.memory
            slots = [(first + h - 1) % self.memory for h in range(hc)]
            dfs = {k: (df if k == new_slot else self.df[k]) for k in slots}
            us = {k: (u if k == new_slot else self.u[k]) for k in slots}
            oms = {k: (om if k == new_slot else self.om[k]) for k in slots}
            c = np.array([oms[k] * (dfs[k] @ res) for k in slots])
            B = np.array([[oms[a] * oms[b] * (dfs[a] @ dfs[b]) + (1e-4 if a == b else 0.0)
                           for b in slots] for a in slots])
            c = np.linalg.solve(B, c)
            mixed = self.cur + self.damp * res
            for h, k in enumerate(slots):
                mixed = mixed - oms[k] * c[h] * us[k]
            self.df[new_slot], self.u[new_slot], self.om[new_slot] = df, u, om
        self.prev = self.cur.copy()
        self.prev_res = res
        self.cur = mixed
        self.it = it_new
        return mixed, rms


# --------------------------------------------------------------------------
# Single point (runtime/gfn2_cpu_execution.cpp:1218-1460, model/gfn2/scc_driver.cpp:706-960,
# 2105-2560, model/gfn2/force.cpp:336-645)
# --------------------------------------------------------------------------
def pc_setup(basis, pos, pc_pos, pc_gam):
    """Softened shell-point Coulomb kernel K[s, p] = (|R_A - R_p|^2 + a_sp^2)^-1/2 with
    a_sp = 2 / (eta_s + gamma_p), eta_s the GFN2 shell hardness
    (model/gfn2/external_point_charges.cpp:277-327, docs/theory/qmmm.md)."""
    eta = shell_hardness(basis)
    d = pos[basis.sh_atom][:, None, :] - pc_pos[None, :, :]
    a = 2.0 / (eta[:, None] + pc_gam[None, :])
    D = np.sum(d * d, axis=-1) + a * a
    return 1.0 / np.sqrt(D), d, D


def pc_gradients(basis, qsh, pc_q, K, d, D, grad):
    """Adds dE_pc/dR_A to grad; returns dE_pc/dR_p and dE_pc/dQ_p
    (external_point_charges.cpp:389-490; dE/dQ_p = sum_s q_s K_sp)."""
    w = qsh[:, None] * pc_q[None, :] * D ** -1.5
    f = w[:, :, None] * d
    np.add.at(grad, basis.sh_atom, -f.sum(axis=1))
    return f.sum(axis=0), qsh @ K


@dataclass
class Result:
    energy: float
    gradient: np.ndarray
    charges: np.ndarray
    iterations: int
    converged: bool
    terms: dict = field(default_factory=dict)
    debug: dict = field(default_factory=dict)
    pc_gradient: np.ndarray | None = None
    pc_dq: np.ndarray | None = None


def singlepoint(numbers, pos, charge=0.0, uhf=0, kt=300.0 * PR.KELVIN_TO_HARTREE,
                ctol=1e-6, etol=1e-8, maxiter=250, memory=8, damping=0.4,
                forces=True, debug=False, pc_pos=None, pc_q=None, pc_gam=None) -> Result:
    numbers = np.asarray(numbers, int)
    pos = np.asarray(pos, float).reshape(-1, 3)
    nat = len(numbers)
    basis = make_basis(numbers)
    cn, dcn = cn_dexp(numbers, pos, with_deriv=True)
    S, D, Q = integrals(basis, pos)
    h0p = make_h0(basis)
    H0 = h0_matrix(basis, h0p, pos, cn, S)
    gam = es2_gamma(basis, pos)
    g3 = shell_gamma3(basis)
    aes = aes2_setup(numbers, pos, cn)
    d4 = d4_setup(numbers, pos)
    ao_at, ao_sh = basis.ao_atom, basis.ao_shell
    ns = len(basis.sh_l)
    have_pc = pc_q is not None and len(pc_q) > 0
    if have_pc:
        pc_pos = np.asarray(pc_pos, float).reshape(-1, 3)
        pc_q = np.asarray(pc_q, float)
        pc_gam = np.asarray(pc_gam, float)
        Kpc, dpc, Dpc = pc_setup(basis, pos, pc_pos, pc_gam)
        vpc = Kpc @ pc_q
    else:
        vpc = np.zeros(ns)
    nel = basis.refocc.sum() - charge
    na, nb = 0.5 * (nel + uhf), 0.5 * (nel - uhf)

    # SAD start (model/gfn2/wavefunction.cpp:733-773)
    refat = np.zeros(nat)
    np.add.at(refat, basis.sh_atom, basis.refocc)
    qat0 = np.full(nat, charge / nat)
    qsh = basis.refocc / refat[basis.sh_atom] * qat0[basis.sh_atom]
    dip = np.zeros((nat, 3))
    qp = np.zeros((nat, 6))
    mixer = Broyden(np.concatenate([qsh, dip.ravel(), qp.ravel()]), memory, damping)

    def atom_sum(x):
        out = np.zeros(nat)
        np.add.at(out, basis.sh_atom, x)
        return out

    def potentials(qsh, dip, qp):
        qat = atom_sum(qsh)
        vsh = gam @ qsh + g3 * qsh * qsh
        vat, vd, vq = aes2_potential(aes, qat, dip, qp)
        _, vd4 = d4_two_body(d4, qat)
        vat = vat + vd4
        return vsh + vat[basis.sh_atom] + vpc, vd, vq

    def fock(vs, vd, vq):
        v = vs[ao_sh]
        H = H0 - 0.5 * S * (v[:, None] + v[None, :])
        # D[c][mu][nu] has origin at atom(nu): potential of atom(nu)
        H -= 0.5 * np.einsum("cmn,nc->mn", D, vd[ao_at])
        H -= 0.5 * np.einsum("cnm,mc->mn", D, vd[ao_at])
        H -= 0.5 * np.einsum("cmn,nc->mn", Q, vq[ao_at])
        H -= 0.5 * np.einsum("cnm,mc->mn", Q, vq[ao_at])
        return H

    def populations(P):
        qsh = basis.refocc - np.bincount(ao_sh, weights=np.sum(P * S, axis=0), minlength=ns)
        dp = np.zeros((nat, 3))
        qq = np.zeros((nat, 6))
        for c in range(3):
            dp[:, c] = -np.bincount(ao_at, weights=np.sum(P * D[c], axis=0), minlength=nat)
        for c in range(6):
            qq[:, c] = -np.bincount(ao_at, weights=np.sum(P * Q[c], axis=0), minlength=nat)
        return qsh, dp, qq

    fold = 0.0
    it = 0
    converged = False
    dbg = {}
    while it < maxiter:
        vs, vd, vq = potentials(qsh, dip, qp)
        H = fock(vs, vd, vq)
        if debug and it == 0:
            dbg["H_first"] = H.copy()
        eps, C = eigh(H, S)
        fa, _, sa = fermi(eps, na, kt)
        fb, _, sb = fermi(eps, nb, kt)
        focc = fa + fb
        P = (C * focc) @ C.T
        W = (C * (focc * eps)) @ C.T
        ent = sa + sb
        rqsh, rdip, rqp = populations(P)
        rqat = atom_sum(rqsh)
        e_core = np.sum(H0 * P)
        e_es2 = 0.5 * rqsh @ gam @ rqsh
        e_es3 = np.sum(g3 * rqsh ** 3) / 3.0
        e_aes2 = aes2_energy(aes, rqat, rdip, rqp)
        e_d4, _ = d4_two_body(d4, rqat)
        e_pc = rqsh @ vpc
        free = e_core + e_es2 + e_es3 + e_aes2 + e_d4 + e_pc - kt * ent
        raw = np.concatenate([rqsh, rdip.ravel(), rqp.ravel()])
        mixed, rms = mixer.step(raw)
        de = free - (0.0 if it == 0 else fold)
        it += 1
        fold = free
        if rms < ctol and abs(de) < etol:
            converged = True
            qsh, dip, qp = rqsh, rdip, rqp
            break
        qsh = mixed[:ns]
        dip = mixed[ns:ns + 3 * nat].reshape(nat, 3)
        qp = mixed[ns + 3 * nat:].reshape(nat, 6)

    qat = atom_sum(qsh)
    e_rep = repulsion(numbers, pos)
    e_atm = d4_atm(d4)
    energy = free + e_rep + e_atm
    terms = dict(core=e_core, es2=e_es2, es3=e_es3, aes2=e_aes2, d4=e_d4, entropy=-kt * ent,
                 rep=e_rep, atm=e_atm, pc=e_pc, free=free)
    grad = np.zeros((nat, 3))
    pc_grad = pc_dq = None
    if forces and converged:
        vs, vd, vq = potentials(qsh, dip, qp)
        # electronic part: H0 VJP, -W, stationary S/D/Q adjoints (model/gfn2/force.cpp:256-300,520-560)
        aS = np.zeros_like(S)
        acn = np.zeros(nat)
        h0_vjp(basis, h0p, pos, cn, S, P, aS, acn, grad)
        aS -= W
        v = vs[ao_sh]
        aS += -0.5 * P * (v[:, None] + v[None, :])
        # dE/dD[c][x][y] = -P[x,y] * vd[atom(y)][c]: the operator origin is atom(y)
        aD = -P[None, :, :] * vd[ao_at].T[:, None, :]
        aQ = -P[None, :, :] * vq[ao_at].T[:, None, :]
        integral_vjp(basis, pos, aS, aD, aQ, grad)
        cn_vjp(pos, dcn, acn, grad)
        es2_grad(basis, pos, gam, qsh, grad)
        acn2 = np.zeros(nat)
        aes2_vjp(aes, qat, dip, qp, grad, acn2)
        cn_vjp(pos, dcn, acn2, grad)
        d4_two_body(d4, qat, grad=grad)
        d4_atm(d4, grad=grad)
        repulsion(numbers, pos, grad=grad)
        if have_pc:
            pc_grad, pc_dq = pc_gradients(basis, qsh, pc_q, Kpc, dpc, Dpc, grad)
    if debug:
        dbg.update(cn=cn, S=S, D=D, Q=Q, H0=H0, P=P, W=W, eps=eps, qsh=qsh, dip=dip, qp=qp,
                   gam=gam, cn_d4=d4.cn, nel=nel)
    return Result(energy, grad, qat, it, converged, terms, dbg, pc_grad, pc_dq)
