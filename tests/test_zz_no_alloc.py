"""The allocation-free tridiagonal eigenvector entry point against the existing compute path.

The existing entry point (xtbloom_compute) orthogonalises every system with the
Loewdin matrix X = S^-1/2 built from the overlap's eigenvectors.  Here the
overlap S it used is tridiagonalised on the host (S = Q T Q^T), the static
entry point forms the eigenvectors of T on the GPU, twice in a row into two
buffers, and X rebuilt from them must equal the X of the existing path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import as_molecule
from xtbloom_b200 import abi

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
linalg = pytest.importorskip("scipy.linalg")


def static_entry(lib):
    f = lib.lib.xtbloom_b200_tridiag_eigenvectors_static
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                  C.c_double, C.c_void_p]
    return f


def fetch(lib, name, system=0, cap=1_000_000):
    f = lib.lib.xtbloom_b200_debug_fetch
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_double), C.c_size_t,
                  C.POINTER(C.c_size_t)]
    out = np.zeros(cap)
    cnt = C.c_size_t()
    assert f(lib.ctx, name.encode(), system, out.ctypes.data_as(C.POINTER(C.c_double)), cap,
             C.byref(cnt)) == 0
    return out[:cnt.value].copy()


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda:0")


def ptr(t):
    return C.c_void_p(t.data_ptr())


def test_static_vectors_rebuild_the_existing_loewdin_matrix_twice(cuda_lib, fixtures):
    s = next(x for x in fixtures if x["name"] == "hetero_chain_7")
    z, x, q, u = as_molecule(s)
    b = abi.ragged_from_lists([z], [x], [q], [u])
    out = cuda_lib.compute(b)
    assert out["per_system_status"][0] == 0
    S = fetch(cuda_lib, "overlap")
    X = fetch(cuda_lib, "x")
    n = int(round(np.sqrt(S.size)))
    S, X = S.reshape(n, n), X.reshape(n, n)
    T, Q = linalg.hessenberg(S, calc_q=True)
    d, e = np.diag(T).copy(), np.diag(T, 1).copy()
    w = linalg.eigh_tridiagonal(d, e, eigvals_only=True)
    d_t, e_t, w_t = dev(d), dev(e), dev(w)
    bufs = [torch.full((n * n,), float("nan"), dtype=torch.float64, device="cuda:0") for _ in range(2)]
    f = static_entry(cuda_lib)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for buf in bufs:   # two calls in a row on one stream reuse the same scratch
        assert f(ptr(d_t), ptr(e_t), ptr(w_t), n, n, ptr(buf), 0.0, stream) == abi.SUCCESS
    torch.cuda.synchronize()
    for buf in bufs:
        Z = buf.view(n, n).cpu().numpy()          # row j: eigenvector j of T
        assert np.isfinite(Z).all()
        Tm = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        assert np.abs(Z @ Tm - w[:, None] * Z).max() < 1e-12
        assert np.abs(Z @ Z.T - np.eye(n)).max() < 1e-10
        U = Q @ Z.T
        Xs = (U * w ** -0.5) @ U.T
        assert np.abs(Xs - X).max() < 1e-10
    assert torch.equal(bufs[0], bufs[1])
    # after the first call has looked up the scratch, repeated calls leave the
    # device's free memory unchanged: nothing is allocated per call
    free0 = torch.cuda.mem_get_info(0)[0]
    for buf in bufs:
        assert f(ptr(d_t), ptr(e_t), ptr(w_t), n, n, ptr(buf), 0.0, stream) == abi.SUCCESS
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert torch.equal(bufs[0], bufs[1])
    # a leading subset gives the same leading vectors
    part = torch.full((n * n,), float("nan"), dtype=torch.float64, device="cuda:0")
    m = n // 2
    assert f(ptr(d_t), ptr(e_t), ptr(w_t), n, m, ptr(part), 0.0, stream) == abi.SUCCESS
    torch.cuda.synchronize()
    assert torch.allclose(part[:m * n], bufs[0][:m * n], rtol=0, atol=1e-12)
    assert torch.isnan(part[m * n:]).all()


def test_static_rejects_sizes_beyond_the_scratch_and_writes_nothing(cuda_lib):
    f = static_entry(cuda_lib)
    n = 257
    d_t, e_t, w_t = dev(np.arange(n, dtype=float)), dev(np.zeros(n - 1)), dev(np.arange(n, dtype=float))
    out = torch.full((n * n,), 7.0, dtype=torch.float64, device="cuda:0")
    st = f(ptr(d_t), ptr(e_t), ptr(w_t), n, n, ptr(out), 0.0, None)
    assert st == abi.INVALID_ARGUMENT
    assert b"256" in cuda_lib.lib.xtbloom_get_last_error()
    assert f(ptr(d_t), ptr(e_t), ptr(w_t), 4, 5, ptr(out), 0.0, None) == abi.INVALID_ARGUMENT
    torch.cuda.synchronize()
    assert (out == 7.0).all()
