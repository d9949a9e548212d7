"""Fixed-topology plans and asynchronous requests through the C ABI.

Plans (reference docs/developer-guide/architecture.md "Fixed-topology plans",
src/api.cpp:636-770): a plan binds the immutable topology and the compute
policy; a batch whose topology or policy differs is refused before any
output is touched; the plan owns its execution cache, reports the bytes it
keeps, and a plan compute of the bound topology allocates nothing.

Requests (src/api.cpp:330,375, src/runtime/request.cpp): enqueue returns once
the submission is accepted, with the request PENDING; a second submission on a
pending request is refused; wait blocks until COMPLETE, and the outputs equal
those of the synchronous call.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from xtbloom_b200 import abi
from xtbloom_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def batch_of(idx, seed=1):
    return W.subset(W.config1(4096, seed=seed), idx)


def moved(b, scale=0.01, seed=5):
    """The same topology with displaced positions."""
    rng = np.random.default_rng(seed)
    out = W.subset(b, np.arange(b.batch_size))
    out.positions = np.ascontiguousarray(b.positions + scale * rng.standard_normal(b.positions.shape))
    return out


def info_of(lib):
    info = abi.RequestInfo()
    lib.lib.xtbloom_request_info_init(C.byref(info), C.sizeof(info))
    return info


def same(a, b):
    for k in ("per_system_status", "scc_iterations", "energies", "atomic_charges"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    assert np.nanmax(np.abs(a["forces"] - b["forces"])) < 1e-12


def test_plan_matches_compute_and_refuses_other_topologies(cuda_lib):
    b = batch_of(np.arange(0, 4096, 97))
    plan = abi.Plan(cuda_lib, b)
    try:
        b2 = moved(b)
        out = plan.compute(b2)
        ref = cuda_lib.compute(b2)
        same(out, ref)
        # other elements: refused, outputs untouched
        bad = moved(b)
        bad.atomic_numbers = bad.atomic_numbers.copy()
        bad.atomic_numbers[0] = 7 if bad.atomic_numbers[0] != 7 else 8
        sentinel = abi.host_outputs(bad, fill=123.0)
        with pytest.raises(abi.XtbloomError) as e:
            plan.compute(bad, sentinel)
        assert "topology" in str(e.value)
        assert (sentinel["energies"] == 123.0).all() and (sentinel["per_system_status"] == -7).all()
        # another charge
        bad = moved(b)
        bad.molecular_charges = bad.molecular_charges + np.eye(1, b.batch_size, 3).ravel()
        with pytest.raises(abi.XtbloomError):
            plan.compute(bad)
        # another policy
        with pytest.raises(abi.XtbloomError) as e:
            plan.compute(b2, options=cuda_lib.make_options(ctol=1e-5))
        assert "policy" in str(e.value)
    finally:
        plan.close()


def test_plan_reports_its_workspace_and_allocates_nothing_per_compute(cuda_lib):
    b = batch_of(np.arange(0, 4096, 37))
    plan = abi.Plan(cuda_lib, b)
    try:
        q = plan.workspace()
        n_ao = np.array([int(np.sum(np.where(W.molecule(b, i)[0] == 1, 1, 4)))
                         for i in range(b.batch_size)])
        mats = int(np.sum(n_ao.astype(np.int64) ** 2)) * 8
        # about twenty packed n x n FP64 matrices per system
        assert q.device_required_bytes > 10 * mats
        assert q.device_required_alignment >= 256 and q.host_required_bytes > 0
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        outs = [plan.compute(moved(b, seed=s)) for s in (11, 12)]
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(0)[0] == free0
        assert plan.workspace().device_required_bytes == q.device_required_bytes
        assert all((o["per_system_status"] == 0).all() for o in outs)
        # a wrong flag set in the query is refused
        q2 = abi.WorkspaceQuery()
        cuda_lib.lib.xtbloom_workspace_query_init(C.byref(q2), C.sizeof(q2))
        q2.compute_flags = abi.COMPUTE_ENERGY
        assert cuda_lib.lib.xtbloom_plan_query_workspace(plan.handle, C.byref(q2)) == abi.INVALID_ARGUMENT
    finally:
        plan.close()


def test_enqueue_returns_pending_and_completes(cuda_lib):
    b = batch_of(np.arange(0, 4096, 8))   # 512 systems: the call takes far longer than admission
    lib = cuda_lib.lib
    req = C.c_void_p()
    assert lib.xtbloom_request_create(cuda_lib.ctx, C.byref(req)) == 0
    try:
        outs = abi.host_outputs(b)
        batch = cuda_lib.make_batch(b)
        opts = cuda_lib.make_options()
        res = cuda_lib.make_result(outs)
        assert lib.xtbloom_compute_enqueue(cuda_lib.ctx, C.byref(batch), C.byref(opts), C.byref(res), req) == 0
        info = info_of(cuda_lib)
        assert lib.xtbloom_request_query(req, C.byref(info)) == 0
        assert info.state == abi.REQUEST_PENDING
        # a second submission on a pending request is refused and changes nothing
        other = abi.host_outputs(b, fill=5.0)
        res2 = cuda_lib.make_result(other)
        assert lib.xtbloom_compute_enqueue(cuda_lib.ctx, C.byref(batch), C.byref(opts), C.byref(res2),
                                           req) == abi.INVALID_ARGUMENT
        assert b"pending" in lib.xtbloom_get_last_error()
        assert lib.xtbloom_request_wait(req, C.byref(info)) == 0
        assert info.state == abi.REQUEST_COMPLETE and info.completion_status == 0
        assert (other["energies"] == 5.0).all()
        same(outs, cuda_lib.compute(b))
        # the request is reusable: a plan submission on it
        plan = abi.Plan(cuda_lib, b)
        try:
            b2 = moved(b)
            outs2 = abi.host_outputs(b2)
            batch2 = cuda_lib.make_batch(b2)
            res3 = cuda_lib.make_result(outs2)
            assert lib.xtbloom_plan_compute_enqueue(plan.handle, C.byref(batch2), C.byref(opts),
                                                    C.byref(res3), req) == 0
            assert lib.xtbloom_request_wait(req, C.byref(info)) == 0
            assert info.state == abi.REQUEST_COMPLETE and info.completion_status == 0
            same(outs2, cuda_lib.compute(b2))
        finally:
            plan.close()
    finally:
        lib.xtbloom_request_destroy(req)


def test_enqueue_rejects_invalid_descriptors_before_admission(cuda_lib):
    b = batch_of([3, 5])
    lib = cuda_lib.lib
    req = C.c_void_p()
    assert lib.xtbloom_request_create(cuda_lib.ctx, C.byref(req)) == 0
    try:
        outs = abi.host_outputs(b)
        batch = cuda_lib.make_batch(b)
        batch.total_atoms = batch.total_atoms + 1   # atom offsets no longer end at total_atoms
        res = cuda_lib.make_result(outs)
        st = lib.xtbloom_compute_enqueue(cuda_lib.ctx, C.byref(batch), C.byref(cuda_lib.make_options()),
                                         C.byref(res), req)
        assert st != 0
        info = info_of(cuda_lib)
        assert lib.xtbloom_request_query(req, C.byref(info)) == 0
        assert info.state in (abi.REQUEST_IDLE, abi.REQUEST_COMPLETE)
        if info.state == abi.REQUEST_COMPLETE:
            assert info.completion_status != 0
    finally:
        lib.xtbloom_request_destroy(req)
