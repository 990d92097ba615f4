"""The allocation-free PCG entry point (femk_pcg_noalloc) against femk_pcg, through the C ABI.

femk_pcg_noalloc serves callers that must not allocate device memory while they run (an XLA FFI
handler, a framework whose caching allocator holds nearly all of HBM, a fixed-budget real-time
loop): its workspace is a static device array of at most FEMK_NOALLOC_MAX_N DOFs. This file is
collected last so that a run stopping at the first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NOALLOC_MAX_N = 262144


def _system(n_h, seed_field):
    from jno_b200.plan import FemPlan
    from oracle import mesh as om

    pf, cf, tets, p1 = om.kuhn_cube(n_h, order=1, seed=0)
    plan = FemPlan(p1, tets, 1)
    logk = torch.as_tensor(om.logk_field(len(tets), seed_field), device="cuda")
    vals, b = plan.assemble(logk)
    return plan, vals, b, plan.jacobi(vals)


def _noalloc(plan, vals, b, inv, tol=1e-8, maxiter=20_000):
    from jno_b200 import _lib

    lib = _lib.load()
    x = torch.zeros(plan.n, dtype=torch.float64, device="cuda")
    it = ctypes.c_int32(-1)
    rel = ctypes.c_double(float("nan"))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = lib.femk_pcg_noalloc(plan.handle, _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv), tol, 0.0,
                              maxiter, ctypes.byref(it), ctypes.byref(rel), _lib.stream_handle())
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return st, x, it.value, rel.value, free0 - free1


def test_noalloc_matches_pcg_on_two_calls_in_a_row():
    for seed_field in (1000, 1001):  # second call sees the first call's leftovers in the scratch
        plan, vals, b, inv = _system(24, seed_field)
        st, x, it, rel, grown = _noalloc(plan, vals, b, inv)
        xr, itr, relr, str_ = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
        assert st == 0 and str_ == 0
        assert it == itr
        assert abs(rel - relr) <= 1e-12 and rel <= 2e-8
        assert (torch.linalg.norm(x - xr) / torch.linalg.norm(xr)).item() <= 1e-12
        if seed_field == 1001:
            assert grown == 0  # no device memory taken by the call


def test_noalloc_rejects_systems_above_the_limit():
    from jno_b200 import _lib

    plan, vals, b, inv = _system(64, 1000)  # (64+1)^3 = 274,625 DOFs > FEMK_NOALLOC_MAX_N
    assert plan.n > NOALLOC_MAX_N
    st, x, it, rel, _ = _noalloc(plan, vals, b, inv)
    assert st == _lib.FEMK_EINVAL
    assert b"FEMK_NOALLOC_MAX_N" in _lib.load().femk_last_error_string()
    assert torch.all(x == 0)
