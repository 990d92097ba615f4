"""CPU tests: the C-ABI library loads and exports every declared symbol; host-side logic of the
jno-shaped surface (form classification, argument checks). No kernel is launched."""

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _declared():
    src = open(os.path.join(ROOT, "include", "femk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(femk_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from jno_b200 import _lib

    lib = _lib.load()
    names = _declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.femk_version() >= 10000
    assert isinstance(lib.femk_last_error_string(), bytes)


def test_bounds_checked_library_exports_the_same_symbols():
    """libfemk_bounds.so (the -DFEMK_BOUNDS_CHECK build of the same sources) exports every declared
    entry point and reports itself as bounds-checked; the product library reports 0."""
    from jno_b200 import _build, _lib

    assert os.path.exists(_build.LIB_BOUNDS), "build it with python -m jno_b200._build --bounds"
    lib = ctypes.CDLL(_build.LIB_BOUNDS)
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.femk_bounds_checked() == 1
    assert _lib.load().femk_bounds_checked() == 0


def test_null_arguments_are_rejected_without_a_gpu():
    from jno_b200 import _lib

    lib = _lib.load()
    out = ctypes.c_void_p()
    st = lib.femk_plan_create(None, 8, None, 1, 1, None, None, ctypes.byref(out))
    assert st == _lib.FEMK_EINVAL
    assert b"NULL" in lib.femk_last_error_string()
    st = lib.femk_plan_create(None, 8, None, 1, 3, None, None, ctypes.byref(out))
    assert st == _lib.FEMK_EINVAL
    assert lib.femk_assemble(None, None, 0, 1.0, 1.0, None, None, None, None) == _lib.FEMK_EINVAL
    assert lib.femk_pcg(None, None, None, None, None, 1e-8, 0.0, 10, None, None, None) == _lib.FEMK_EINVAL
    assert lib.femk_plan_destroy(None) == _lib.FEMK_OK


def test_plan_options_defaults_and_validation_without_a_gpu():
    """femk_plan_options_default fills the documented defaults; femk_plan_create_ex rejects an unknown
    value before touching a device (the pointers are never dereferenced on that path)."""
    from jno_b200 import _lib

    lib = _lib.load()
    o = _lib.PlanOptions()
    lib.femk_plan_options_default(ctypes.byref(o))
    assert o.size == ctypes.sizeof(_lib.PlanOptions)
    assert (o.solver_layout, o.column_tables, o.cols16, o.graph_replay, o.split_updates) == (1, 1, 1, 1, 1)
    assert (o.l2_hints, o.ring64, o.ring32, o.sell_batch, o.test_skip_arrival) == (-1, -1, -1, 16, -1)
    assert o.mixed_delta2 == 0.0 and o.barrier_limit_ms == 0.0
    fake = ctypes.c_void_p(16)
    for field, bad in (("ring64", 13), ("sell_batch", 4), ("l2_hints", 7), ("solver_layout", 2),
                       ("barrier_limit_ms", -1.0), ("mixed_delta2", 1.5), ("csr_lanes", 3), ("size", 8)):
        b = _lib.PlanOptions()
        lib.femk_plan_options_default(ctypes.byref(b))
        setattr(b, field, bad)
        out = ctypes.c_void_p()
        st = lib.femk_plan_create_ex(fake, 3, 8, fake, 1, 1, None, ctypes.byref(b), None, ctypes.byref(out))
        assert st == _lib.FEMK_EINVAL and out.value is None, field
        assert b"femk_plan_create_ex" in lib.femk_last_error_string()


def _recipe():
    import jno_b200 as jno

    d = jno.domain(jno.domain.equi_distant_box(nx=2, ny=2, nz=2))
    u, v = d.fem_symbols()
    _r, s = d.fem_symbols(space="P0", names=("r", "s"))
    xi, yi, zi = d.variable("interior", split=True)
    xb, yb, zb = d.variable("boundary", split=True)
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    return jno, d, u, v, s, ui, vi, (xb, yb, zb)


def test_form_classification():
    from jno_b200 import _lib
    from jno_b200.trace import classify_dirichlet, classify_volume, evaluate_on

    jno, d, u, v, s, ui, vi, xb = _recipe()
    logk = jno.np.parameter(s, name="logk")
    f = classify_volume(jno.np.exp(logk) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi)
    assert (f.mode, f.scale, f.param, f.f, f.order) == (_lib.COEF_EXP, 1.0, "logk", 1.0, 1)
    f = classify_volume(2.0 * logk * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) + 3.0 * vi)
    assert (f.mode, f.scale, f.f) == (_lib.COEF_LINEAR, 2.0, -3.0)
    f = classify_volume(ui.x * vi.x + ui.y * vi.y + ui.z * vi.z)
    assert (f.mode, f.f) == (_lib.COEF_CONST, 0.0)
    sym, g = classify_dirichlet(u(*xb) - (1.0 + 2.0 * xb[0]))
    pts = np.array([[0.5, 0.0, 0.0], [1.0, 1.0, 1.0]])
    assert np.allclose(evaluate_on(g, pts), [2.0, 3.0])
    with pytest.raises(NotImplementedError):
        classify_volume(ui.x * vi.y + ui.y * vi.x + ui.z * vi.z)
    with pytest.raises(NotImplementedError):
        classify_volume(ui.x * vi.x + ui.y * vi.y)
    with pytest.raises(NotImplementedError):
        classify_volume(logk * (ui.x * vi.x) + ui.y * vi.y + ui.z * vi.z)
    # a P1 symbol gives a nodal parameter (models.py:85-117); P2 symbols are refused like the reference
    k = jno.np.parameter(u, name="nodal")
    f = classify_volume(jno.np.exp(k) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi)
    assert (f.mode, f.param) == (_lib.COEF_NODAL_EXP, "nodal")
    f = classify_volume(k * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z))
    assert f.mode == _lib.COEF_NODAL_LINEAR
    u2, _ = d.fem_symbols(order=2)
    with pytest.raises(NotImplementedError):
        jno.np.parameter(u2, name="p2")


def test_product_has_no_cpu_fallback():
    """Without a CUDA device the product refuses to run instead of computing on the CPU."""
    import torch

    from jno_b200.plan import FemPlan

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        FemPlan(np.zeros((4, 3)), np.array([[0, 1, 2, 3]]), 1)


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "jno_b200")
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith((".py", ".cu", ".cuh")):
                src = open(os.path.join(dirpath, fn)).read()
                assert "import oracle" not in src and "from oracle" not in src, fn


def test_batched_workload_is_deterministic():
    from jno_b200.batch import batched_workload

    s1, p1 = batched_workload(count=6, seed=42, lo=2, hi=5)
    s2, p2 = batched_workload(count=6, seed=42, lo=2, hi=5)
    assert np.array_equal(s1, s2) and s1.min() >= 2 and s1.max() <= 5
    for (a, b_, c), (d, e, f) in zip(p1, p2):
        assert np.array_equal(a, d) and np.array_equal(b_, e) and np.array_equal(c, f)
        n = int(round((len(b_) / 6) ** (1 / 3)))
        assert len(a) == (n + 1) ** 3
