"""The bounds-checked build (libfemk_bounds.so: every checked index records FEMK_EBOUNDS and skips the
access instead of faulting) runs the path's parity checks in a separate process that binds it in
place of libfemk.so: plan, assembly, Jacobi-PCG and the mixed solver against the oracle on small P1
and P2 meshes, and no check fires on a valid plan."""

import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

SCRIPT = textwrap.dedent("""
    import numpy as np, torch
    from jno_b200 import _build, _lib
    _lib.LIB_PATH = _build.LIB_BOUNDS
    lib = _lib.load()
    assert lib.femk_bounds_checked() == 1
    from jno_b200.plan import FemPlan
    from oracle import assemble as oa, mesh as om, pcg as op
    for order, n in ((1, 6), (2, 3)):
        pf, cf, tets, p1 = om.kuhn_cube(n, order=order, seed=0)
        logk = om.logk_field(len(tets), 1000)
        plan = FemPlan(p1, tets, order)
        vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
        s = oa.assemble(pf, cf, order, om.boundary_nodes(cf, order), np.exp(logk))
        assert np.abs(vals.cpu().numpy() - s.data).max() <= 1e-12 * np.abs(s.data).max()
        inv = plan.jacobi(vals)
        x, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
        xo, ito, _ = op.pcg(s.csr(), s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8)
        assert st == 0 and abs(it - ito) <= 1 and np.linalg.norm(x.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)
        xm, inner, outer, relm, stm = plan.pcg_mixed(vals, b, inv, tol=1e-8)
        assert stm == 0 and relm <= 1e-8
        y = plan.spmv(vals, x)
        assert torch.linalg.norm(y - b) <= 2e-8 * torch.linalg.norm(b)
    print("bounds-checked build ok")
""")


def test_bounds_checked_build_parity():
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    out = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    assert "bounds-checked build ok" in out.stdout
