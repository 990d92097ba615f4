"""GPU edge cases of the operator and solver paths on the smallest meshes: one hexahedron (6 Kuhn
tetrahedra) and one square (2 triangles). P1 has no free DOF there (every vertex is on the boundary),
P2 exactly one (the midpoint of the interior diagonal). Bars as in the other parity tests: FP64
values within 1e-12 of the oracle; solves against the oracle's direct solution."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import assemble as oa  # noqa: E402
from oracle import mesh as om  # noqa: E402
from oracle import pcg as op  # noqa: E402

VAL_TOL = 1e-12


def _single_cell(dim, order):
    if dim == 3:
        return om.kuhn_cube(1, order=order, seed=0)
    return om.unit_square(1, order=order, seed=0)


@pytest.mark.parametrize("dim,order", [(3, 1), (3, 2), (2, 1), (2, 2)])
def test_single_cell_assembly_and_solvers(dim, order):
    from jno_b200.plan import FemPlan

    pf, cf, cells, p1 = _single_cell(dim, order)
    nv = dim + 1
    logk = om.logk_field(len(cells), 1010)
    plan = FemPlan(p1, cells, order)
    bnd = om.boundary_nodes(cf, order, nv=nv)
    assert plan.n - len(bnd) == (0 if order == 1 else 1)
    lk = torch.as_tensor(logk, device="cuda")
    vals, b = plan.assemble(lk)
    s = oa.assemble(pf, cf, order, bnd, np.exp(logk))
    assert np.abs(vals.cpu().numpy() - s.data).max() <= VAL_TOL * np.abs(s.data).max()
    assert np.abs(b.cpu().numpy() - s.b).max() <= VAL_TOL * max(np.abs(s.b).max(), 1e-300)
    inv = plan.jacobi(vals)
    A = s.csr()
    xo, ito, _ = op.pcg(A, s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8)
    u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
    um, inner, outer, relm, stm = plan.pcg_mixed(vals, b, inv, tol=1e-8)
    ub, itb, relb, stb = plan.bicgstab(vals, b, inv_diag=inv, tol=1e-8)
    xb, itbo = op.bicgstab(A, s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8)
    assert st == stm == stb == 0
    assert it == ito and itb == itbo
    if order == 1:
        # all-Dirichlet with g = 0: b = 0, so no iteration and x stays 0 (jax's loop test fails at once)
        assert it == 0 and inner == 0 and itb == 0
        assert torch.all(u == 0) and torch.all(um == 0) and torch.all(ub == 0)
    else:
        # one free DOF: Jacobi-PCG is exact after one step; BiCGStab exits early in its first one
        assert it == 1 and itb == 1
        scale = np.abs(xo).max()
        for sol in (u, ub):
            assert np.abs(sol.cpu().numpy() - xo).max() <= 1e-14 * scale
        assert np.abs(um.cpu().numpy() - xo).max() <= 1e-8 * scale
        assert np.abs(xb - xo).max() <= 1e-14 * scale


@pytest.mark.parametrize("dim,order", [(3, 1), (3, 2), (2, 1), (2, 2)])
def test_single_cell_inhomogeneous_dirichlet(dim, order):
    """Dirichlet data on every boundary DOF: the solve returns g there, and for g linear (P1) or
    quadratic (P2, with the matching constant source) the exact field at the interior DOF."""
    from jno_b200.plan import FemPlan

    pf, cf, cells, p1 = _single_cell(dim, order)
    nv = dim + 1
    xs = pf.T
    if order == 1:
        exact = 1.0 + sum((i + 2.0) * xs[i] for i in range(dim))
        f = 0.0
    else:
        exact = 0.5 + sum((i + 1.0) * xs[i] ** 2 for i in range(dim))
        f = -2.0 * sum(i + 1.0 for i in range(dim))  # -lap(exact)
    plan = FemPlan(p1, cells, order)
    g = torch.as_tensor(exact, device="cuda")
    vals, b = plan.assemble(None, mode=2, scale=1.0, f=f, g=g)
    bnd = om.boundary_nodes(cf, order, nv=nv)
    s = oa.assemble(pf, cf, order, bnd, np.ones(len(cells)), f=f, g=exact)
    assert np.abs(vals.cpu().numpy() - s.data).max() <= VAL_TOL * np.abs(s.data).max()
    assert np.abs(b.cpu().numpy() - s.b).max() <= 1e-11 * np.abs(s.b).max()
    inv = plan.jacobi(vals)
    u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-13)
    ub, itb, relb, stb = plan.bicgstab(vals, b, inv_diag=inv, tol=1e-13)
    assert st == 0 and stb == 0
    for sol in (u, ub):
        assert np.abs(sol.cpu().numpy() - exact).max() <= 1e-12 * np.abs(exact).max()
