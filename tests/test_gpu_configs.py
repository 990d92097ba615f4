"""Parity at the benchmark configurations (the sizes the bench times, not only toy meshes):

* P1 32^3 Kuhn tets (196,608 tets, 35,937 DOF), interior jitter +-0.1h from seed 0, k = exp(N(0, 0.5^2))
  per tet from seed 1000, u = 0 on the boundary: the plan (CSR pattern, slot map, boundary set,
  diagonal slots) bit-exact against the oracle's compress plan, values and load within 1e-12 of the
  largest entry, Jacobi-PCG iterations within one of the oracle's restated jax cg and the solution
  within 1e-7, the mixed solver to the same stop rule;
* the same at P2 12^3;
* the adjoint configuration at P1 64^3 (1,572,864 tets): dJ/dlogk of J = 1/2 sum M_ii (u_i - u*_i)^2
  (u* from the seed-2000 field) against the oracle's adjoint on every element (1e-8 of max |g|), and
  against central differences on 32 elements (cancellation-free, jno_b200.autograd.central_difference).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import adjoint as oadj  # noqa: E402
from oracle import assemble as oa  # noqa: E402
from oracle import mesh as om  # noqa: E402
from oracle import pcg as op  # noqa: E402


@pytest.mark.parametrize("n,order", [(32, 1), (12, 2)])
def test_benchmark_config_parity(n, order):
    from jno_b200.plan import FemPlan

    pf, cf, tets, p1 = om.kuhn_cube(n, order=order, seed=0)
    logk = om.logk_field(len(tets), 1000)
    plan = FemPlan(p1, tets, order)
    ex = plan.export()
    indptr, indices, slot = oa.csr_pattern_fast(cf, pf.shape[0])
    assert plan.n == pf.shape[0] and plan.nnz == indices.size
    assert np.array_equal(ex["cells"].cpu().numpy(), cf)
    assert np.array_equal(ex["indptr"].cpu().numpy(), indptr)
    assert np.array_equal(ex["indices"].cpu().numpy(), indices)
    assert np.array_equal(ex["slot"].cpu().numpy().reshape(-1), slot)
    bnd = om.boundary_nodes(cf, order)
    assert np.array_equal(np.flatnonzero(ex["dirichlet_mask"].cpu().numpy()), bnd)
    rows = np.repeat(np.arange(plan.n), np.diff(indptr))
    assert np.array_equal(ex["diag_slot"].cpu().numpy(), np.flatnonzero(rows == indices))
    if order == 1:
        assert plan.n == 35_937 and len(tets) == 196_608 and plan.nnz == 513_313
    s = oa.assemble(pf, cf, order, bnd, np.exp(logk), plan=(indptr, indices, slot))
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    v = vals.cpu().numpy()
    assert np.abs(v - s.data).max() <= 1e-12 * np.abs(s.data).max()
    assert np.abs(b.cpu().numpy() - s.b).max() <= 1e-12 * np.abs(s.b).max()
    assert np.array_equal(v == 0.0, s.data == 0.0)
    inv = plan.jacobi(vals)
    A = s.csr()
    inv_o = oa.jacobi_inverse(oa.matrix_diagonal(s))
    u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
    xo, ito, _ = op.pcg(A, s.b, inv_o, tol=1e-8)
    assert st == 0 and abs(it - ito) <= 1, (it, ito)
    assert np.linalg.norm(u.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)
    assert rel <= 1e-8 * (1 + 1e-6) or abs(rel - op.residual_check(A, s.b, u.cpu().numpy())) <= 1e-12
    um, inner, outer, relm, stm = plan.pcg_mixed(vals, b, inv, tol=1e-8)
    assert stm == 0 and relm <= 1e-8
    assert np.linalg.norm(um.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)
    _, ito_m, _ = op.mixed_pcg(A, s.b, inv_o, tol=1e-8)
    assert abs(inner - ito_m) <= 0.1 * ito_m + 3, (inner, ito_m)


def test_adjoint_config_p1_64():
    from jno_b200.autograd import central_difference, solve_p0
    from jno_b200.plan import FemPlan

    n = 64
    pf, cf, tets, p1 = om.kuhn_cube(n, order=1, seed=0)
    plan = FemPlan(p1, tets, 1)
    logk = om.logk_field(len(tets), 1000)
    lk_star = om.logk_field(len(tets), 2000)
    bnd = om.boundary_nodes(cf, 1)
    indptr, indices, slot = oa.csr_pattern_fast(cf, pf.shape[0])
    ustar, _, _ = oadj.solve(pf, cf, 1, bnd, lk_star, tol=1e-12, plan=(indptr, indices, slot))
    mass = oadj.lumped_mass(pf, cf, 1)
    _, g_o = _oracle_gradient(pf, cf, bnd, logk, ustar, mass, (indptr, indices, slot))
    lk = torch.as_tensor(logk, device="cuda").requires_grad_(True)
    u = solve_p0(plan, lk, tol=1e-13)
    J = 0.5 * torch.sum(torch.as_tensor(mass, device="cuda") * (u - torch.as_tensor(ustar, device="cuda")) ** 2)
    (g,) = torch.autograd.grad(J, lk)
    g = g.cpu().numpy()
    gmax = np.abs(g_o).max()
    assert np.abs(g - g_o).max() <= 1e-8 * gmax
    idx = np.random.default_rng(7).choice(len(tets), 32, replace=False)
    fd = central_difference(plan, logk, ustar, mass, idx, eps=1e-6)
    assert np.abs(fd - g[idx]).max() <= 1e-6 * gmax
    big = np.abs(g[idx]) > 1e-3 * gmax
    assert np.all(np.abs(fd - g[idx])[big] <= 1e-6 * np.abs(g[idx])[big])


def _oracle_gradient(pf, cf, bnd, logk, ustar, mass, plan):
    """oracle.adjoint.gradient with the fast pattern (the same restatement; np.unique over 25M keys
    is the slow part of the reference's compress plan at this size)."""
    from oracle import element as oe
    from oracle.assemble import assemble, jacobi_inverse, matrix_diagonal

    element = oe.element_matrices(oe.vertices(pf, cf), 1)
    sysm = assemble(pf, cf, 1, bnd, np.exp(logk), plan=plan, element=element)
    A = sysm.csr()
    inv = jacobi_inverse(matrix_diagonal(sysm))
    u, _, _ = op.pcg(A, sysm.b, inv, tol=1e-13)
    lam, _, _ = op.pcg(A, mass * (u - ustar), inv, tol=1e-13)
    m = (~sysm.dirichlet).astype(np.float64)
    le, ue = (m * lam)[cf], (m * u)[cf]
    grad = -np.exp(logk) * np.einsum("ta,tab,tb->t", le, element[0], ue)
    return oadj.misfit(u, ustar, mass), grad
