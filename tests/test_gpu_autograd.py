"""Gradients through the drop-in surface: ``fem.operator.evaluate({name: theta})`` -> (A, b) ->
a solve -> loss, differentiated by torch autograd on the device kernels (``femk_assemble_vjp``,
``femk_adjoint_grad`` and the adjoint solves), against finite differences and the oracle's adjoint.

The first test ports the reference's inverse-problem check (tests/test_fem_native_lagrange.py:
688-711: ``loss(a) = sum(solve(A(a).todense(), b(a))^2)``, ``jax.grad`` against a central difference,
``|g_ad - g_fd| <= 1e-5 max(1, |g_fd|)``) onto a structured triangle mesh with a constant source
(the reference uses a gmsh disc-free box with a polynomial source; meshing and spatially varying
sources are outside this path)."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import adjoint as oadj  # noqa: E402
from oracle import assemble as oa  # noqa: E402
from oracle import element as oe  # noqa: E402
from oracle import mesh as om  # noqa: E402


def _scalar_poisson(dim=2, n=8, g_boundary=None):
    import jno_b200 as jno

    ctor = jno.domain.equi_distant_rect(nx=n, ny=n) if dim == 2 else jno.domain.equi_distant_box(nx=n, ny=n, nz=n)
    d = jno.domain(ctor)
    u, phi = d.fem_symbols()
    coords = d.variable("interior", split=True)
    bcoords = d.variable("boundary", split=True)
    alpha = jno.np.parameter((1,), name="alpha")
    ui, vi = u.bind(x=coords[0], y=coords[1]), phi.bind(x=coords[0], y=coords[1])
    grad = ui.x * vi.x + ui.y * vi.y + (ui.z * vi.z if dim == 3 else 0.0)
    g = 0.0 if g_boundary is None else g_boundary(bcoords)
    return jno, jno.fem([alpha * grad - 2.0 * vi, u(*bcoords[:dim]) - g], quad_degree=2)


def test_inverse_recipe_dense_solve_matches_finite_difference():
    jno, fem = _scalar_poisson()
    sys = fem.operator
    assert sys.is_parametric and list(sys.runtime_parameter_exprs) == ["alpha"]

    def loss(a):
        A, b = sys.evaluate({"alpha": a})
        u = torch.linalg.solve(A.todense(), b.reshape(-1))
        return torch.sum(u**2)

    a0 = torch.tensor([1.3], dtype=torch.float64, device="cuda", requires_grad=True)
    (g_ad,) = torch.autograd.grad(loss(a0), a0)
    g_ad = float(g_ad)
    eps = 1e-6
    with torch.no_grad():
        ap = torch.tensor([1.3 + eps], dtype=torch.float64, device="cuda")
        am = torch.tensor([1.3 - eps], dtype=torch.float64, device="cuda")
        g_fd = float((loss(ap) - loss(am)) / (2 * eps))
    assert abs(g_ad) > 1e-8
    assert abs(g_ad - g_fd) <= 1e-5 * max(1.0, abs(g_fd))


@pytest.mark.parametrize("solver", ["cg", "mixed", "bicgstab"])
def test_inverse_recipe_through_the_b200_solvers(solver):
    """The same loss with ``jno.solve.*(A, b)`` in place of the dense solve: the adjoint (one more
    solve + the element contraction) gives the dense path's gradient."""
    jno, fem = _scalar_poisson()
    sys = fem.operator
    make = {"cg": lambda: jno.solve.cg(tol=1e-12), "mixed": lambda: jno.solve.cg(tol=1e-12, precision="mixed"),
            "bicgstab": lambda: jno.solve.bicgstab(tol=1e-12)}[solver]

    def loss(a, dense):
        A, b = sys.evaluate({"alpha": a})
        u = torch.linalg.solve(A.todense(), b) if dense else make()(A, b, M=jno.precond.jacobi())
        return torch.sum(u**2)

    grads = []
    for dense in (True, False):
        a0 = torch.tensor([1.3], dtype=torch.float64, device="cuda", requires_grad=True)
        (g,) = torch.autograd.grad(loss(a0, dense), a0)
        grads.append(float(g))
    assert abs(grads[1] - grads[0]) <= 1e-8 * abs(grads[0])


def test_assembly_vjp_matches_restatement():
    """femk_assemble_vjp against numpy on the oracle's element matrices and slot map: P0 exp
    coefficient, random cotangents of the values and the load, inhomogeneous Dirichlet data."""
    from jno_b200.plan import FemPlan

    for order in (1, 2):
        pf, cf, tets, p1 = om.kuhn_cube(3, order=order, seed=1)
        plan = FemPlan(p1, tets, order)
        rng = np.random.default_rng(5)
        lk = rng.normal(0, 0.5, len(tets))
        gv = rng.standard_normal(plan.nnz)
        gb = rng.standard_normal(plan.n)
        g = np.sin(pf[:, 0]) + pf[:, 1]
        out = plan.assemble_vjp(torch.as_tensor(lk, device="cuda"), torch.as_tensor(gv, device="cuda"),
                                torch.as_tensor(gb, device="cuda"), 0, 1.0,
                                torch.as_tensor(g, device="cuda")).cpu().numpy()
        _, inverse, _ = oa.compress_plan(cf)
        K, _ = oe.element_matrices(p1[tets], order)
        nd = cf.shape[1]
        free = np.ones(pf.shape[0], bool)
        free[om.boundary_nodes(cf, order)] = False
        fa = free[cf][:, :, None]
        fb = free[cf][:, None, :]
        S = np.sum(np.where(fa & fb, gv[inverse.reshape(-1, nd, nd)] * K, 0.0), axis=(1, 2))
        S -= np.sum(np.where(fa & ~fb, gb[cf][:, :, None] * K * g[cf][:, None, :], 0.0), axis=(1, 2))
        ref = np.exp(lk) * S
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


def _p0_system(n=6):
    import jno_b200 as jno

    pf, cf, tets, p1 = om.kuhn_cube(n, order=1, seed=0)
    d = jno.domain.from_mesh(p1, tets)
    u, v = d.fem_symbols()
    _r, s = d.fem_symbols(space="P0", names=("r", "s"))
    xi, yi, zi = d.variable("interior")
    xb, yb, zb = d.variable("boundary")
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    logk = jno.np.parameter(s, name="logk")
    fem = jno.fem([jno.np.exp(logk) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi, u(xb, yb, zb) - 0.0])
    return jno, fem, pf, cf, tets


def test_p0_gradient_through_the_surface_matches_the_oracle_adjoint():
    """dJ/dlogk of the misfit J = 1/2 sum M_ii (u_i - u*_i)^2 with u = jno.solve.cg(A, b) through
    ``evaluate``: the fused parameter path (femk_adjoint_grad), the values path (a copy of A.data,
    so the backward runs femk_assemble_vjp) and the oracle's adjoint agree to 1e-8 of max |g|."""
    jno, fem, pf, cf, tets = _p0_system()
    sys = fem.operator
    lk0 = om.logk_field(len(tets), 1002)
    bnd = om.boundary_nodes(cf, 1)
    ustar, _, _ = oadj.solve(pf, cf, 1, bnd, om.logk_field(len(tets), 2000))
    mass = oadj.lumped_mass(pf, cf, 1)
    _, g_o = oadj.gradient(pf, cf, 1, bnd, lk0, ustar, mass)
    us, m = torch.as_tensor(ustar, device="cuda"), torch.as_tensor(mass, device="cuda")
    from jno_b200.sparse import CsrMatrix

    for copy in (False, True):
        lk = torch.as_tensor(lk0, device="cuda").requires_grad_(True)
        A, b = sys.evaluate({"logk": lk})
        if copy:
            A = CsrMatrix(A.plan, A.data * 1.0)
        u = jno.solve.cg(tol=1e-13)(A, b, M=jno.precond.jacobi())
        J = 0.5 * torch.sum(m * (u - us) ** 2)
        (g,) = torch.autograd.grad(J, lk)
        assert np.abs(g.cpu().numpy() - g_o).max() <= 1e-8 * np.abs(g_o).max(), copy


def test_fem_solve_call_is_differentiable():
    """``FemLinearSystem.solve(solve_fn)`` returns a callable of the parameter value whose result
    carries the gradient (the default solve_fn, and a caller's dense one)."""
    jno, fem, pf, cf, tets = _p0_system(4)
    sys = fem.operator
    lk0 = torch.as_tensor(om.logk_field(len(tets), 1003), device="cuda")
    w = torch.as_tensor(np.random.default_rng(2).standard_normal(fem.dofs), device="cuda")
    grads = []
    for call in (sys.solve(), sys.solve(lambda A, b: torch.linalg.solve(A.todense(), b))):
        assert call.params == ["logk"]
        lk = lk0.clone().requires_grad_(True)
        u = call(lk)
        assert torch.equal(u.detach(), call({"logk": lk0}).detach()) or torch.allclose(u, call({"logk": lk0}),
                                                                                        rtol=0, atol=1e-12)
        (g,) = torch.autograd.grad(torch.dot(w, u), lk)
        grads.append(g)
    assert torch.linalg.norm(grads[0] - grads[1]) <= 1e-7 * torch.linalg.norm(grads[1])
    with pytest.raises(NotImplementedError):
        sys.solve(periodic={})


def test_gradient_through_the_dirichlet_lift():
    """With u = g != 0 on the boundary the load depends on the coefficient (b -= A e g): the
    gradient through cg, through the dense solve, and a central difference of a scalar parameter agree."""
    jno, fem = _scalar_poisson(dim=3, n=4, g_boundary=lambda c: 1.0 + c[0] + 0.5 * c[2])
    sys = fem.operator

    def loss(a, how):
        A, b = sys.evaluate({"alpha": a})
        if how == "dense":
            u = torch.linalg.solve(A.todense(), b)
        else:
            u = jno.solve.cg(tol=1e-13)(A, b, M=jno.precond.jacobi())
        return torch.sum(torch.sin(u))

    gs = {}
    for how in ("dense", "cg"):
        a0 = torch.tensor([0.7], dtype=torch.float64, device="cuda", requires_grad=True)
        (g,) = torch.autograd.grad(loss(a0, how), a0)
        gs[how] = float(g)
    eps = 1e-6
    with torch.no_grad():
        ap = torch.tensor([0.7 + eps], dtype=torch.float64, device="cuda")
        am = torch.tensor([0.7 - eps], dtype=torch.float64, device="cuda")
        fd = float((loss(ap, "dense") - loss(am, "dense")) / (2 * eps))
    assert abs(gs["dense"]) > 1e-6
    assert abs(gs["cg"] - gs["dense"]) <= 1e-8 * abs(gs["dense"])
    assert abs(gs["dense"] - fd) <= 1e-6 * max(1.0, abs(fd))


def test_nodal_parameter_gradient_through_the_surface():
    import jno_b200 as jno

    pf, cf, tets, p1 = om.kuhn_cube(5, order=1, seed=0)
    d = jno.domain.from_mesh(p1, tets)
    u, v = d.fem_symbols()
    xi, yi, zi = d.variable("interior")
    xb, yb, zb = d.variable("boundary")
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    kfield = jno.np.parameter(u, name="k")
    fem = jno.fem([jno.np.exp(kfield) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi, u(xb, yb, zb) - 0.0])
    sys = fem.operator
    rng = np.random.default_rng(4)
    p0 = rng.normal(0, 0.3, pf.shape[0])
    bnd = om.boundary_nodes(cf, 1)
    mass = oadj.lumped_mass(pf, cf, 1)
    ustar = rng.normal(0, 0.01, pf.shape[0])
    _, g_o = oadj.gradient_nodal(pf, cf, bnd, p0, "exp", ustar, mass)
    p = torch.as_tensor(p0, device="cuda").requires_grad_(True)
    A, b = sys.evaluate({"k": p})
    uu = jno.solve.cg(tol=1e-13)(A, b, M=jno.precond.jacobi())
    J = 0.5 * torch.sum(torch.as_tensor(mass, device="cuda") * (uu - torch.as_tensor(ustar, device="cuda")) ** 2)
    (g,) = torch.autograd.grad(J, p)
    assert np.abs(g.cpu().numpy() - g_o).max() <= 1e-8 * np.abs(g_o).max()
