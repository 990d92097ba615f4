"""GPU parity of the transient theta step: the consistent mass, the step operators of both
Dirichlet routes and the march, through the C ABI and the jno surface, against the oracle.

Bars: mass and step-operator values within 1e-12 of the oracle relative to the largest entry;
trajectories within 1e-8 of the oracle's (per-step BiCGStab to 1e-10); step residuals below the
reference's 1e-9 check.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import mesh as om  # noqa: E402
from oracle import transient as ot  # noqa: E402

VAL_TOL = 1e-12


def _plan(points, cells, order):
    from jno_b200.plan import FemPlan

    return FemPlan(points, cells, order)


def _mesh(dim, n, order, seed=0):
    if dim == 2:
        pf, cf, cells, p1 = om.unit_square(n, order, seed=seed)
        return pf, cf, cells, p1, om.boundary_nodes(cf, order, nv=3)
    pf, cf, cells, p1 = om.kuhn_cube(n, order, seed=seed)
    return pf, cf, cells, p1, om.boundary_nodes(cf, order)


def _csr_of(plan, vals):
    import scipy.sparse as sp

    ex = plan.export()
    return sp.csr_matrix((vals.cpu().numpy(), ex["indices"].cpu().numpy(), ex["indptr"].cpu().numpy()),
                         shape=(plan.n, plan.n))


CASES = [(2, 12, 1), (2, 6, 2), (3, 4, 1), (3, 3, 2)]


@pytest.mark.parametrize("dim,n,order", CASES)
def test_mass_matrix_matches_oracle(dim, n, order):
    pf, cf, cells, p1, bnd = _mesh(dim, n, order, seed=1)
    plan = _plan(p1, cells, order)
    for zero in (False, True):
        m = _csr_of(plan, plan.mass_matrix(zero_dirichlet=zero)).toarray()
        mo = ot.mass_csr(pf, cf, order, bnd if zero else None).toarray()
        assert np.abs(m - mo).max() <= VAL_TOL * np.abs(mo).max()
    assert abs(_csr_of(plan, plan.mass_matrix()).sum() - 1.0) <= 1e-12


@pytest.mark.parametrize("dim,n,order", CASES)
@pytest.mark.parametrize("rows", [True, False])
def test_step_operators_match_oracle(dim, n, order, rows):
    from jno_b200 import _lib

    pf, cf, cells, p1, bnd = _mesh(dim, n, order, seed=2)
    logk = om.logk_field(len(cells), 11)
    g = 0.5 + pf[:, 0] - 0.25 * pf[:, 1]
    plan = _plan(p1, cells, order)
    theta, dt = 0.5, 0.02
    route = _lib.DIRICHLET_ROWS if rows else _lib.DIRICHLET_SYMMETRIC
    S, R, q = plan.assemble_theta(torch.as_tensor(logk, device="cuda"), f=1.5,
                                  g=torch.as_tensor(g, device="cuda"), theta=theta, dt=dt, dirichlet=route)
    blk = ot.block(pf, cf, order, bnd, np.exp(logk), f=1.5, g=g, parametric=rows)
    So = (blk.M + theta * dt * blk.A).toarray()
    Ro = (blk.M - (1 - theta) * dt * blk.A).toarray()
    qo = dt * (blk.c + blk.f)
    Sd, Rd = _csr_of(plan, S).toarray(), _csr_of(plan, R).toarray()
    assert np.abs(Sd - So).max() <= VAL_TOL * np.abs(So).max()
    assert np.abs(Rd - Ro).max() <= VAL_TOL * np.abs(Ro).max()
    assert np.abs(q.cpu().numpy() - qo).max() <= VAL_TOL * np.abs(qo).max()


@pytest.mark.parametrize("dim,n,order", [(2, 24, 1), (2, 10, 2), (3, 6, 1), (3, 4, 2)])
@pytest.mark.parametrize("theta,rows", [(1.0, True), (0.5, True), (1.0, False)])
def test_march_matches_oracle(dim, n, order, theta, rows):
    from jno_b200 import _lib

    pf, cf, cells, p1, bnd = _mesh(dim, n, order, seed=3)
    logk = om.logk_field(len(cells), 12)
    g = 0.2 + 0.3 * pf[:, 0]
    u0 = np.sin(np.pi * pf[:, 0]) * np.sin(np.pi * pf[:, 1])
    plan = _plan(p1, cells, order)
    dt, nsteps = 0.005, 8
    route = _lib.DIRICHLET_ROWS if rows else _lib.DIRICHLET_SYMMETRIC
    S, R, q = plan.assemble_theta(torch.as_tensor(logk, device="cuda"), f=1.0,
                                  g=torch.as_tensor(g, device="cuda"), theta=theta, dt=dt, dirichlet=route)
    u = torch.as_tensor(u0, device="cuda").clone()
    traj = torch.empty((nsteps, plan.n), dtype=torch.float64, device="cuda")
    _, iters, worst = plan.theta_march(S, R, q, u, nsteps, traj=traj)
    blk = ot.block(pf, cf, order, bnd, np.exp(logk), f=1.0, g=g, parametric=rows)
    to, ito, wo = ot.march(blk, u0, dt, nsteps, theta=theta)
    t = traj.cpu().numpy()
    assert np.abs(t - to[1:]).max() <= 1e-8 * np.abs(to).max()
    assert torch.equal(u, traj[-1])
    assert worst < 1e-9 and wo < 1e-9
    assert np.all(np.abs(iters - ito) <= np.maximum(2, ito // 4)), (iters, ito)


def test_march_status_paths():
    from jno_b200 import _lib

    pf, cf, cells, p1, bnd = _mesh(2, 8, 1)
    plan = _plan(p1, cells, 1)
    lk = torch.zeros(len(cells), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.FemkError):
        plan.assemble_theta(lk, theta=0.0, dt=0.01)  # forward Euler leaves the Dirichlet rows empty
    with pytest.raises(_lib.FemkError):
        plan.assemble_theta(lk, theta=1.0, dt=-1.0)
    S, R, q = plan.assemble_theta(lk, theta=1.0, dt=0.01)
    with pytest.raises(_lib.FemkError, match="nsteps"):
        plan.theta_march(S, R, q, torch.zeros(plan.n, dtype=torch.float64, device="cuda"), -1)
    # the solver-slot path (no step check) keeps BiCGStab's own status: a capped step stops the march
    u = torch.as_tensor(np.sin(np.pi * pf[:, 0]), device="cuda").clone()
    with pytest.raises(_lib.FemkError, match="step 0"):
        plan.theta_march(S, R, q, u, 3, maxiter=1, step_check=0.0)
    u2 = torch.zeros(plan.n, dtype=torch.float64, device="cuda")
    _, iters, worst = plan.theta_march(S, R, q, u2, 0)
    assert iters.size == 0 and worst == 0.0


def _heat(jno, n, time, rows=False, order=1):
    d = jno.domain(jno.domain.equi_distant_rect(nx=n, ny=n), jitter=0.1, seed=0, time=time)
    u, v = d.fem_symbols(order=order)
    xi, yi, ti = d.variable("interior", split=True)
    xb, yb, _ = d.variable("boundary", split=True)
    ci = d.variable("initial", split=True)
    ui, vi = u.bind(x=xi, y=yi, t=ti), v.bind(x=xi, y=yi, t=ti)
    ic = jno.np.sin(np.pi * ci[0]) * jno.np.sin(np.pi * ci[1])
    stiff = ui.x * vi.x + ui.y * vi.y
    if rows:
        _r, s = d.fem_symbols(space="P0", names=("r", "s"))
        stiff = jno.np.exp(jno.np.parameter(s, name="logk")) * stiff
    return jno.fem([ui.t * vi + stiff, u(xb, yb) - 0.0, u(ci[0], ci[1]) - ic])


def test_jno_surface_heat_theta_override():
    """Port of tests/test_fem_time_schemes.py:60-67 onto the B200 path: theta = 1 reproduces the
    default (backward Euler), theta = 1/2 gives a different valid answer; the trajectory matches
    the oracle's march (state0 first, n_steps rows)."""
    import jno_b200 as jno

    n, time = 12, (0.0, 0.03, 7)
    fem = _heat(jno, n, time)
    default = fem.solve().fn()
    assert default.shape == (7, fem.dofs)
    be = fem.solve(time=jno.solve.theta(1.0)).fn()
    cn = fem.solve(time=jno.solve.theta(0.5)).fn()
    assert torch.allclose(be, default, atol=1e-10)
    assert not torch.allclose(cn[-1], default[-1], atol=1e-4)
    assert torch.isfinite(cn).all()
    pf, cf, cells, p1 = om.unit_square(n, 1, seed=0)
    bnd = om.boundary_nodes(cf, 1, nv=3)
    u0 = np.sin(np.pi * pf[:, 0]) * np.sin(np.pi * pf[:, 1])
    to, _, _ = ot.march(ot.block(pf, cf, 1, bnd, np.ones(len(cells)), f=0.0, parametric=False), u0, 0.005, 6)
    assert np.abs(default.cpu().numpy() - to).max() <= 1e-8 * np.abs(to).max()
    # the parametric route through evaluate-time arguments
    fp = _heat(jno, n, time, rows=True)
    lk = om.logk_field(2 * n * n, 13)
    tp = fp.solve(args={"logk": lk}).fn().cpu().numpy()
    top, _, _ = ot.march(ot.block(pf, cf, 1, bnd, np.exp(lk), f=0.0, parametric=True), u0, 0.005, 6)
    assert np.abs(tp - top).max() <= 1e-8 * np.abs(top).max()
    with pytest.raises(ValueError):
        fem.solve(x0=torch.zeros(fem.dofs, dtype=torch.float64, device="cuda"))
    with pytest.raises(NotImplementedError):
        fem.operator  # noqa: B018 -- a transient form has no single (A, b)
    S, R, q = fem.step_operators(theta=0.5)
    assert S.numel() == fem.plan.nnz and q.numel() == fem.dofs


def test_jno_surface_march_reaches_steady_state():
    """P2 heat with a source and inhomogeneous Dirichlet data: a long backward-Euler march ends at
    the steady fem.solve() of the same form without the ui.t * vi term."""
    import jno_b200 as jno

    n = 6
    d = jno.domain(jno.domain.equi_distant_rect(nx=n, ny=n), jitter=0.1, seed=1, time=(0.0, 40.0, 41))
    u, v = d.fem_symbols(order=2)
    xi, yi, ti = d.variable("interior", split=True)
    xb, yb, _ = d.variable("boundary", split=True)
    ui, vi = u.bind(x=xi, y=yi, t=ti), v.bind(x=xi, y=yi, t=ti)
    bc = u(xb, yb) - (1.0 + xb - 0.5 * yb)
    fem_t = jno.fem([ui.t * vi + 2.0 * (ui.x * vi.x + ui.y * vi.y) - 1.0 * vi, bc])
    final = fem_t.solve().fn()[-1]
    fem_s = jno.fem([2.0 * (ui.x * vi.x + ui.y * vi.y) - 1.0 * vi, bc])
    steady = fem_s.solve(linear=jno.solve.bicgstab(tol=1e-12))
    assert (torch.linalg.norm(final - steady) / torch.linalg.norm(steady)).item() <= 1e-8


def test_jno_surface_3d_parametric_crank_nicolson():
    """The parametric route on the Kuhn box: exp(logk) P0 coefficient, source 1, u = 0.1 on the
    boundary, u0 = sin(pi x) sin(pi y) sin(pi z), Crank-Nicolson over 5 steps, against the oracle."""
    import jno_b200 as jno

    n, time = 5, (0.0, 0.02, 6)
    d = jno.domain(jno.domain.equi_distant_box(nx=n, ny=n, nz=n), jitter=0.1, seed=0, time=time)
    u, v = d.fem_symbols()
    _r, s = d.fem_symbols(space="P0", names=("r", "s"))
    xi, yi, zi, ti = d.variable("interior", split=True)
    xb, yb, zb, _ = d.variable("boundary", split=True)
    ci = d.variable("initial", split=True)
    ui, vi = u.bind(x=xi, y=yi, z=zi, t=ti), v.bind(x=xi, y=yi, z=zi, t=ti)
    logk = jno.np.parameter(s, name="logk")
    ic = jno.np.sin(np.pi * ci[0]) * jno.np.sin(np.pi * ci[1]) * jno.np.sin(np.pi * ci[2])
    fem = jno.fem([ui.t * vi + jno.np.exp(logk) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi,
                   u(xb, yb, zb) - 0.1, u(ci[0], ci[1], ci[2]) - ic])
    lk = om.logk_field(6 * n**3, 14)
    sol = fem.solve(args={"logk": lk}, time=jno.solve.theta(0.5))
    traj = sol.fn().cpu().numpy()
    assert traj.shape == (6, fem.dofs) and np.allclose(sol.ts, np.linspace(0.0, 0.02, 6))
    pf, cf, cells, p1 = om.kuhn_cube(n, 1, seed=0)
    bnd = om.boundary_nodes(cf, 1)
    u0 = np.sin(np.pi * pf[:, 0]) * np.sin(np.pi * pf[:, 1]) * np.sin(np.pi * pf[:, 2])
    blk = ot.block(pf, cf, 1, bnd, np.exp(lk), f=1.0, g=np.full(pf.shape[0], 0.1), parametric=True)
    to, _, _ = ot.march(blk, u0, 0.004, 5, theta=0.5)
    assert np.abs(traj - to).max() <= 1e-8 * np.abs(to).max()
    assert fem.stats["transient"]["step_residual"] < 1e-9


def test_jno_surface_transient_solver_slots_match_default():
    """Port of tests/test_fem_solver_transient.py:54-69: with solver slots the per-step solve is
    the slot solver at its own tolerance with the step operator's Jacobi preconditioner
    (compose_transient_step_solvers); CG + Jacobi at 1e-10 and BiCGStab + Jacobi (the precond-only
    slot, tolerance 1e-8) reproduce the default backward-Euler trajectory."""
    import jno_b200 as jno

    fem = _heat(jno, 10, (0.0, 0.2, 21))
    ref = fem.solve().fn()
    cg = fem.solve(linear=jno.solve.cg(tol=1e-10), precond=jno.precond.jacobi()).fn()
    assert (cg - ref).abs().max().item() < 1e-8
    bi = fem.solve(precond=jno.precond.jacobi()).fn()
    assert (bi - ref).abs().max().item() < 1e-6
    assert fem.stats["transient"]["step_residual"] <= 1e-4
    with pytest.raises(NotImplementedError):
        fem.solve(linear=jno.solve.cg(precision="mixed"))
