"""GPU parity of restarted GMRES (jax.scipy.sparse.linalg.gmres semantics: jno.solve.gmres and the
theta march's step rescue) against the oracle on the same seeded systems. Bars: the solution within
1e-7 of the direct solve (1e-8 stop rule on the preconditioned residual); restart cycles within one
of the oracle's (a cycle that ends at the threshold may land on either side of it) and Arnoldi
steps within one cycle of the oracle's; the march trajectory within 1e-8 of the oracle's."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import assemble as oa  # noqa: E402
from oracle import mesh as om  # noqa: E402
from oracle import pcg as op  # noqa: E402
from oracle import transient as ot  # noqa: E402


def _system(dim, n, order, seed, options=None):
    from jno_b200.plan import FemPlan

    pf, cf, cells, p1 = om.kuhn_cube(n, order, seed=1) if dim == 3 else om.unit_square(n, order, seed=1)
    logk = om.logk_field(len(cells), seed)
    plan = FemPlan(p1, cells, order, options=options)
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    s = oa.assemble(pf, cf, order, om.boundary_nodes(cf, order, nv=dim + 1), np.exp(logk))
    return plan, vals, b, s


def _direct(s):
    import scipy.sparse.linalg as spla

    return spla.spsolve(s.csr().tocsc(), s.b)


@pytest.mark.parametrize("dim,n,order,restart", [(3, 8, 1, 30), (3, 4, 2, 30), (2, 16, 1, 30), (2, 16, 1, 5),
                                                 (2, 6, 2, 12)])
def test_gmres_matches_oracle(dim, n, order, restart):
    plan, vals, b, s = _system(dim, n, order, 1020)
    inv = plan.jacobi(vals)
    x, steps, cycles, rel, st = plan.gmres(vals, b, inv_diag=inv, tol=1e-8, restart=restart)
    xo, so, co, beta = op.gmres(s.csr(), s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8, restart=restart)
    assert st == 0
    assert abs(cycles - co) <= 1, (cycles, co)
    assert abs(steps - so) <= restart, (steps, so)
    xd = _direct(s)
    xx = x.cpu().numpy()
    assert np.linalg.norm(xx - xd) <= 1e-7 * np.linalg.norm(xd)
    assert np.linalg.norm(xx - xo) <= 1e-7 * np.linalg.norm(xd)
    # ||b - A x|| / ||b|| carries the rounding of b - A x itself: about 1e-15 of ||b|| per evaluation
    assert rel == pytest.approx(op.residual_check(s.csr(), s.b, xx, rtol=1.0), rel=1e-6, abs=1e-13)


def test_gmres_unpreconditioned_warm_start_zero_rhs_and_cap():
    from jno_b200 import _lib

    plan, vals, b, s = _system(2, 12, 1, 1021)
    xd = _direct(s)
    x, steps, cycles, rel, st = plan.gmres(vals, b, tol=1e-9, restart=20)
    xo, so, co, _ = op.gmres(s.csr(), s.b, None, tol=1e-9, restart=20)
    assert st == 0 and abs(cycles - co) <= 1 and abs(steps - so) <= 20
    assert np.linalg.norm(x.cpu().numpy() - xd) <= 1e-7 * np.linalg.norm(xd)
    # warm start at the solution: no cycle, x untouched
    x2, steps2, cycles2, _, st2 = plan.gmres(vals, b, x=x.clone(), tol=1e-6, restart=20)
    assert st2 == 0 and cycles2 == 0 and steps2 == 0 and torch.equal(x2, x)
    # b = 0: the residual normalises to zero, no cycle, x stays 0
    z, steps3, cycles3, _, st3 = plan.gmres(vals, torch.zeros_like(b), tol=1e-8)
    assert st3 == 0 and steps3 == 0 and cycles3 == 0 and torch.all(z == 0)
    # a cap of one cycle reports NOT_CONVERGED with x written
    xc, stepsc, cyclesc, relc, stc = plan.gmres(vals, b, tol=1e-12, restart=2, maxiter=1)
    assert stc == _lib.FEMK_NOT_CONVERGED and cyclesc == 1 and stepsc == 2 and relc < 1.0


def test_gmres_breakdown_ignores_stale_basis_columns():
    """An Arnoldi breakdown ends a cycle early; the basis columns past it are never written in that
    cycle (jax starts every cycle from a zero basis). Here they hold NaN left by an earlier call: a
    restart-30 solve sizes the plan's Krylov workspace, a restart-5 call on NaN values leaves NaN in
    the scratch vector that a restart-20 cycle sees as basis column 6, and a right-hand side e_d on a
    Dirichlet DOF d (A e_d = e_d, diag 1) then breaks down after one step. The update must read only
    the written column: x = e_d exactly."""
    import ctypes

    from jno_b200 import _lib

    plan, vals, b, s = _system(3, 6, 1, 1022)
    inv = plan.jacobi(vals)
    plan.gmres(vals, b, inv_diag=inv, tol=1e-8, restart=30)
    bad = vals.clone()
    bad[::7] = float("nan")
    x = torch.zeros_like(b)
    it, cyc, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
    st = plan._lib.femk_gmres(plan.handle, _lib.ptr(bad), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv), 1e-8, 0.0, 5, -1,
                              ctypes.byref(it), ctypes.byref(cyc), ctypes.byref(rr), _lib.stream_handle())
    assert st == _lib.FEMK_NONFINITE
    d = int(torch.nonzero(plan.export()["dirichlet_mask"]).flatten()[0])
    e = torch.zeros_like(b)
    e[d] = 1.0
    x, steps, cycles, rel, st = plan.gmres(vals, e, inv_diag=inv, tol=1e-8, restart=20)
    assert st == 0 and steps == 1 and cycles == 1 and rel == 0.0
    assert torch.equal(x, e)
    xo, so, co, beta = op.gmres(s.csr(), e.cpu().numpy(), oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8,
                                restart=20)
    assert (so, co, beta) == (1, 1, 0.0) and np.array_equal(xo, e.cpu().numpy())


def test_gmres_maxiter_zero_runs_no_cycle_and_restart_is_validated():
    import jno_b200 as jno

    plan, vals, b, s = _system(2, 8, 1, 1023)
    x, steps, cycles, rel, st = plan.gmres(vals, b, tol=1e-8, restart=10, maxiter=0)
    assert st == 4 and steps == 0 and cycles == 0 and torch.count_nonzero(x) == 0
    with pytest.raises(ValueError):
        jno.solve.gmres(restart=65)
    with pytest.raises(ValueError):
        jno.solve.gmres(maxiter=-1)


def test_gmres_on_the_canonical_csr_path_matches():
    plan, vals, b, s = _system(3, 6, 1, 1022, options={"solver_layout": 0})
    inv = plan.jacobi(vals)
    x, steps, cycles, rel, st = plan.gmres(vals, b, inv_diag=inv, tol=1e-8, restart=30)
    xo, so, co, _ = op.gmres(s.csr(), s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8, restart=30)
    assert st == 0 and abs(cycles - co) <= 1 and abs(steps - so) <= 30
    xd = _direct(s)
    assert np.linalg.norm(x.cpu().numpy() - xd) <= 1e-7 * np.linalg.norm(xd)


def test_gmres_replay_is_bitwise_reproducible():
    plan, vals, b, s = _system(3, 8, 1, 1023)
    inv = plan.jacobi(vals)
    a = plan.gmres(vals, b, inv_diag=inv, tol=1e-10, restart=25)
    c = plan.gmres(vals, b, inv_diag=inv, tol=1e-10, restart=25)
    assert a[1] == c[1] and a[2] == c[2] and torch.equal(a[0], c[0])


def test_jno_solve_gmres_surface():
    import jno_b200 as jno
    from jno_b200.sparse import CsrMatrix

    plan, vals, b, s = _system(3, 6, 2, 1024)
    A = CsrMatrix(plan, vals)
    solver = jno.solve.gmres(restart=30)
    x = solver(A, b, M=jno.precond.jacobi())
    xd = _direct(s)
    assert np.linalg.norm(x.cpu().numpy() - xd) <= 1e-7 * np.linalg.norm(xd)
    assert solver.last_info.outer >= 1 and solver.last_info.iterations >= 1
    assert jno.solve.gmres(restart=30) == jno.solve.gmres(restart=30) != jno.solve.gmres(restart=20)
    with pytest.raises(RuntimeError, match="did not solve"):
        jno.solve.gmres(restart=1, maxiter=1)(A, b, M=jno.precond.jacobi())


@pytest.mark.parametrize("dim,theta", [(2, 1.0), (3, 0.5)])
def test_march_rescues_failed_steps_with_gmres(dim, theta):
    """BiCGStab capped at one iteration fails every step check; each step is re-solved from the
    previous state by GMRES (restart min(n, 40), tol 1e-10) as the reference's step does, and the
    trajectory matches the oracle's march with the same cap and rescue."""
    from jno_b200 import _lib
    from jno_b200.plan import FemPlan

    if dim == 2:
        pf, cf, cells, p1 = om.unit_square(10, 1, seed=2)
    else:
        pf, cf, cells, p1 = om.kuhn_cube(5, 1, seed=2)
    bnd = om.boundary_nodes(cf, 1, nv=dim + 1)
    logk = om.logk_field(len(cells), 1025)
    plan = FemPlan(p1, cells, 1)
    u0 = np.prod([np.sin(np.pi * pf[:, i]) for i in range(dim)], axis=0)
    dt, nsteps = 0.01, 4
    S, R, q = plan.assemble_theta(torch.as_tensor(logk, device="cuda"), f=1.0, theta=theta, dt=dt,
                                  dirichlet=_lib.DIRICHLET_ROWS)
    u = torch.as_tensor(u0, device="cuda").clone()
    traj = torch.empty((nsteps, plan.n), dtype=torch.float64, device="cuda")
    _, iters, worst, rescue = plan.theta_march(S, R, q, u, nsteps, maxiter=1, traj=traj, with_rescue=True)
    assert np.all(iters == 1) and np.all(rescue > 0) and worst >= 1e-9
    blk = ot.block(pf, cf, 1, bnd, np.exp(logk), f=1.0, parametric=True)
    info = {}
    to, _, _ = ot.march(blk, u0, dt, nsteps, theta=theta, maxiter=1, info=info)
    assert info["gmres_steps"] > 0
    assert np.abs(traj.cpu().numpy() - to[1:]).max() <= 1e-8 * np.abs(to).max()
    # without the cap no step needs the rescue, and the march lands on the same states
    u2 = torch.as_tensor(u0, device="cuda").clone()
    _, _, worst2, rescue2 = plan.theta_march(S, R, q, u2, nsteps, with_rescue=True)
    assert np.all(rescue2 == 0) and worst2 < 1e-9
    assert (torch.linalg.norm(u2 - u) / torch.linalg.norm(u2)).item() <= 1e-8
