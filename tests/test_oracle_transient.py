"""CPU tests of the transient oracle (theta-method march of the linear first-order block): the
consistent mass, the reference's known-answer properties of the time schemes, and the two
Dirichlet routes (no GPU)."""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import assemble as oa
from oracle import element as oe
from oracle import mesh as om
from oracle import transient as ot


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 2), (3, 1), (3, 2)])
def test_mass_integrates_the_domain_and_lumps_to_the_load(dim, order):
    """sum M = |domain| (the P1 mass check of tests/test_fem_convergence.py:771-775) and
    sum_b M[a, b] = integral(phi_a), the unit load."""
    if dim == 2:
        pf, cf, _, _ = om.unit_square(4, order, seed=1)
    else:
        pf, cf, _, _ = om.kuhn_cube(2, order, seed=1)
    M = ot.mass_csr(pf, cf, order)
    assert abs(M.sum() - 1.0) <= 1e-13
    _, F = oe.element_matrices(oe.vertices(pf, cf), order)
    lump = np.bincount(cf.reshape(-1), weights=F.reshape(-1), minlength=pf.shape[0])
    assert np.abs(np.asarray(M.sum(axis=1)).ravel() - lump).max() <= 1e-15
    assert abs(M - M.T).max() <= 1e-17


def _heat_2d(n, order, seed=0):
    pf, cf, tris, _ = om.unit_square(n, order, seed=seed)
    bnd = om.boundary_nodes(cf, order, nv=3)
    u0 = np.sin(np.pi * pf[:, 0]) * np.sin(np.pi * pf[:, 1])
    return pf, cf, bnd, u0


def test_backward_euler_decay_matches_the_discrete_factor():
    """Homogeneous heat from the first mode: each backward-Euler step divides the mode by
    (1 + dt lambda_h) with lambda_h the discrete Rayleigh quotient of the mode."""
    pf, cf, bnd, u0 = _heat_2d(16, 1)
    blk = ot.block(pf, cf, 1, bnd, np.ones(len(cf)), f=0.0)
    traj, iters, worst = ot.march(blk, u0, 0.01, 10)
    lam = float(u0 @ (blk.A @ u0)) / float(u0 @ (blk.M @ u0))
    assert abs(lam - 2 * np.pi**2) < 0.05 * 2 * np.pi**2
    ratio = np.linalg.norm(traj[-1]) / np.linalg.norm(u0)
    assert abs(ratio - (1.0 / (1.0 + 0.01 * lam)) ** 10) < 2e-3
    assert worst < 1e-9 and np.all(iters > 0)


@pytest.mark.parametrize("theta,lo,hi", [(1.0, 0.8, 1.2), (0.5, 1.8, 2.2)])
def test_theta_scheme_time_order(theta, lo, hi):
    """Observed order in dt on a fixed mesh against a fine Crank-Nicolson march: backward Euler
    first order, Crank-Nicolson second order (the schemes of jno.solve.theta, jno/solve.py:1160)."""
    pf, cf, bnd, u0 = _heat_2d(8, 1, seed=2)
    blk = ot.block(pf, cf, 1, bnd, np.exp(om.logk_field(len(cf), 3)), f=1.0)
    T = 0.05
    ref = ot.march(blk, u0, T / 640, 640, theta=0.5)[0][-1]
    errs = []
    for nsteps in (10, 20, 40):
        u = ot.march(blk, u0, T / nsteps, nsteps, theta=theta)[0][-1]
        errs.append(np.linalg.norm(u - ref))
    p = np.polyfit(np.log([T / 10, T / 20, T / 40]), np.log(errs), 1)[0]
    assert lo <= p <= hi, (p, errs)


def test_long_march_reaches_the_steady_solution():
    """With a constant source and Dirichlet data the march converges to the steady solve."""
    pf, cf, bnd, u0 = _heat_2d(8, 2, seed=3)
    k = np.exp(om.logk_field(len(cf), 4))
    g = 1.0 + pf[:, 0] - 0.5 * pf[:, 1]
    for parametric in (True, False):
        blk = ot.block(pf, cf, 2, bnd, k, f=2.0, g=g, parametric=parametric)
        traj, _, _ = ot.march(blk, u0, 1.0, 40)
        s = oa.assemble(pf, cf, 2, bnd, k, f=2.0, g=g)
        steady = spla.spsolve(s.csr().tocsc(), s.b)
        assert np.abs(traj[-1] - steady).max() <= 1e-8 * np.abs(steady).max()


def test_failed_step_check_is_rescued_by_gmres():
    """A BiCGStab capped at one iteration fails every step check; the GMRES rescue
    (backend_blocks.py:402-413) re-solves each step and the march lands on the uncapped one."""
    pf, cf, bnd, u0 = _heat_2d(8, 1, seed=2)
    blk = ot.block(pf, cf, 1, bnd, np.exp(om.logk_field(len(cf), 3)), f=1.0)
    info = {}
    a, it, worst = ot.march(blk, u0, 0.01, 3, maxiter=1, info=info)
    b = ot.march(blk, u0, 0.01, 3)[0]
    assert np.all(it == 1) and worst > 1e-9
    assert info["gmres_steps"] > 0 and info["rescued_residual"] <= 1e-12
    assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()


def test_routes_agree_for_homogeneous_dirichlet_and_differ_in_the_held_rows():
    """With g = 0 and u0 = 0 on the boundary both Dirichlet routes give the same trajectory; with
    theta = 1/2 and u0 != g on the boundary the parametric route's held rows follow
    u_d' = (g - (1 - theta) u_d) / theta, while the symmetric route's free rows never see u_d."""
    pf, cf, bnd, u0 = _heat_2d(6, 1, seed=4)
    k = np.exp(om.logk_field(len(cf), 5))
    a = ot.march(ot.block(pf, cf, 1, bnd, k, f=1.0, parametric=True), u0, 0.01, 5)[0]
    b = ot.march(ot.block(pf, cf, 1, bnd, k, f=1.0, parametric=False), u0, 0.01, 5)[0]
    assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()
    g = np.full(pf.shape[0], 0.3)
    u1 = u0 + 1.0
    tr = ot.march(ot.block(pf, cf, 1, bnd, k, f=0.0, g=g, parametric=True), u1, 0.01, 3, theta=0.5)[0]
    held = [u1[bnd]]
    for _ in range(3):
        held.append((0.3 - 0.5 * held[-1]) / 0.5)
    assert np.abs(tr[:, bnd] - np.array(held)).max() <= 1e-9
