"""Oracle: the linear first-order transient block and its theta-method march (test infrastructure).

Restates, with the reference's separate operators applied one product at a time:
* the consistent mass of the temporal term ``u_t * v`` -- the jacobian of the mass terms
  (``jno/utils/solver/fem_native.py:2846-2850``): ``M[a, b] = integral(phi_a phi_b)``, by an
  independent collapsed-Gauss quadrature here (exact for the degree <= 4 integrands);
* the two Dirichlet treatments of the block:
  - non-parametric route, ``_apply_dirichlet_transient`` (``jno/utils/solver/fem_1d.py:939-949``):
    ``A``, ``c`` by symmetric elimination (the steady parametric assembly: Dirichlet rows/columns
    zero, ``A[d, d] = 1``, ``c = load - A e``, ``c[d] = g``), ``M`` rows and columns zeroed;
  - parametric route (``fem_native.py:3058-3087``): ``A`` with Dirichlet rows replaced by identity
    rows (``bcoo_set_dirichlet_rows``, columns kept), ``M`` rows and columns zeroed,
    ``c[d] = g[d]`` (the affine bias) and the forcing ``f = free-mask * load``;
* ``SemidiscreteTimeBlock.step`` for a linear block (``jno/utils/solver/backend_blocks.py:332-413``):
  ``rhs = M u - (1 - theta) dt (A u) + dt c + dt f``, ``step(w) = M w + theta dt (A w)``,
  ``inv = 1 / where(|d| > 1e-30, d, 1)`` with ``d = diag(M) + theta dt diag(A)``, then
  ``jax.scipy.sparse.linalg.bicgstab(step, rhs, x0=u, tol=1e-10, atol=0, maxiter=20000, M=inv)``
  and the step check ``||step(u') - rhs|| / max(||rhs||, eps) < max(1e-9, 1e4 eps)``; a step that
  fails it is re-solved from ``x0 = u`` by ``jax.scipy.sparse.linalg.gmres`` (``tol=max(1e-10,
  100 eps)``, ``atol=0``, ``restart=min(n, 40)``, the same Jacobi ``M``; ``backend_blocks.py:402-413``);
* ``_default_transient_integrate`` (``backend_blocks.py:475-530``): the grid of ``n_steps`` points
  from ``t0`` to ``t1`` (``_infer_time_window``, ``jno/utils/solver/time_route.py:32-58``,
  ``dt = (t1 - t0) / (n_steps - 1)``), trajectory = state0 followed by every step.
"""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .assemble import assemble, compress_plan, plan_to_csr
from .element import _collapsed_gauss, _collapsed_gauss_tri, _ref_basis, vertices
from .pcg import bicgstab, gmres


def mass_matrices(X, order, npts=5):
    """Element mass matrices f64[T, nd, nd] by collapsed-Gauss quadrature (X f64[T, d+1, d])."""
    d = X.shape[2]
    xi, w = _collapsed_gauss(npts) if d == 3 else _collapsed_gauss_tri(npts)
    phi, _ = _ref_basis(order, xi)
    J = np.stack([X[:, k + 1] - X[:, 0] for k in range(d)], axis=-1)
    meas = np.abs(np.linalg.det(J))
    return np.einsum("q,t,qa,qb->tab", w, meas, phi, phi)


def mass_csr(points, cells, order, dirichlet=None):
    """Consistent mass in the canonical CSR (scipy), Dirichlet rows/columns zeroed when given."""
    cells = np.asarray(cells, dtype=np.int64)
    n = np.asarray(points).shape[0]
    idx, inverse, nse = compress_plan(cells)
    indptr, indices = plan_to_csr(idx, n)
    Me = mass_matrices(vertices(points, cells), order)
    data = np.bincount(inverse.astype(np.int64), weights=Me.reshape(-1), minlength=nse)
    if dirichlet is not None:
        isd = np.zeros(n, dtype=bool)
        isd[np.asarray(dirichlet, dtype=np.int64)] = True
        rows = np.repeat(np.arange(n), np.diff(indptr))
        data[isd[rows] | isd[indices]] = 0.0
    return sp.csr_matrix((data, indices, indptr), shape=(n, n))


class Block:
    """Linear block ``M u' + A u = c + f`` with the reference's Dirichlet treatment for its route."""

    def __init__(self, M, A, c, f):
        self.M, self.A, self.c, self.f = M, A, c, f


def block(points, cells, order, dirichlet, coef, f=1.0, g=None, parametric=True):
    n = np.asarray(points).shape[0]
    dirichlet = np.asarray(dirichlet, dtype=np.int64)
    M = mass_csr(points, cells, order, dirichlet)
    if not parametric:
        s = assemble(points, cells, order, dirichlet, coef, f=f, g=g)
        return Block(M, s.csr(), s.b.copy(), np.zeros(n))
    # stiffness and load with no Dirichlet treatment, then row replacement
    s = assemble(points, cells, order, np.zeros(0, dtype=np.int64), coef, f=f)
    A = s.csr().tolil()
    for d in dirichlet:
        A.rows[d] = [int(d)]
        A.data[d] = [1.0]
    A = A.tocsr()
    c = np.zeros(n)
    if g is not None:
        c[dirichlet] = np.asarray(g, dtype=np.float64)[dirichlet]
    load = s.b.copy()
    load[dirichlet] = 0.0
    return Block(M, A, c, load)


def step(blk, u, dt, theta=1.0, tol=1e-10, maxiter=20_000, info=None):
    """One theta step; returns (u_next, bicgstab iteration count k, step residual). The step
    residual is BiCGStab's; when it fails the check the GMRES rescue runs, and ``info`` (a dict,
    optional) receives its Arnoldi steps and the rescued solution's residual."""
    M, A = blk.M, blk.A
    rhs = M @ u - (1.0 - theta) * dt * (A @ u) + dt * blk.c + dt * blk.f
    n = u.shape[0]
    op = spla.LinearOperator((n, n), matvec=lambda w: M @ w + theta * dt * (A @ w), dtype=np.float64)
    d = M.diagonal() + theta * dt * A.diagonal()
    inv = 1.0 / np.where(np.abs(d) > 1e-30, d, 1.0)
    wn, k = bicgstab(op, rhs, inv, x0=u, tol=tol, atol=0.0, maxiter=maxiter)
    eps = np.finfo(np.float64).eps
    r_rel = float(np.linalg.norm(op @ wn - rhs) / max(np.linalg.norm(rhs), eps))
    if not (r_rel < max(1e-9, 1e4 * eps)):
        wn, steps, _, _ = gmres(op, rhs, inv, x0=u, tol=max(1e-10, 100.0 * eps), atol=0.0, restart=min(n, 40))
        if info is not None:
            info["gmres_steps"] = info.get("gmres_steps", 0) + steps
            info["rescued_residual"] = float(np.linalg.norm(op @ wn - rhs) / max(np.linalg.norm(rhs), eps))
    return wn, k, r_rel


def march(blk, u0, dt, nsteps, theta=1.0, tol=1e-10, maxiter=20_000, info=None):
    """Trajectory f64[nsteps + 1, n] (state0 first), iteration counts, worst BiCGStab step residual."""
    u = np.array(u0, dtype=np.float64)
    traj, iters, worst = [u.copy()], [], 0.0
    for _ in range(nsteps):
        u, k, r = step(blk, u, dt, theta, tol, maxiter, info)
        traj.append(u.copy())
        iters.append(k)
        worst = max(worst, r)
    return np.array(traj), np.array(iters), worst
