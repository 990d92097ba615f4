"""Oracle: gradient of a nodal misfit through the FP64 solve w.r.t. per-element log k (test infrastructure).

The reference differentiates with ``jax.grad`` through ``lax.custom_linear_solve`` inside
``jax.scipy.sparse.linalg.cg`` (``jno/solve.py:202-206``), back through the Dirichlet mask
(``jno/utils/solver/fem_utils.py:3332-3337``), ``segment_sum`` (``fem_native.py:2326``) and the
per-cell ``jacfwd`` (``:2333-2334``) to the P0 value ``flat[c]`` (``fem_native.py:1619-1622``).
``custom_linear_solve`` differentiates the solve implicitly (the preconditioner does not enter), so
with ``A u = b`` and ``J(u)``:

    lambda = A^-T dJ/du;  dJ/dlogk_c = -lambda^T (dA/dlogk_c) u = -k_c (m o lambda)_e^T K_hat_e (m o u)_e

with ``m = 1 - isDirichlet`` (the zeroed rows/columns do not depend on k; ``b`` does not depend on k).
The misfit is ``J = 1/2 sum_i M_ii (u_i - u*_i)^2`` with the lumped mass ``M_ii = sum_{e ni i} int phi_i``.
"""

import numpy as np

from .assemble import assemble
from .element import element_matrices, vertices
from .pcg import pcg


def lumped_mass(points, cells, order):
    _, F = element_matrices(vertices(points, cells), order)
    return np.bincount(cells.reshape(-1), weights=F.reshape(-1), minlength=points.shape[0])


def misfit(u, ustar, mass):
    d = u - ustar
    return 0.5 * float(np.sum(mass * d * d))


def solve(points, cells, order, dirichlet, logk, tol=1e-12, plan=None, element=None):
    sysm = assemble(points, cells, order, dirichlet, np.exp(logk), plan=plan, element=element)
    A = sysm.csr()
    from .assemble import jacobi_inverse, matrix_diagonal

    x, it, _ = pcg(A, sysm.b, jacobi_inverse(matrix_diagonal(sysm)), tol=tol)
    return x, sysm, it


def gradient(points, cells, order, dirichlet, logk, ustar, mass, tol=1e-12):
    """(J, dJ/dlogk f64[T]) by the adjoint method, FP64."""
    u, sysm, _ = solve(points, cells, order, dirichlet, logk, tol=tol)
    A = sysm.csr()
    from .assemble import jacobi_inverse, matrix_diagonal

    lam, _, _ = pcg(A.T.tocsr(), mass * (u - ustar), jacobi_inverse(matrix_diagonal(sysm)), tol=tol)
    m = (~sysm.dirichlet).astype(np.float64)
    Khat, _ = element_matrices(vertices(points, cells), order)
    le = (m * lam)[cells]
    ue = (m * u)[cells]
    grad = -np.exp(logk) * np.einsum("ta,tab,tb->t", le, Khat, ue)
    return misfit(u, ustar, mass), grad


def gradient_nodal(points, cells, dirichlet, values, mode, ustar, mass, tol=1e-12):
    """(J, dJ/dp f64[nvert]) for a nodal P1 parameter p: the element gradient dJ/dk_e (as above,
    with k_e from ``element.nodal_coefficient``) spread onto the vertices by dk_e/dp_i."""
    from .assemble import jacobi_inverse, matrix_diagonal
    from .element import nodal_coefficient, nodal_rule

    ke = nodal_coefficient(cells, values, mode)
    sysm = assemble(points, cells, 1, dirichlet, ke)
    A = sysm.csr()
    inv = jacobi_inverse(matrix_diagonal(sysm))
    u, _, _ = pcg(A, sysm.b, inv, tol=tol)
    lam, _, _ = pcg(A.T.tocsr(), mass * (u - ustar), inv, tol=tol)
    m = (~sysm.dirichlet).astype(np.float64)
    Khat, _ = element_matrices(vertices(points, cells), 1)
    dJdk = -np.einsum("ta,tab,tb->t", (m * lam)[cells], Khat, (m * u)[cells])
    p = np.asarray(values, dtype=np.float64)[cells]
    nv = p.shape[1]
    if mode == "linear":
        dk = np.full(p.shape, 1.0 / nv)
    else:
        qa, qb = nodal_rule(nv)
        lamq = np.full((nv, nv), qa) + np.eye(nv) * (qb - qa)
        e = np.exp(p @ lamq.T)
        dk = (qa * e.sum(axis=1, keepdims=True) + (qb - qa) * e) / nv
    grad = np.bincount(cells.reshape(-1), weights=(dJdk[:, None] * dk).reshape(-1), minlength=points.shape[0])
    return misfit(u, ustar, mass), grad

