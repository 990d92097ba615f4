"""Oracle: P1/P2 tetrahedral element stiffness and load (test infrastructure).

Follows ``_cell_fields`` (``jno/utils/solver/fem_native.py:1461-1497``) and
``identity_pushforward`` (``jno/utils/solver/fem_lagrange.py:348-381``): the affine map has
``J = [x1-x0, x2-x0, x3-x0]`` (edge vectors as columns), ``meas = |det J|`` and physical gradients
``dphi/dx = dphi/dxi . J^-1``. The element residual of ``k*grad u.grad v - f*v``
(``_vol_elem_res`` ``fem_native.py:1645-1691``) differentiated by ``jax.jacfwd`` (``:2333-2334``)
gives ``K_e[a, b] = k * integral(grad phi_b . grad phi_a)`` with rows = test dof a, columns = trial
dof b, and ``b_e[a] = f * integral(phi_a)``.

Closed forms in barycentric coordinates (g_i = grad lambda_i, G_ij = g_i . g_j, V = |det J| / 6):
* P1: ``K = k V G``; ``F = f V / 4``.
* P2 (basix order: vertices 0..3, then edges ``(2,3),(1,3),(1,2),(0,3),(0,2),(0,1)``):
  ``grad phi_i = (4 lambda_i - 1) g_i`` and ``grad phi_ij = 4 (lambda_j g_i + lambda_i g_j)``
  integrated with ``int lambda_i lambda_j = V (1 + delta_ij) / 20`` and ``int lambda_i = V / 4``;
  ``F_vertex = -f V / 20``, ``F_edge = f V / 5``.
"""

import numpy as np

from .mesh import TET_EDGES


def p1_geometry(X):
    """Barycentric gradients g f64[T,4,3] and signed det J f64[T] for vertex coords X f64[T,4,3]."""
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=-1)
    det = np.linalg.det(J)
    Jinv = np.linalg.inv(J)  # Jinv[t, n, d] = d xi_n / d x_d
    g = np.empty((X.shape[0], 4, 3))
    g[:, 1:, :] = Jinv
    g[:, 0, :] = -Jinv.sum(axis=1)
    return g, det


def _p2_coeffs():
    """Constant tensors C[p, q, i, j] with K_hat[p, q] = V * sum_ij C[p,q,i,j] G_ij."""
    # Each P2 gradient is sum_m (alpha_m + sum_l beta_ml lambda_l) g_m; write it as a linear form in
    # (1, lambda_0..3) times g_m: coef[p, m, s] with s = 0 for the constant, s = 1 + l for lambda_l.
    coef = np.zeros((10, 4, 5))
    for i in range(4):
        coef[i, i, 0] = -1.0
        coef[i, i, 1 + i] = 4.0
    for e, (i, j) in enumerate(TET_EDGES):
        coef[4 + e, i, 1 + j] = 4.0
        coef[4 + e, j, 1 + i] = 4.0
    # moments M[s, t] = (1/V) * integral(s-th basis monomial * t-th), monomials (1, lambda_0..3)
    M = np.zeros((5, 5))
    M[0, 0] = 1.0
    M[0, 1:] = M[1:, 0] = 0.25
    M[1:, 1:] = (np.ones((4, 4)) + np.eye(4)) / 20.0
    return np.einsum("pms,qnt,st->pqmn", coef, coef, M)


_P2C = _p2_coeffs()


def element_matrices(X, order):
    """Unit-coefficient element stiffness K_hat f64[T,nd,nd] and unit-source load F_hat f64[T,nd]."""
    g, det = p1_geometry(X)
    V = np.abs(det) / 6.0
    G = np.einsum("tid,tjd->tij", g, g)
    if order == 1:
        K = V[:, None, None] * G
        F = np.repeat((V / 4.0)[:, None], 4, axis=1)
        return K, F
    K = V[:, None, None] * np.einsum("pqij,tij->tpq", _P2C, G)
    F = np.empty((X.shape[0], 10))
    F[:, :4] = (-V / 20.0)[:, None]
    F[:, 4:] = (V / 5.0)[:, None]
    return K, F


def _collapsed_gauss(npts):
    """Points xi f64[q,3] and weights w f64[q] on the reference tet from a collapsed Gauss rule."""
    x, w = np.polynomial.legendre.leggauss(npts)
    x, w = 0.5 * (x + 1.0), 0.5 * w
    U, Vv, W = np.meshgrid(x, x, x, indexing="ij")
    wu, wv, ww = np.meshgrid(w, w, w, indexing="ij")
    xi0 = U
    xi1 = (1.0 - U) * Vv
    xi2 = (1.0 - U) * (1.0 - Vv) * W
    jac = (1.0 - U) ** 2 * (1.0 - Vv)
    pts = np.stack([xi0.ravel(), xi1.ravel(), xi2.ravel()], axis=1)
    return pts, (wu * wv * ww * jac).ravel()


def _ref_basis(order, xi):
    """Reference values f64[q,nd] and gradients f64[q,nd,3] of the P1/P2 basis at points xi."""
    lam = np.column_stack([1.0 - xi.sum(axis=1), xi])
    dlam = np.array([[-1.0, -1.0, -1.0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    if order == 1:
        return lam, np.broadcast_to(dlam, (xi.shape[0], 4, 3)).copy()
    phi = np.empty((xi.shape[0], 10))
    dphi = np.empty((xi.shape[0], 10, 3))
    for i in range(4):
        phi[:, i] = lam[:, i] * (2 * lam[:, i] - 1)
        dphi[:, i] = (4 * lam[:, i] - 1)[:, None] * dlam[i]
    for e, (i, j) in enumerate(TET_EDGES):
        phi[:, 4 + e] = 4 * lam[:, i] * lam[:, j]
        dphi[:, 4 + e] = 4 * (lam[:, j][:, None] * dlam[i] + lam[:, i][:, None] * dlam[j])
    return phi, dphi


def element_matrices_quadrature(X, order, npts=4):
    """Same matrices by numerical quadrature (independent cross-check of the closed forms)."""
    xi, w = _collapsed_gauss(npts)
    phi, dphi = _ref_basis(order, xi)
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=-1)
    meas = np.abs(np.linalg.det(J))
    Kinv = np.linalg.inv(J)
    dphys = np.einsum("qnd,tdD->tqnD", dphi, Kinv)
    K = np.einsum("q,t,tqaD,tqbD->tab", w, meas, dphys, dphys)
    F = np.einsum("q,t,qa->ta", w, meas, phi)
    return K, F


# symmetric 4-point degree-2 tetrahedron rule: barycentric (b, a, a, a) and permutations, weights 1/4
_Q4_A = (5.0 - np.sqrt(5.0)) / 20.0
_Q4_B = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0


def nodal_coefficient(tets, values, mode):
    """Per-element k_e of a nodal P1 parameter for P1 stiffness (whose integrand is constant per
    element, so K_e = V G mean_q k(x_q)).

    The reference passes a nodal field parameter as the cell's local nodal values
    (``_runtime_vals``, ``jno/utils/solver/fem_native.py:1597-1630``) and interpolates them to the
    quadrature points of the degree-2 rule P1 forms use (``jno/_fem.py:4551``); basix (which
    supplies that rule) is absent here, so the symmetric 4-point rule is used.
    ``mode`` "linear": k = p_h (the vertex mean, exact); "exp": k = exp(p_h) averaged over the rule.
    """
    p = np.asarray(values, dtype=np.float64)[np.asarray(tets)]
    if mode == "linear":
        return 0.25 * p.sum(axis=1)
    lam = np.full((4, 4), _Q4_A) + np.eye(4) * (_Q4_B - _Q4_A)  # lam[q, i]
    return 0.25 * np.exp(p @ lam.T).sum(axis=1)

