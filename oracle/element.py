"""Oracle: P1/P2 tetrahedral and triangular element stiffness and load (test infrastructure).

Follows ``_cell_fields`` (``jno/utils/solver/fem_native.py:1461-1497``) and
``identity_pushforward`` (``jno/utils/solver/fem_lagrange.py:348-381``): the affine map has
``J = [x1-x0, ..., x_d-x0]`` (edge vectors as columns), ``meas = |det J|`` and physical gradients
``dphi/dx = dphi/dxi . J^-1``; a triangle (d = 2) reads its points as ``[:, :2]``. The element residual of ``k*grad u.grad v - f*v``
(``_vol_elem_res`` ``fem_native.py:1645-1691``) differentiated by ``jax.jacfwd`` (``:2333-2334``)
gives ``K_e[a, b] = k * integral(grad phi_b . grad phi_a)`` with rows = test dof a, columns = trial
dof b, and ``b_e[a] = f * integral(phi_a)``.

Closed forms in barycentric coordinates (g_i = grad lambda_i, G_ij = g_i . g_j, V = |det J| / 6):
* P1: ``K = k V G``; ``F = f V / 4``.
* P2 (basix order: vertices 0..3, then edges ``(2,3),(1,3),(1,2),(0,3),(0,2),(0,1)``):
  ``grad phi_i = (4 lambda_i - 1) g_i`` and ``grad phi_ij = 4 (lambda_j g_i + lambda_i g_j)``
  integrated with ``int lambda_i lambda_j = V (1 + delta_ij) / 20`` and ``int lambda_i = V / 4``;
  ``F_vertex = -f V / 20``, ``F_edge = f V / 5``.
* Triangles (A = |det J| / 2; P2 edges ``(1,2),(0,2),(0,1)``): the same forms with
  ``int lambda_i lambda_j = A (1 + delta_ij) / 12`` and ``int lambda_i = A / 3``; P1 ``F = f A / 3``,
  P2 ``F_vertex = 0``, ``F_edge = f A / 3``.
"""

import math

import numpy as np

from .mesh import TET_EDGES, TRI_EDGES


def vertices(points, cells):
    """Vertex coordinates f64[T, d+1, d] of the cells of a d-dimensional mesh (points f64[n, d])."""
    points = np.asarray(points, dtype=np.float64)
    d = points.shape[1]
    return points[np.asarray(cells)[:, : d + 1]]


def p1_geometry(X):
    """Barycentric gradients g f64[T,d+1,d] and signed det J f64[T] for vertex coords X f64[T,d+1,d]."""
    d = X.shape[2]
    J = np.stack([X[:, k + 1] - X[:, 0] for k in range(d)], axis=-1)
    det = np.linalg.det(J)
    Jinv = np.linalg.inv(J)  # Jinv[t, n, d] = d xi_n / d x_d
    g = np.empty((X.shape[0], d + 1, d))
    g[:, 1:, :] = Jinv
    g[:, 0, :] = -Jinv.sum(axis=1)
    return g, det


def _p2_coeffs(nv):
    """Constant tensors C[p, q, i, j] with K_hat[p, q] = V * sum_ij C[p,q,i,j] G_ij (nv vertices)."""
    # Each P2 gradient is sum_m (alpha_m + sum_l beta_ml lambda_l) g_m; write it as a linear form in
    # (1, lambda_0..) times g_m: coef[p, m, s] with s = 0 for the constant, s = 1 + l for lambda_l.
    edges = TET_EDGES if nv == 4 else TRI_EDGES
    nd = nv + len(edges)
    coef = np.zeros((nd, nv, nv + 1))
    for i in range(nv):
        coef[i, i, 0] = -1.0
        coef[i, i, 1 + i] = 4.0
    for e, (i, j) in enumerate(edges):
        coef[nv + e, i, 1 + j] = 4.0
        coef[nv + e, j, 1 + i] = 4.0
    # moments M[s, t] = (1/V) * integral(s-th basis monomial * t-th), monomials (1, lambda_0..)
    M = np.zeros((nv + 1, nv + 1))
    M[0, 0] = 1.0
    M[0, 1:] = M[1:, 0] = 1.0 / nv
    M[1:, 1:] = (np.ones((nv, nv)) + np.eye(nv)) / (nv * (nv + 1))
    return np.einsum("pms,qnt,st->pqmn", coef, coef, M)


_P2C = {4: _p2_coeffs(4), 3: _p2_coeffs(3)}


def element_matrices(X, order):
    """Unit-coefficient element stiffness K_hat f64[T,nd,nd] and unit-source load F_hat f64[T,nd]
    for vertex coordinates X f64[T, d+1, d] (d = 3: tetrahedra, d = 2: triangles)."""
    g, det = p1_geometry(X)
    nv = X.shape[1]
    V = np.abs(det) / math.factorial(nv - 1)
    G = np.einsum("tid,tjd->tij", g, g)
    if order == 1:
        K = V[:, None, None] * G
        F = np.repeat((V / nv)[:, None], nv, axis=1)
        return K, F
    K = V[:, None, None] * np.einsum("pqij,tij->tpq", _P2C[nv], G)
    nd = K.shape[1]
    F = np.empty((X.shape[0], nd))
    F[:, :nv] = (V * (3.0 - nv) / (nv * (nv + 1)))[:, None]
    F[:, nv:] = (4.0 * V / (nv * (nv + 1)))[:, None]
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


def _collapsed_gauss_tri(npts):
    """Points xi f64[q,2] and weights w f64[q] on the reference triangle (collapsed Gauss)."""
    x, w = np.polynomial.legendre.leggauss(npts)
    x, w = 0.5 * (x + 1.0), 0.5 * w
    U, Vv = np.meshgrid(x, x, indexing="ij")
    wu, wv = np.meshgrid(w, w, indexing="ij")
    pts = np.stack([U.ravel(), ((1.0 - U) * Vv).ravel()], axis=1)
    return pts, (wu * wv * (1.0 - U)).ravel()


def _ref_basis(order, xi):
    """Reference values f64[q,nd] and gradients f64[q,nd,d] of the P1/P2 basis at points xi f64[q,d]."""
    d = xi.shape[1]
    nv = d + 1
    lam = np.column_stack([1.0 - xi.sum(axis=1), xi])
    dlam = np.vstack([-np.ones((1, d)), np.eye(d)])
    if order == 1:
        return lam, np.broadcast_to(dlam, (xi.shape[0], nv, d)).copy()
    edges = TET_EDGES if nv == 4 else TRI_EDGES
    nd = nv + len(edges)
    phi = np.empty((xi.shape[0], nd))
    dphi = np.empty((xi.shape[0], nd, d))
    for i in range(nv):
        phi[:, i] = lam[:, i] * (2 * lam[:, i] - 1)
        dphi[:, i] = (4 * lam[:, i] - 1)[:, None] * dlam[i]
    for e, (i, j) in enumerate(edges):
        phi[:, nv + e] = 4 * lam[:, i] * lam[:, j]
        dphi[:, nv + e] = 4 * (lam[:, j][:, None] * dlam[i] + lam[:, i][:, None] * dlam[j])
    return phi, dphi


def element_matrices_quadrature(X, order, npts=4):
    """Same matrices by numerical quadrature (independent cross-check of the closed forms)."""
    d = X.shape[2]
    xi, w = _collapsed_gauss(npts) if d == 3 else _collapsed_gauss_tri(npts)
    phi, dphi = _ref_basis(order, xi)
    J = np.stack([X[:, k + 1] - X[:, 0] for k in range(d)], axis=-1)
    meas = np.abs(np.linalg.det(J))
    Kinv = np.linalg.inv(J)
    dphys = np.einsum("qnd,tdD->tqnD", dphi, Kinv)
    K = np.einsum("q,t,tqaD,tqbD->tab", w, meas, dphys, dphys)
    F = np.einsum("q,t,qa->ta", w, meas, phi)
    return K, F


# symmetric degree-2 rules, equal weights: tetrahedron 4 points with barycentric (b, a, a, a) and
# permutations; triangle 3 points (2/3, 1/6, 1/6) and permutations
_Q4_A = (5.0 - np.sqrt(5.0)) / 20.0
_Q4_B = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0
_Q3_A = 1.0 / 6.0
_Q3_B = 2.0 / 3.0


def nodal_rule(nv):
    """(a, b) of the degree-2 rule of a simplex with nv vertices: point q has lambda_q = b, others a."""
    return (_Q4_A, _Q4_B) if nv == 4 else (_Q3_A, _Q3_B)


def nodal_coefficient(tets, values, mode):
    """Per-element k_e of a nodal P1 parameter for P1 stiffness (whose integrand is constant per
    element, so K_e = V G mean_q k(x_q)); ``tets`` i64[T, nv] (nv = 4 tetrahedra, 3 triangles).

    The reference passes a nodal field parameter as the cell's local nodal values
    (``_runtime_vals``, ``jno/utils/solver/fem_native.py:1597-1630``) and interpolates them to the
    quadrature points of the degree-2 rule P1 forms use (``jno/_fem.py:4551``); basix (which
    supplies that rule) is absent here, so the symmetric 4-point (tetrahedron) / 3-point (triangle)
    rule is used. ``mode`` "linear": k = p_h (the vertex mean, exact); "exp": k = exp(p_h) averaged
    over the rule.
    """
    p = np.asarray(values, dtype=np.float64)[np.asarray(tets)]
    nv = p.shape[1]
    if mode == "linear":
        return p.sum(axis=1) / nv
    a, b = nodal_rule(nv)
    lam = np.full((nv, nv), a) + np.eye(nv) * (b - a)  # lam[q, i]
    return np.exp(p @ lam.T).sum(axis=1) / nv


def exact_poisson_2d(x, y):
    """A solution of -Laplace u = 1 on the unit square: u = x(1-x)/2 + sin(pi x) sinh(pi y) / sinh(pi)."""
    return 0.5 * x * (1.0 - x) + np.sin(np.pi * x) * np.sinh(np.pi * y) / np.sinh(np.pi)


def l2_error_2d(pf, cf, order, u, exact, npts=8):
    """True L2 error of the P1/P2 triangle field u (nodal values f64[n]) against exact(x, y), by a
    collapsed Gauss rule of npts x npts points per triangle."""
    xi, w = _collapsed_gauss_tri(npts)
    phi, _ = _ref_basis(order, xi)
    X = vertices(pf, cf)
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]], axis=-1)
    meas = np.abs(np.linalg.det(J))
    xq = X[:, 0][:, None, :] + np.einsum("tdn,qn->tqd", J, xi)
    uh = np.einsum("qa,ta->tq", phi, np.asarray(u)[np.asarray(cf)])
    err = uh - exact(xq[..., 0], xq[..., 1])
    return float(np.sqrt(np.einsum("q,t,tq->", w, meas, err * err)))
