"""CPU tests of the 2-D (triangle) oracle: against the reference-generated golden fixtures of
``Geometries.equi_distant_rect``, ``_promote_to_degree``, ``compress_plan`` and ``_boundary_facets``
(tests/golden/make_golden.py) and the reference's known-answer properties (no GPU)."""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import assemble as oa
from oracle import element as oe
from oracle import mesh as om

CASES = [(2, 2), (3, 2), (5, 4)]


@pytest.mark.parametrize("nx,ny", CASES)
def test_rect_mesh_matches_reference(golden2d, nx, ny):
    tag = f"{nx}x{ny}"
    pts, tris = om.equi_distant_rect(nx, ny)
    assert np.array_equal(pts, golden2d[f"{tag}/points"])
    assert np.array_equal(tris, golden2d[f"{tag}/tris"])
    assert float(golden2d[f"{tag}/ds"]) == min(1.0 / nx, 1.0 / ny)


@pytest.mark.parametrize("nx,ny", CASES)
def test_tri_p2_numbering_matches_reference(golden2d, nx, ny):
    tag = f"{nx}x{ny}"
    pts, cells = om.promote_p2(golden2d[f"{tag}/jittered"], golden2d[f"{tag}/tris"])
    assert np.array_equal(cells, golden2d[f"{tag}/p2_cells"])
    assert np.array_equal(pts, golden2d[f"{tag}/p2_points"])


@pytest.mark.parametrize("nx,ny", CASES)
@pytest.mark.parametrize("order", [1, 2])
def test_tri_compress_plan_matches_reference(golden2d, nx, ny, order):
    tag = f"{nx}x{ny}"
    cells = golden2d[f"{tag}/tris"] if order == 1 else golden2d[f"{tag}/p2_cells"]
    idx, inverse, nse = oa.compress_plan(cells)
    assert nse == int(golden2d[f"{tag}/p{order}_nse"])
    assert np.array_equal(idx, golden2d[f"{tag}/p{order}_idx"])
    assert np.array_equal(inverse, golden2d[f"{tag}/p{order}_inverse"])
    n = int(cells.max()) + 1
    indptr, indices, slot = oa.csr_pattern_fast(cells, n)
    ip2, ind2 = oa.plan_to_csr(idx, n)
    assert np.array_equal(indptr, ip2) and np.array_equal(indices, ind2)
    assert np.array_equal(slot, inverse)


@pytest.mark.parametrize("nx,ny", CASES)
@pytest.mark.parametrize("order", [1, 2])
def test_tri_boundary_nodes_match_reference(golden2d, nx, ny, order):
    tag = f"{nx}x{ny}"
    cells = golden2d[f"{tag}/tris"] if order == 1 else golden2d[f"{tag}/p2_cells"]
    assert np.array_equal(om.boundary_nodes(cells, order, nv=3), golden2d[f"{tag}/p{order}_boundary"])


def test_tri_sizes():
    """n^2 rectangles: (n+1)^2 vertices, E = 2n(n+1) + n^2 edges, nse = N + 2E, 4n boundary
    vertices; P2 adds E nodes and 4n boundary midpoints."""
    for nh in (3, 8):
        pts, tris = om.equi_distant_rect(nh, nh)
        E = 2 * nh * (nh + 1) + nh * nh
        N = (nh + 1) ** 2
        assert oa.compress_plan(tris)[2] == N + 2 * E
        assert om.boundary_nodes(tris, 1, nv=3).size == 4 * nh
        p2p, p2c = om.promote_p2(pts, tris)
        assert p2p.shape == (N + E, 2) and p2c.shape == (2 * nh * nh, 6)
        assert om.boundary_nodes(p2c, 2, nv=3).size == 8 * nh


@pytest.mark.parametrize("order", [1, 2])
def test_tri_closed_form_equals_quadrature(order):
    pts, tris = om.equi_distant_rect(4, 3)
    pts = om.jitter_interior_2d(pts, 4, 3, seed=5)
    pf, cf = (pts, tris) if order == 1 else om.promote_p2(pts, tris)
    X = oe.vertices(pf, cf)
    K1, F1 = oe.element_matrices(X, order)
    K2, F2 = oe.element_matrices_quadrature(X, order, npts=5)
    assert np.abs(K1 - K2).max() <= 1e-12 * np.abs(K1).max()
    assert np.abs(F1 - F2).max() <= 1e-12 * np.abs(F1).max()
    assert np.abs(K1 - K1.transpose(0, 2, 1)).max() <= 1e-13 * np.abs(K1).max()
    assert np.abs(K1.sum(axis=2)).max() <= 1e-12 * np.abs(K1).max()
    area = 0.5 * np.abs(np.linalg.det(np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]], -1)))
    assert np.allclose(F1.sum(axis=1), area, rtol=1e-13)
    if order == 2:
        assert np.all(F1[:, :3] == 0.0)  # P2 vertex functions integrate to zero on a triangle


def _solve_direct(system):
    return spla.spsolve(system.csr().tocsc(), system.b)


def test_tri_p1_recovers_linear_field():
    """The 2-D form of tests/test_fem_3d.py:76-89: u = 1 + 2x + 3y is reproduced exactly by P1."""
    n = 6
    pts, tris = om.equi_distant_rect(n, n)
    pts = om.jitter_interior_2d(pts, n, n, seed=3)
    bnd = om.boundary_nodes(tris, 1, nv=3)
    g = 1 + 2 * pts[:, 0] + 3 * pts[:, 1]
    s = oa.assemble(pts, tris, 1, bnd, np.full(len(tris), 1.7), f=0.0, g=g)
    assert np.abs(_solve_direct(s) - g).max() < 1e-11


def test_tri_p2_reproduces_quadratic_exactly():
    """The 2-D form of tests/test_fem_native_lagrange.py:377-395: u = x^2 + 2y^2 + xy, f = -6."""
    n = 4
    pts, tris = om.equi_distant_rect(n, n)
    pts = om.jitter_interior_2d(pts, n, n, seed=4)
    p2p, p2c = om.promote_p2(pts, tris)
    bnd = om.boundary_nodes(p2c, 2, nv=3)
    x, y = p2p.T
    exact = x**2 + 2 * y**2 + x * y
    s = oa.assemble(p2p, p2c, 2, bnd, np.ones(len(tris)), f=-6.0, g=exact)
    assert np.abs(_solve_direct(s) - exact).max() < 1e-11


@pytest.mark.parametrize("order,lo,hi", [(1, 1.7, 2.4), (2, 2.6, 3.4)])
def test_tri_poisson_convergence_order(order, lo, hi):
    """The gate of tests/test_fem_convergence.py:209-235 and :771-779 (observed L2 order of P1 in
    [1.7, 2.4], of P2 in [2.6, 3.4]) on a transcendental solution with a constant source, the
    inhomogeneous Dirichlet data carrying the harmonic part."""
    errs, hs = [], []
    for n in (4, 8, 16):
        pf, cf, _, _ = om.unit_square(n, order, seed=1, amp=0.1)
        bnd = om.boundary_nodes(cf, order, nv=3)
        g = oe.exact_poisson_2d(pf[:, 0], pf[:, 1])
        s = oa.assemble(pf, cf, order, bnd, np.ones(cf.shape[0]), f=1.0, g=g)
        errs.append(oe.l2_error_2d(pf, cf, order, _solve_direct(s), oe.exact_poisson_2d))
        hs.append(1.0 / n)
    assert np.all(np.diff(errs) < 0)
    p = np.polyfit(np.log(hs), np.log(errs), 1)[0]
    assert lo <= p <= hi, (p, errs)


def test_tri_nodal_coefficient_rule():
    """The 3-point rule integrates quadratics exactly on a triangle; linear mode is the vertex mean."""
    pts, tris = om.equi_distant_rect(3, 3)
    vals = np.random.default_rng(9).normal(size=pts.shape[0])
    assert np.allclose(oe.nodal_coefficient(tris, vals, "linear"), vals[tris].mean(axis=1), rtol=0, atol=1e-15)
    assert np.allclose(oe.nodal_coefficient(tris, np.full(pts.shape[0], 0.3), "exp"), np.exp(0.3), rtol=1e-15)
    xi, w = oe._collapsed_gauss_tri(6)
    lam = np.column_stack([1.0 - xi.sum(axis=1), xi])
    f = lam[:, 0] * lam[:, 1] + 0.5 * lam[:, 2] ** 2 + lam[:, 1]
    exact = (w * f).sum() * 2.0  # mean over the unit triangle (area 1/2)
    a, b = oe.nodal_rule(3)
    lamq = np.full((3, 3), a) + np.eye(3) * (b - a)
    fq = lamq[:, 0] * lamq[:, 1] + 0.5 * lamq[:, 2] ** 2 + lamq[:, 1]
    assert abs(fq.mean() - exact) <= 1e-14


@pytest.mark.parametrize("mode", ["exp", "linear"])
def test_tri_oracle_nodal_gradient_matches_fd(mode):
    from oracle import adjoint as oadj

    pf, cf, _, _ = om.unit_square(5, 1, seed=2)
    rng = np.random.default_rng(5)
    vals = rng.normal(0.0, 0.4, pf.shape[0]) if mode == "exp" else rng.uniform(0.5, 2.0, pf.shape[0])
    bnd = om.boundary_nodes(cf, 1, nv=3)
    ustar = rng.normal(size=pf.shape[0])
    mass = oadj.lumped_mass(pf, cf, 1)
    J, g = oadj.gradient_nodal(pf, cf, bnd, vals, mode, ustar, mass, tol=1e-14)

    def Jof(v):
        s = oa.assemble(pf, cf, 1, bnd, oe.nodal_coefficient(cf, v, mode))
        return oadj.misfit(_solve_direct(s), ustar, mass)

    interior = np.setdiff1d(np.arange(pf.shape[0]), bnd)
    for i in interior[:5]:
        e = np.zeros(pf.shape[0])
        e[i] = 1e-6
        fd = (Jof(vals + e) - Jof(vals - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * np.abs(g).max() + 1e-6 * abs(g[i])


@pytest.mark.parametrize("order", [1, 2])
def test_tri_oracle_p0_gradient_matches_fd(order):
    from oracle import adjoint as oadj

    pf, cf, _, _ = om.unit_square(4, order, seed=6)
    rng = np.random.default_rng(7)
    logk = rng.normal(0.0, 0.5, cf.shape[0])
    bnd = om.boundary_nodes(cf, order, nv=3)
    ustar = rng.normal(size=pf.shape[0])
    mass = oadj.lumped_mass(pf, cf, order)
    J, g = oadj.gradient(pf, cf, order, bnd, logk, ustar, mass, tol=1e-14)

    def Jof(lk):
        s = oa.assemble(pf, cf, order, bnd, np.exp(lk))
        return oadj.misfit(_solve_direct(s), ustar, mass)

    for c in (0, 7, 19):
        e = np.zeros(cf.shape[0])
        e[c] = 1e-6
        fd = (Jof(logk + e) - Jof(logk - e)) / 2e-6
        assert abs(fd - g[c]) <= 1e-6 * np.abs(g).max() + 1e-6 * abs(g[c])
