"""CPU tests: the oracle against the reference-generated golden fixtures and the reference's
known-answer properties (no GPU)."""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import assemble as oa
from oracle import element as oe
from oracle import mesh as om
from oracle import pcg as op

CASES = [(2, 2, 2), (3, 2, 4), (4, 4, 4)]


@pytest.mark.parametrize("nx,ny,nz", CASES)
def test_mesh_matches_reference(golden, nx, ny, nz):
    tag = f"{nx}x{ny}x{nz}"
    pts, tets = om.equi_distant_box(nx, ny, nz)
    assert np.array_equal(pts, golden[f"{tag}/points"])
    assert np.array_equal(tets, golden[f"{tag}/tets"])


@pytest.mark.parametrize("nx,ny,nz", CASES)
def test_p2_numbering_matches_reference(golden, nx, ny, nz):
    tag = f"{nx}x{ny}x{nz}"
    pts, cells = om.promote_p2(golden[f"{tag}/jittered"], golden[f"{tag}/tets"])
    assert np.array_equal(cells, golden[f"{tag}/p2_cells"])
    assert np.array_equal(pts, golden[f"{tag}/p2_points"])


@pytest.mark.parametrize("nx,ny,nz", CASES)
@pytest.mark.parametrize("order", [1, 2])
def test_compress_plan_matches_reference(golden, nx, ny, nz, order):
    tag = f"{nx}x{ny}x{nz}"
    cells = golden[f"{tag}/tets"] if order == 1 else golden[f"{tag}/p2_cells"]
    idx, inverse, nse = oa.compress_plan(cells)
    assert nse == int(golden[f"{tag}/p{order}_nse"])
    assert np.array_equal(idx, golden[f"{tag}/p{order}_idx"])
    assert np.array_equal(inverse, golden[f"{tag}/p{order}_inverse"])
    n = int(cells.max()) + 1
    indptr, indices, slot = oa.csr_pattern_fast(cells, n)
    ip2, ind2 = oa.plan_to_csr(idx, n)
    assert np.array_equal(indptr, ip2) and np.array_equal(indices, ind2)
    assert np.array_equal(slot, inverse)


@pytest.mark.parametrize("nx,ny,nz", CASES)
@pytest.mark.parametrize("order", [1, 2])
def test_boundary_nodes_match_reference(golden, nx, ny, nz, order):
    tag = f"{nx}x{ny}x{nz}"
    cells = golden[f"{tag}/tets"] if order == 1 else golden[f"{tag}/p2_cells"]
    assert np.array_equal(om.boundary_nodes(cells, order), golden[f"{tag}/p{order}_boundary"])


def test_sizes_of_the_configs():
    """Appendix sizes: n, boundary DOFs and nse at P1 8^3 / P2 4^3 follow the closed formulas."""
    for nh in (3, 8):
        pts, tets = om.equi_distant_box(nh, nh, nh)
        E = 3 * nh * (nh + 1) ** 2 + 3 * nh**2 * (nh + 1) + nh**3
        n = (nh + 1) ** 3
        _, _, nse = oa.compress_plan(tets)
        assert nse == n + 2 * E
        assert om.boundary_nodes(tets, 1).size == 6 * nh * nh + 2
        p2p, p2c = om.promote_p2(pts, tets)
        assert p2p.shape[0] == n + E
        assert om.boundary_nodes(p2c, 2).size == 6 * (2 * nh) ** 2 + 2


@pytest.mark.parametrize("order", [1, 2])
def test_closed_form_equals_quadrature(order):
    pts, tets = om.equi_distant_box(3, 3, 3)
    pts = om.jitter_interior(pts, 3, 3, 3, seed=5)
    X = pts[tets]
    K1, F1 = oe.element_matrices(X, order)
    K2, F2 = oe.element_matrices_quadrature(X, order)
    assert np.abs(K1 - K2).max() <= 1e-12 * np.abs(K1).max()
    assert np.abs(F1 - F2).max() <= 1e-12 * np.abs(F1).max()
    # symmetric, rows sum to zero (constants are in the kernel), partition of unity on the load
    assert np.abs(K1 - K1.transpose(0, 2, 1)).max() <= 1e-13 * np.abs(K1).max()
    assert np.abs(K1.sum(axis=2)).max() <= 1e-12 * np.abs(K1).max()
    vol = np.abs(np.linalg.det(np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], -1))) / 6
    assert np.allclose(F1.sum(axis=1), vol, rtol=1e-13)


def _solve_direct(system):
    return spla.spsolve(system.csr().tocsc(), system.b)


def test_p1_recovers_linear_field():
    """Port of tests/test_fem_3d.py:76-89: u = 1 + 2x + 3y + 4z is reproduced exactly by P1."""
    n = 4
    pts, tets = om.equi_distant_box(n, n, n)
    pts = om.jitter_interior(pts, n, n, n, seed=3)
    bnd = om.boundary_nodes(tets, 1)
    g = 1 + 2 * pts[:, 0] + 3 * pts[:, 1] + 4 * pts[:, 2]
    s = oa.assemble(pts, tets, 1, bnd, np.ones(len(tets)), f=0.0, g=g)
    u = _solve_direct(s)
    assert np.abs(u - g).max() < 1e-9


def test_p2_reproduces_quadratic_exactly():
    """Port of tests/test_fem_native_lagrange.py:377-395 (P2 patch test, f = -12)."""
    n = 3
    pts, tets = om.equi_distant_box(n, n, n)
    pts = om.jitter_interior(pts, n, n, n, seed=4)
    p2p, p2c = om.promote_p2(pts, tets)
    bnd = om.boundary_nodes(p2c, 2)
    x, y, z = p2p.T
    exact = x**2 + 2 * y**2 + 3 * z**2 + x * y
    s = oa.assemble(p2p, p2c, 2, bnd, np.ones(len(tets)), f=-12.0, g=exact)
    u = _solve_direct(s)
    assert np.abs(u - exact).max() < 1e-9


def test_p0_linearity_and_support():
    """Port of tests/test_topology_optimisation.py:210-237 on the free block."""
    n = 3
    pts, tets = om.equi_distant_box(n, n, n)
    bnd = om.boundary_nodes(tets, 1)
    T = len(tets)
    full = oa.assemble(pts, tets, 1, bnd, np.ones(T)).csr().toarray()
    free = np.setdiff1d(np.arange(full.shape[0]), bnd)
    acc = np.zeros((free.size, free.size))
    for j in range(T):
        acc += oa.assemble(pts, tets, 1, bnd, np.eye(T)[j]).csr().toarray()[np.ix_(free, free)]
    assert np.abs(acc - full[np.ix_(free, free)]).max() <= 1e-12
    j = 40
    kj = oa.assemble(pts, tets, 1, bnd, np.eye(T)[j]).csr().toarray()
    cell = set(tets[j].tolist())
    off = [i for i in range(kj.shape[0]) if i not in cell and i not in set(bnd.tolist())]
    assert np.abs(kj[np.ix_(off, off)]).max() == 0.0


def test_dirichlet_rows_are_identity_and_zeros_kept():
    n = 3
    pts, tets = om.equi_distant_box(n, n, n)
    bnd = om.boundary_nodes(tets, 1)
    s = oa.assemble(pts, tets, 1, bnd, np.exp(om.logk_field(len(tets), 1)))
    _, _, nse = oa.compress_plan(tets)
    assert s.data.size == nse  # explicit zeros stay stored (parametric route)
    A = s.csr().toarray()
    assert np.array_equal(A[bnd][:, bnd], np.eye(bnd.size))
    assert np.abs(A[bnd]).sum() == bnd.size and np.abs(A[:, bnd]).sum() == bnd.size
    assert np.allclose(A, A.T, atol=0, rtol=0) or np.abs(A - A.T).max() < 1e-15
    assert oa.compact(s).nnz < nse


def test_pcg_matches_direct_and_jacobi_guard():
    n = 6
    pts, tets = om.equi_distant_box(n, n, n)
    pts = om.jitter_interior(pts, n, n, n, seed=0)
    bnd = om.boundary_nodes(tets, 1)
    s = oa.assemble(pts, tets, 1, bnd, np.exp(om.logk_field(len(tets), 1000)))
    A = s.csr()
    d = oa.matrix_diagonal(s)
    x, it, hist = op.pcg(A, s.b, oa.jacobi_inverse(d), tol=1e-8)
    xd = _solve_direct(s)
    assert it > 5 and hist[-1] <= 1e-16 * np.dot(s.b, s.b)
    assert np.abs(x - xd).max() <= 1e-7 * np.abs(xd).max()
    assert op.residual_check(A, s.b, x) < 1e-7
    assert np.array_equal(oa.jacobi_inverse(np.array([0.0, 2.0, 1e-31])), np.array([1.0, 0.5, 1.0]))


def test_pcg_zero_rhs_takes_no_iteration():
    A = np.eye(3)
    x, it, _ = op.pcg(A, np.zeros(3), np.ones(3))
    assert it == 0 and np.all(x == 0)


def test_bicgstab_matches_direct_and_stops_like_jax():
    n = 6
    pts, tets = om.equi_distant_box(n, n, n)
    pts = om.jitter_interior(pts, n, n, n, seed=0)
    bnd = om.boundary_nodes(tets, 1)
    s = oa.assemble(pts, tets, 1, bnd, np.exp(om.logk_field(len(tets), 1000)))
    A = s.csr()
    inv = oa.jacobi_inverse(oa.matrix_diagonal(s))
    x, k = op.bicgstab(A, s.b, inv, tol=1e-8)
    xd = _solve_direct(s)
    assert k > 3 and np.linalg.norm(s.b - A @ x) <= 1e-8 * np.linalg.norm(s.b) * 1.0000001
    assert np.abs(x - xd).max() <= 1e-7 * np.abs(xd).max()
    # zero right-hand side: no iteration; a cap of one iteration stops after one
    x0, k0 = op.bicgstab(A, np.zeros_like(s.b), inv)
    assert k0 == 0 and np.all(x0 == 0)
    _, k1 = op.bicgstab(A, s.b, inv, maxiter=1)
    assert k1 == 1


def test_gmres_restatement_converges_restarts_and_breaks_down():
    """The restated jax gmres: one long cycle and many short restart cycles reach the direct
    solution; a non-symmetric system converges; a Krylov space that closes early (a diagonal with
    three distinct values) gives the exact answer in one cycle (with one Gram-Schmidt pass the
    rounding left after step three stays above the eps v0 threshold, so the cycle runs on); an
    eigenvector right-hand side breaks down exactly after one step; b = 0 runs no cycle."""
    import scipy.sparse as sp

    n = 6
    pts, tets = om.equi_distant_box(n, n, n)
    pts = om.jitter_interior(pts, n, n, n, seed=1)
    s = oa.assemble(pts, tets, 1, om.boundary_nodes(tets, 1), np.exp(om.logk_field(len(tets), 3)))
    A = s.csr()
    inv = oa.jacobi_inverse(oa.matrix_diagonal(s))
    xd = _solve_direct(s)
    for restart, cycles_at_least in ((30, 1), (5, 5)):
        x, steps, cycles, _ = op.gmres(A, s.b, inv, tol=1e-10, restart=restart)
        assert cycles >= cycles_at_least and steps <= cycles * restart
        assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    skew = sp.random(A.shape[0], A.shape[0], density=5.0 / A.shape[0], random_state=1)
    B = (A + 0.05 * (skew - skew.T)).tocsr()
    import scipy.sparse.linalg as spla

    xb = spla.spsolve(B.tocsc(), s.b)
    x, _, _, _ = op.gmres(B, s.b, inv, tol=1e-10, restart=30)
    assert np.linalg.norm(x - xb) <= 1e-8 * np.linalg.norm(xb)
    D = sp.diags(np.repeat([1.0, 2.0, 5.0], 10)).tocsr()
    x, steps, cycles, beta = op.gmres(D, np.ones(30), None, tol=1e-12, restart=20)
    assert steps >= 3 and cycles == 1 and np.abs(D @ x - 1.0).max() <= 1e-14
    e = np.zeros(30)
    e[4] = 1.0
    x, steps, cycles, beta = op.gmres(D, e, None, tol=1e-12, restart=20)
    assert steps == 1 and cycles == 1 and beta == 0.0 and np.array_equal(x, e)
    x0, steps0, cycles0, _ = op.gmres(A, np.zeros_like(s.b), inv)
    assert steps0 == 0 and cycles0 == 0 and np.all(x0 == 0)


def test_nodal_coefficient_rule():
    """The 4-point rule integrates degree-2 polynomials exactly; a linear nodal field's element
    mean is its vertex mean; a constant log-field gives exp of it."""
    pts, tets = om.equi_distant_box(2, 2, 2)
    rng = np.random.default_rng(9)
    vals = rng.normal(size=pts.shape[0])
    lin = oe.nodal_coefficient(tets, vals, "linear")
    assert np.allclose(lin, vals[tets].mean(axis=1), rtol=0, atol=1e-15)
    assert np.allclose(oe.nodal_coefficient(tets, np.full(pts.shape[0], 0.3), "exp"), np.exp(0.3), rtol=1e-15)
    # the rule against a collapsed-Gauss rule on a quadratic in barycentric coordinates
    xi, w = oe._collapsed_gauss(6)
    lam = np.column_stack([1.0 - xi.sum(axis=1), xi])
    f = lam[:, 0] * lam[:, 1] + 0.5 * lam[:, 2] ** 2 + lam[:, 3]
    exact = (w * f).sum() * 6.0  # mean over the unit tet (volume 1/6)
    lamq = np.full((4, 4), oe._Q4_A) + np.eye(4) * (oe._Q4_B - oe._Q4_A)
    fq = lamq[:, 0] * lamq[:, 1] + 0.5 * lamq[:, 2] ** 2 + lamq[:, 3]
    assert abs(fq.mean() - exact) <= 1e-14


@pytest.mark.parametrize("mode", ["exp", "linear"])
def test_oracle_nodal_gradient_matches_fd(mode):
    from oracle import adjoint as oadj

    n = 3
    pf, cf, tets, p1 = om.kuhn_cube(n, 1, seed=2)
    rng = np.random.default_rng(5)
    vals = rng.normal(0.0, 0.4, pf.shape[0]) if mode == "exp" else rng.uniform(0.5, 2.0, pf.shape[0])
    bnd = om.boundary_nodes(cf, 1)
    ustar = rng.normal(size=pf.shape[0])
    mass = oadj.lumped_mass(pf, cf, 1)
    J, g = oadj.gradient_nodal(pf, cf, bnd, vals, mode, ustar, mass, tol=1e-14)

    def Jof(v):
        s = oa.assemble(pf, cf, 1, bnd, oe.nodal_coefficient(cf, v, mode))
        u = _solve_direct(s)
        return oadj.misfit(u, ustar, mass)

    interior = np.setdiff1d(np.arange(pf.shape[0]), bnd)
    for i in interior[:5]:
        e = np.zeros(pf.shape[0])
        e[i] = 1e-6
        fd = (Jof(vals + e) - Jof(vals - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * np.abs(g).max() + 1e-6 * abs(g[i])


@pytest.mark.parametrize("dim,n", [(2, 32), (3, 12)])
def test_mixed_single_reduction_matches_textbook_loop(dim, n):
    """The mixed solver's FP32 iteration in single-reduction form (all products of an iteration in
    one reduction, <p', A p'> expanded) runs the same iteration as the textbook FP32 loop: FP32
    iteration counts within a few, FP64 updates equal, both meet the FP64 stop rule, and the solutions
    agree with a tight FP64 solve to 1e-7. Restart mode (beta = 0 at each update) also converges."""
    pf, cf, cells, p1 = om.unit_square(n, 1, seed=0) if dim == 2 else om.kuhn_cube(n, 1, seed=0)
    s = oa.assemble(pf, cf, 1, om.boundary_nodes(cf, 1, nv=dim + 1), np.exp(om.logk_field(len(cells), 1000)))
    A = s.csr()
    inv = oa.jacobi_inverse(oa.matrix_diagonal(s))
    xt, _, _ = op.pcg(A, s.b, inv, tol=1e-13)
    out = {}
    for tag, kw in (("single", {}), ("textbook", {"single_reduction": False}), ("restart", {"restart": True})):
        x, it, outer = op.mixed_pcg(A, s.b, inv, tol=1e-8, **kw)
        assert np.linalg.norm(s.b - A @ x) <= 1e-8 * np.linalg.norm(s.b)
        assert np.linalg.norm(x - xt) <= 1e-7 * np.linalg.norm(xt)
        out[tag] = (it, outer)
    assert abs(out["single"][0] - out["textbook"][0]) <= 3 and out["single"][1] == out["textbook"][1]
