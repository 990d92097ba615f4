"""GPU parity: the CUDA path through the C ABI against the oracle on the same seeded inputs.

Bars: integer/index outputs bit-exact; FP64 matrix values and loads within 1e-12 of the oracle
relative to the largest entry; solves to the 1e-8 stop rule with the solution within 1e-7 of the
oracle's; adjoint gradient within 1e-8 of the oracle's adjoint and 1e-6 of central differences.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import adjoint as oadj  # noqa: E402
from oracle import assemble as oa  # noqa: E402
from oracle import element as oe  # noqa: E402
from oracle import mesh as om  # noqa: E402
from oracle import pcg as op  # noqa: E402

VAL_TOL = 1e-12


def _plan(points, tets, order, options=None):
    from jno_b200.plan import FemPlan

    return FemPlan(points, tets, order, options=options)


def _mesh(n, order, seed=0):
    return om.kuhn_cube(n, order=order, seed=seed)


def _oracle_system(pf, cf, order, logk, f=1.0, g=None):
    bnd = om.boundary_nodes(cf, order)
    return oa.assemble(pf, cf, order, bnd, np.exp(logk), f=f, g=g), bnd


@pytest.mark.parametrize("n,order", [(2, 1), (4, 1), (8, 1), (2, 2), (4, 2), (6, 2)])
def test_plan_matches_oracle_bit_exact(n, order):
    pf, cf, tets, p1 = _mesh(n, order)
    plan = _plan(p1, tets, order)
    ex = plan.export()
    idx, inverse, nse = oa.compress_plan(cf)
    indptr, indices = oa.plan_to_csr(idx, pf.shape[0])
    assert plan.n == pf.shape[0] and plan.nnz == nse
    assert np.array_equal(ex["cells"].cpu().numpy(), cf)
    assert np.array_equal(ex["indptr"].cpu().numpy(), indptr)
    assert np.array_equal(ex["indices"].cpu().numpy(), indices)
    assert np.array_equal(ex["slot"].cpu().numpy().reshape(-1), inverse)
    assert np.array_equal(ex["points"].cpu().numpy(), pf)
    bnd = om.boundary_nodes(cf, order)
    assert np.array_equal(np.flatnonzero(ex["dirichlet_mask"].cpu().numpy()), bnd)
    rows = np.repeat(np.arange(plan.n), np.diff(indptr))
    assert np.array_equal(ex["diag_slot"].cpu().numpy(), np.flatnonzero(rows == indices))


def test_plan_golden_reference_fixture(golden):
    """The device plan reproduces the reference-generated fixture directly (4x4x4, P1 and P2)."""
    tag = "4x4x4"
    plan1 = _plan(golden[f"{tag}/jittered"], golden[f"{tag}/tets"], 1)
    ex = plan1.export()
    idx = golden[f"{tag}/p1_idx"]
    assert np.array_equal(ex["indices"].cpu().numpy(), idx[:, 1])
    assert np.array_equal(ex["slot"].cpu().numpy().reshape(-1), golden[f"{tag}/p1_inverse"])
    plan2 = _plan(golden[f"{tag}/jittered"], golden[f"{tag}/tets"], 2)
    ex2 = plan2.export()
    assert np.array_equal(ex2["cells"].cpu().numpy(), golden[f"{tag}/p2_cells"])
    assert np.array_equal(ex2["points"].cpu().numpy(), golden[f"{tag}/p2_points"])
    assert np.array_equal(ex2["slot"].cpu().numpy().reshape(-1), golden[f"{tag}/p2_inverse"])
    assert np.array_equal(np.flatnonzero(ex2["dirichlet_mask"].cpu().numpy()), golden[f"{tag}/p2_boundary"])


@pytest.mark.parametrize("n,order", [(3, 1), (8, 1), (16, 1), (3, 2), (6, 2)])
def test_assembly_matches_oracle(n, order):
    pf, cf, tets, p1 = _mesh(n, order, seed=1)
    logk = om.logk_field(len(tets), 1000)
    plan = _plan(p1, tets, order)
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    s, _ = _oracle_system(pf, cf, order, logk)
    v = vals.cpu().numpy()
    assert np.abs(v - s.data).max() <= VAL_TOL * np.abs(s.data).max()
    assert np.abs(b.cpu().numpy() - s.b).max() <= VAL_TOL * np.abs(s.b).max()
    # Dirichlet entries are explicit zeros, diagonal exactly 1
    assert np.array_equal(v == 0.0, s.data == 0.0)
    kh, fh = plan.element_matrices()
    K, F = oe.element_matrices(p1[tets], order)
    assert np.abs(kh.cpu().numpy() - K).max() <= VAL_TOL * np.abs(K).max()
    assert np.abs(fh.cpu().numpy() - F).max() <= VAL_TOL * np.abs(F).max()


@pytest.mark.parametrize("order", [1, 2])
def test_inhomogeneous_dirichlet_patch(order):
    """P1 reproduces a linear field, P2 a quadratic one (tests/test_fem_3d.py:76-89,
    tests/test_fem_native_lagrange.py:377-395), through the CUDA assembly and CG."""
    n = 4
    pf, cf, tets, p1 = _mesh(n, order, seed=3)
    x, y, z = pf.T
    if order == 1:
        exact, f = 1 + 2 * x + 3 * y + 4 * z, 0.0
    else:
        exact, f = x**2 + 2 * y**2 + 3 * z**2 + x * y, -12.0
    plan = _plan(p1, tets, order)
    g = torch.as_tensor(exact, device="cuda")
    vals, b = plan.assemble(None, mode=2, scale=1.0, f=f, g=g)
    s, _ = _oracle_system(pf, cf, order, np.zeros(len(tets)), f=f, g=exact)
    assert np.abs(vals.cpu().numpy() - s.data).max() <= VAL_TOL * np.abs(s.data).max()
    assert np.abs(b.cpu().numpy() - s.b).max() <= 1e-11 * np.abs(s.b).max()
    inv = plan.jacobi(vals)
    u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-13)
    assert np.abs(u.cpu().numpy() - exact).max() < 1e-9


@pytest.mark.parametrize("n,order", [(8, 1), (24, 1), (4, 2), (8, 2)])
def test_pcg_matches_oracle(n, order):
    pf, cf, tets, p1 = _mesh(n, order)
    logk = om.logk_field(len(tets), 1000)
    plan = _plan(p1, tets, order)
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    inv = plan.jacobi(vals)
    u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
    s, _ = _oracle_system(pf, cf, order, logk)
    A = s.csr()
    xo, ito, hist = op.pcg(A, s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8)
    assert st == 0
    assert abs(it - ito) <= 1, (it, ito)
    uu = u.cpu().numpy()
    assert np.linalg.norm(uu - xo) <= 1e-7 * np.linalg.norm(xo)
    assert rel <= 2e-8 and abs(rel - op.residual_check(A, s.b, uu)) <= 1e-12
    # inverse diagonal matches the reference's materialize
    assert np.abs(inv.cpu().numpy() - oa.jacobi_inverse(oa.matrix_diagonal(s))).max() <= 1e-12 * np.abs(
        oa.jacobi_inverse(oa.matrix_diagonal(s))).max()


def test_spmv_and_matrix_free_match():
    for n, order in ((8, 1), (4, 2)):
        pf, cf, tets, p1 = _mesh(n, order, seed=2)
        logk = om.logk_field(len(tets), 7)
        plan = _plan(p1, tets, order)
        lk = torch.as_tensor(logk, device="cuda")
        vals, b = plan.assemble(lk)
        xv = torch.as_tensor(np.random.default_rng(0).standard_normal(plan.n), device="cuda")
        y1 = plan.spmv(vals, xv).cpu().numpy()
        s, _ = _oracle_system(pf, cf, order, logk)
        yo = s.csr() @ xv.cpu().numpy()
        assert np.abs(y1 - yo).max() <= 1e-12 * np.abs(yo).max()
        y2 = plan.spmv_matfree(lk, xv).cpu().numpy()
        assert np.abs(y2 - yo).max() <= 1e-12 * np.abs(yo).max()
        inv = plan.jacobi(vals)
        inv_mf = plan.jacobi_matfree(lk)
        assert np.abs(inv.cpu().numpy() - inv_mf.cpu().numpy()).max() <= 1e-12 * inv.abs().max().item()
        u1, it1, _, _ = plan.pcg(vals, b, inv_diag=inv)
        u2, it2, rel2, _ = plan.pcg_matfree(lk, b, inv_diag=inv_mf)
        assert abs(it1 - it2) <= 1 and rel2 <= 2e-8
        assert torch.linalg.norm(u1 - u2) <= 1e-7 * torch.linalg.norm(u1)


def test_matrix_free_p1_kuhn_blocks_and_per_element():
    """The P1 matrix-free operator works a hexahedron a thread when the elements come in Kuhn blocks
    (the box constructor's order) and an element a thread otherwise (here the first two tetrahedra of
    every block swapped, so the plan's block check fails). Both products match the assembled
    operator, and so do the solves."""
    pf, cf, tets, p1 = _mesh(8, 1, seed=2)
    logk = om.logk_field(len(tets), 7)
    perm = np.arange(len(tets)).reshape(-1, 6)
    perm[:, [0, 1]] = perm[:, [1, 0]]
    perm = perm.ravel()
    xv = torch.as_tensor(np.random.default_rng(3).standard_normal(len(p1)), device="cuda")
    sols = []
    for t, lk in ((tets, logk), (tets[perm], logk[perm])):
        plan = _plan(p1, t, 1)
        lkd = torch.as_tensor(lk, device="cuda")
        vals, b = plan.assemble(lkd)
        y_asm = plan.spmv(vals, xv)
        y_mf = plan.spmv_matfree(lkd, xv)
        assert (y_mf - y_asm).abs().max().item() <= 1e-12 * y_asm.abs().max().item()
        u, it, rel, st = plan.pcg_matfree(lkd, b, inv_diag=plan.jacobi_matfree(lkd))
        assert st == 0 and rel <= 2e-8
        sols.append(u)
    assert torch.linalg.norm(sols[0] - sols[1]) <= 1e-7 * torch.linalg.norm(sols[0])


@pytest.mark.parametrize("mode", [0, 1])
def test_mixed_precision_reaches_fp64_accuracy(mode):
    pf, cf, tets, p1 = _mesh(16, 1)
    logk = om.logk_field(len(tets), 1001)
    plan = _plan(p1, tets, 1)
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    inv = plan.jacobi(vals)
    u64, it64, rel64, _ = plan.pcg(vals, b, inv_diag=inv, tol=1e-12)
    u, inner, outer, rel, st = plan.pcg_mixed(vals, b, inv, tol=1e-8, mode=mode)
    assert st == 0 and rel <= 1e-8 and outer >= 2
    # true FP64 residual of the returned x
    r = b - plan.spmv(vals, u)
    assert (torch.linalg.norm(r) / torch.linalg.norm(b)).item() <= 1e-8
    assert (torch.linalg.norm(u - u64) / torch.linalg.norm(u64)).item() <= 1e-7


def test_adjoint_gradient_matches_oracle_and_fd():
    n = 6
    pf, cf, tets, p1 = _mesh(n, 1)
    logk = om.logk_field(len(tets), 1002)
    ustar_logk = om.logk_field(len(tets), 2000)
    bnd = om.boundary_nodes(cf, 1)
    ustar, _, _ = oadj.solve(pf, cf, 1, bnd, ustar_logk)
    mass = oadj.lumped_mass(pf, cf, 1)
    J_o, g_o = oadj.gradient(pf, cf, 1, bnd, logk, ustar, mass)

    from jno_b200.autograd import solve_p0

    plan = _plan(p1, tets, 1)
    m = plan.lumped_mass()
    assert np.abs(m.cpu().numpy() - mass).max() <= 1e-13 * mass.max()
    us = torch.as_tensor(ustar, device="cuda")
    lk = torch.as_tensor(logk, device="cuda").requires_grad_(True)
    u = solve_p0(plan, lk, tol=1e-13)
    J = 0.5 * torch.sum(m * (u - us) ** 2)
    J.backward()
    g = lk.grad.cpu().numpy()
    assert abs(J.item() - J_o) <= 1e-10 * abs(J_o)
    assert np.abs(g - g_o).max() <= 1e-8 * np.abs(g_o).max()

    def Jof(v):
        with torch.no_grad():
            uu = solve_p0(plan, torch.as_tensor(v, device="cuda"), tol=1e-14)
            return (0.5 * torch.sum(m * (uu - us) ** 2)).item()

    rng = np.random.default_rng(5)
    for c in rng.choice(len(tets), 8, replace=False):
        e = np.zeros(len(tets))
        e[c] = 1e-6
        fd = (Jof(logk + e) - Jof(logk - e)) / 2e-6
        assert abs(fd - g[c]) <= 1e-6 * np.abs(g).max() + 1e-6 * abs(g[c])


def test_status_paths_do_not_fault():
    pf, cf, tets, p1 = _mesh(4, 1)
    plan = _plan(p1, tets, 1)
    lk = torch.zeros(len(tets), dtype=torch.float64, device="cuda")
    vals, b = plan.assemble(lk)
    inv = plan.jacobi(vals)
    # iteration cap -> NOT_CONVERGED status, x written
    u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, maxiter=1)
    assert st == 4 and it == 1 and rel > 1e-8
    # zero right-hand side -> no iteration
    u, it, rel, st = plan.pcg(vals, torch.zeros_like(b), inv_diag=inv)
    assert it == 0 and st == 0 and torch.all(u == 0)
    # negative definite operator -> breakdown reported, no fault
    from jno_b200._lib import FemkError

    vneg, bneg = plan.assemble(-torch.ones(len(tets), dtype=torch.float64, device="cuda"), mode=1)
    with pytest.raises(FemkError):
        plan.pcg(vneg, bneg, inv_diag=None)
    # out-of-range or degenerate connectivity is rejected on the host before any GPU work
    bad = tets.copy()
    bad[3, 2] = 10**6
    with pytest.raises(ValueError):
        _plan(p1, bad, 1)
    bad = tets.copy()
    bad[3, 2] = bad[3, 1]
    with pytest.raises(ValueError):
        _plan(p1, bad, 1)
    # the guard of _maybe_residual_check raises on a non-solution
    import jno_b200 as jno
    from jno_b200.sparse import CsrMatrix

    A = CsrMatrix(plan, vals)
    with pytest.raises(RuntimeError, match="did not solve"):
        jno.solve.cg(maxiter=1)(A, b, M=jno.precond.jacobi())


def test_jno_surface_end_to_end():
    """The reference recipe (tests/test_topology_optimisation.py:176-195 shape) on the B200 path."""
    import jno_b200 as jno

    n = 8
    d = jno.domain(jno.domain.equi_distant_box(nx=n, ny=n, nz=n), jitter=0.1, seed=0)
    u, v = d.fem_symbols()
    _r, s = d.fem_symbols(space="P0", names=("r", "s"))
    xi, yi, zi = d.variable("interior", split=True)
    xb, yb, zb = d.variable("boundary", split=True)
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    logk = jno.np.parameter(s, name="logk")
    fem = jno.fem([jno.np.exp(logk) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi, u(xb, yb, zb) - 0.0])
    assert fem.problem is None and fem.dofs == (n + 1) ** 3
    lk = om.logk_field(6 * n**3, 1000)
    A, b = fem.operator.evaluate({"logk": lk})
    x = jno.solve.cg(tol=1e-8)(A, b, M=jno.precond.jacobi())
    pf, cf, tets, p1 = _mesh(n, 1)
    so, _ = _oracle_system(pf, cf, 1, lk)
    xo = op.pcg(so.csr(), so.b, oa.jacobi_inverse(oa.matrix_diagonal(so)))[0]
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)
    idx, data = A.to_bcoo(appended=True)
    assert idx.shape[0] == A.nnz + plan_dirichlet(fem)
    xm = jno.solve.cg(tol=1e-8, precision="mixed")(A, b, M=jno.precond.jacobi())
    assert np.linalg.norm(xm.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)
    Amf, bmf = fem.matrix_free({"logk": lk})
    xf = jno.solve.cg(tol=1e-8)(Amf, bmf, M=jno.precond.jacobi())
    assert np.linalg.norm(xf.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)


def plan_dirichlet(fem):
    return fem.plan.n_dirichlet


def test_profiled_solve_matches_and_times_every_iteration():
    pf, cf, tets, p1 = _mesh(12, 1)
    logk = om.logk_field(len(tets), 1003)
    plan = _plan(p1, tets, 1)
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    inv = plan.jacobi(vals)
    u0, it0, _, _ = plan.pcg(vals, b, inv_diag=inv)
    plan.set_profiling(True)
    u1, it1, _, _ = plan.pcg(vals, b, inv_diag=inv)
    step, upd, pup, iters = plan.profile()
    plan.set_profiling(False)
    assert it1 == it0 and iters == it1
    assert torch.equal(u0, u1)  # same kernels, same order: bit-identical with or without graph replay
    assert step > 0 and upd > 0 and pup > 0


@pytest.mark.parametrize("n,order,jitter", [(3, 1, True), (8, 1, True), (6, 1, False), (3, 2, True), (4, 2, False)])
def test_compact_export_matches_compress_eager(n, order, jitter):
    """femk_compact keeps exactly the entries compress_eager keeps (|v| > 0, plan order)."""
    pf, cf, tets, p1 = om.kuhn_cube(n, order=order, seed=4, amp=0.1 if jitter else 0.0)
    logk = om.logk_field(len(tets), 1004)
    plan = _plan(p1, tets, order)
    x, y, z = pf.T
    g = 1.0 + x - 2.0 * y + 0.5 * z
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"), g=torch.as_tensor(g, device="cuda"))
    ip, ind, dat = plan.compact(vals)
    ex = plan.export()
    # selection rule, bit-exact, on the same (device-assembled) values
    ipo, indo, dato = oa.compact_csr(ex["indptr"].cpu().numpy(), ex["indices"].cpu().numpy(), vals.cpu().numpy())
    assert np.array_equal(ip.cpu().numpy(), ipo)
    assert np.array_equal(ind.cpu().numpy(), indo)
    assert np.array_equal(dat.cpu().numpy(), dato)
    assert ind.numel() < plan.nnz  # the Dirichlet rows/columns always go
    # against the oracle's own assembly: same kept pattern on jittered meshes, values within 1e-12
    s, _ = _oracle_system(pf, cf, order, logk, g=g)
    B = oa.compact(s)
    if jitter:
        assert np.array_equal(ip.cpu().numpy(), B.indptr) and np.array_equal(ind.cpu().numpy(), B.indices)
        assert np.abs(dat.cpu().numpy() - B.data).max() <= VAL_TOL * np.abs(B.data).max()
    A = B.toarray()
    D = np.zeros((plan.n, plan.n))
    rows = np.repeat(np.arange(plan.n), np.diff(ip.cpu().numpy()))
    D[rows, ind.cpu().numpy()] = dat.cpu().numpy()
    assert np.abs(D - A).max() <= VAL_TOL * np.abs(A).max()


def test_compact_export_drops_nan_and_signed_zero_and_checks_capacity():
    import ctypes

    from jno_b200 import _lib

    pf, cf, tets, p1 = _mesh(3, 1)
    plan = _plan(p1, tets, 1)
    vals, b = plan.assemble(torch.zeros(len(tets), dtype=torch.float64, device="cuda"))
    ex = plan.export()
    planted = vals.clone()
    nz = torch.nonzero(planted != 0).flatten()
    planted[nz[5]] = float("nan")
    planted[nz[9]] = -0.0
    planted[nz[11]] = float("inf")  # |inf| > 0: kept
    ip, ind, dat = plan.compact(planted)
    ipo, indo, dato = oa.compact_csr(ex["indptr"].cpu().numpy(), ex["indices"].cpu().numpy(), planted.cpu().numpy())
    assert np.array_equal(ip.cpu().numpy(), ipo) and np.array_equal(ind.cpu().numpy(), indo)
    assert np.array_equal(dat.cpu().numpy(), dato)
    assert ind.numel() == nz.numel() - 2
    # a capacity below the kept count is refused before any entry is written
    lib = _lib.load()
    out_ptr = torch.full((plan.n + 1,), -7, dtype=torch.int32, device="cuda")
    out_idx = torch.full((8,), -7, dtype=torch.int32, device="cuda")
    out_val = torch.full((8,), -7.0, dtype=torch.float64, device="cuda")
    m = ctypes.c_int64(-1)
    st = lib.femk_compact(plan.handle, _lib.ptr(vals), _lib.ptr(out_ptr), _lib.ptr(out_idx), _lib.ptr(out_val), 8,
                          ctypes.byref(m), _lib.stream_handle())
    torch.cuda.synchronize()
    assert st == _lib.FEMK_EINVAL and b"cap" in lib.femk_last_error_string()
    assert torch.all(out_idx == -7) and torch.all(out_val == -7.0)


def test_jno_surface_non_parametric_route():
    """A form without a parameter: (A, b) with A compacted, inhomogeneous Dirichlet lifted into b
    (jno/utils/solver/fem_native.py:3371-3379), solved through fem.solve()."""
    import jno_b200 as jno

    n = 6
    d = jno.domain(jno.domain.equi_distant_box(nx=n, ny=n, nz=n), jitter=0.1, seed=0)
    u, v = d.fem_symbols()
    xi, yi, zi = d.variable("interior", split=True)
    xb, yb, zb = d.variable("boundary", split=True)
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    fem = jno.fem([2.0 * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi,
                   u(xb, yb, zb) - (1.0 + xb + 2.0 * yb - zb)])
    A, b = fem.operator
    pf, cf, tets, p1 = _mesh(n, 1)
    g = 1.0 + pf[:, 0] + 2.0 * pf[:, 1] - pf[:, 2]
    bnd = om.boundary_nodes(cf, 1)
    so = oa.assemble(pf, cf, 1, bnd, np.full(len(tets), 2.0), f=1.0, g=g)
    B = oa.compact(so)
    assert A.nnz == B.nnz
    assert np.array_equal(A.indptr.cpu().numpy(), B.indptr) and np.array_equal(A.indices.cpu().numpy(), B.indices)
    assert np.abs(A.data.cpu().numpy() - B.data).max() <= VAL_TOL * np.abs(B.data).max()
    assert np.abs(b.cpu().numpy() - so.b).max() <= 1e-11 * np.abs(so.b).max()
    idx, data = A.to_bcoo()
    assert idx.shape == (B.nnz, 2)
    xs = fem.solve()  # the reference's steady default: Jacobi-BiCGStab
    xo = op.bicgstab(B, so.b, oa.jacobi_inverse(oa.matrix_diagonal(so)), tol=1e-8)[0]
    assert np.linalg.norm(xs.cpu().numpy() - xo) <= 1e-7 * np.linalg.norm(xo)
    assert np.abs(xs.cpu().numpy()[bnd] - g[bnd]).max() <= 1e-7 * np.abs(g).max()
    yv = torch.as_tensor(np.random.default_rng(1).standard_normal(plan_n(fem)), device="cuda")
    assert np.abs((A @ yv).cpu().numpy() - B @ yv.cpu().numpy()).max() <= 1e-12 * np.abs(B @ yv.cpu().numpy()).max()


def plan_n(fem):
    return fem.plan.n


@pytest.mark.parametrize("n,order,bulk", [(8, 1, True), (8, 1, False), (24, 1, True), (4, 2, True)])
def test_bicgstab_matches_oracle(n, order, bulk):
    """femk_bicgstab against the oracle's restatement of jax.scipy.sparse.linalg.bicgstab (bulk-copy
    SpMV ring, and the thread-per-row kernel with ring64 = 0)."""
    pf, cf, tets, p1 = _mesh(n, order)
    logk = om.logk_field(len(tets), 1005)
    plan = _plan(p1, tets, order, None if bulk else {"ring64": 0})
    vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
    inv = plan.jacobi(vals)
    u, it, rel, st = plan.bicgstab(vals, b, inv_diag=inv, tol=1e-8)
    s, _ = _oracle_system(pf, cf, order, logk)
    A = s.csr()
    xo, ko = op.bicgstab(A, s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8)
    assert st == 0 and ko > 0
    # BiCGStab's iteration count moves with the summation order of its dot products (the grid shape
    # of the reductions); the contract is the stop rule and the solution
    assert abs(it - ko) <= max(2, ko // 10), (it, ko)
    uu = u.cpu().numpy()
    assert np.linalg.norm(uu - xo) <= 1e-7 * np.linalg.norm(xo)
    assert abs(rel - op.residual_check(A, s.b, uu)) <= 1e-12
    # a second solve from the first solution's neighbourhood reuses the captured graph
    u2, it2, rel2, st2 = plan.bicgstab(vals, b, inv_diag=inv, tol=1e-8)
    assert st2 == 0 and it2 == it and torch.equal(u2, u)
    # no preconditioner, through the jno surface
    import jno_b200 as jno
    from jno_b200.sparse import CsrMatrix

    xn = jno.solve.bicgstab(tol=1e-8)(CsrMatrix(plan, vals), b)
    xon, _ = op.bicgstab(A, s.b, None, tol=1e-8)
    assert np.linalg.norm(xn.cpu().numpy() - xon) <= 1e-7 * np.linalg.norm(xon)


def test_bicgstab_status_paths():
    pf, cf, tets, p1 = _mesh(4, 1)
    plan = _plan(p1, tets, 1)
    vals, b = plan.assemble(torch.zeros(len(tets), dtype=torch.float64, device="cuda"))
    inv = plan.jacobi(vals)
    u, it, rel, st = plan.bicgstab(vals, b, inv_diag=inv, maxiter=1)
    assert st == 4 and it == 1  # iteration cap: NOT_CONVERGED, x written
    u, it, rel, st = plan.bicgstab(vals, torch.zeros_like(b), inv_diag=inv)
    assert st == 0 and it == 0 and torch.all(u == 0)
    import jno_b200 as jno
    from jno_b200.sparse import CsrMatrix

    with pytest.raises(RuntimeError, match="jno.solve.bicgstab did not solve"):
        jno.solve.bicgstab(maxiter=1)(CsrMatrix(plan, vals), b, M=jno.precond.jacobi())


def test_spmv_layouts_agree():
    """The CG-step SpMV has three layouts: bulk-copy slices with per-slice column tables (the
    default), bulk-copy slices with per-entry columns (column_tables = 0), and the thread-per-row
    kernel (ring64 = ring32 = 0), here also on int32 columns (cols16 = 0: the FP64 form keeps 32
    entries in flight, as on P2 plans). All sum each row in the same order; the two bulk forms (same
    grid, same reductions) give bit-identical solves, the thread-per-row forms agree to rounding of
    their dot products (other grids). 64^3 hexes: z-lines of 65 rows, so about half the 32-row
    slices share one offset sequence."""
    pf, cf, tets, p1 = _mesh(64, 1)
    lk = torch.as_tensor(om.logk_field(len(tets), 1006), device="cuda")
    out = {}
    vals = b = inv = None
    for tag, opts in (("table", None), ("entry", {"column_tables": 0}), ("thread", {"ring64": 0, "ring32": 0}),
                      ("int32", {"cols16": 0, "ring64": 0, "ring32": 0})):
        plan = _plan(p1, tets, 1, opts)
        if tag == "entry":
            assert plan.sell_col_units == plan.sell_nnz
        elif tag != "int32":  # (info.cols16 is the mesh's property; the option switches the FP64 stream)
            assert plan.sell_col_units < 0.7 * plan.sell_nnz
        if vals is None:
            vals, b = plan.assemble(lk)
            inv = plan.jacobi(vals)
        u, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
        um, inner, outer, relm, stm = plan.pcg_mixed(vals, b, inv, tol=1e-8)
        ub, itb, relb, stb = plan.bicgstab(vals, b, inv_diag=inv, tol=1e-8)
        assert st == 0 and stm == 0 and stb == 0 and rel <= 2e-8 and relm <= 1e-8 and relb <= 2e-8
        out[tag] = (u, it, um, inner, ub, itb)
    a, c, e, w = out["thread"], out["table"], out["entry"], out["int32"]
    assert c[1] == e[1] and torch.equal(c[0], e[0])
    assert c[3] == e[3] and torch.equal(c[2], e[2])
    assert c[5] == e[5] and torch.equal(c[4], e[4])
    assert abs(a[1] - c[1]) <= 1 and (torch.linalg.norm(a[0] - c[0]) / torch.linalg.norm(c[0])).item() <= 1e-9
    assert abs(a[3] - c[3]) <= 10 and (torch.linalg.norm(a[2] - c[2]) / torch.linalg.norm(c[2])).item() <= 1e-7
    assert abs(w[1] - a[1]) <= 1 and (torch.linalg.norm(w[0] - a[0]) / torch.linalg.norm(a[0])).item() <= 1e-9
    assert abs(w[3] - a[3]) <= 10 and (torch.linalg.norm(w[2] - a[2]) / torch.linalg.norm(a[2])).item() <= 1e-7


def test_canonical_csr_solver_path_matches():
    """A plan without the sliced-ELL operator (the path taken when the sliced-ELL entry count passes
    2^31; chosen here with the solver_layout = 0 plan option) runs FP64 PCG and the mixed solver on
    the canonical-CSR kernels. Its row sums are lane-split shuffle reductions, so it agrees with the
    sliced-ELL plan to rounding, and both meet the oracle's solution."""
    pf, cf, tets, p1 = _mesh(32, 1)
    lk = torch.as_tensor(om.logk_field(len(tets), 1007), device="cuda")
    sell = _plan(p1, tets, 1)
    vals, b = sell.assemble(lk)
    inv = sell.jacobi(vals)
    u, it, rel, st = sell.pcg(vals, b, inv_diag=inv, tol=1e-8)
    um, inner, _, relm, stm = sell.pcg_mixed(vals, b, inv, tol=1e-8)
    csr = _plan(p1, tets, 1, {"solver_layout": 0})
    uc, itc, relc, stc = csr.pcg(vals, b, inv_diag=inv, tol=1e-8)
    umc, innerc, _, relmc, stmc = csr.pcg_mixed(vals, b, inv, tol=1e-8)
    assert st == stm == stc == stmc == 0
    assert relc <= 2e-8 and relmc <= 1e-8
    assert abs(itc - it) <= 2 and abs(innerc - inner) <= 10
    ref = torch.linalg.norm(u)
    assert (torch.linalg.norm(uc - u) / ref).item() <= 1e-8
    assert (torch.linalg.norm(umc - um) / ref).item() <= 1e-7
    import scipy.sparse.linalg as spla

    s = oa.assemble(pf, cf, 1, om.boundary_nodes(cf, 1), np.exp(lk.cpu().numpy()))
    x_ref = spla.spsolve(s.csr().tocsc(), s.b)
    assert np.linalg.norm(uc.cpu().numpy() - x_ref) <= 1e-6 * np.linalg.norm(x_ref)
    from jno_b200._lib import FemkError

    with pytest.raises(FemkError, match="sliced-ELL"):
        csr.bicgstab(vals, b, inv_diag=inv, tol=1e-8)


@pytest.mark.parametrize("mode", ["exp", "linear"])
def test_nodal_p1_parameter_matches_oracle(mode):
    """A nodal P1 coefficient (jno.np.parameter of a P1 symbol) through assembly, the matrix-free
    operator and the jno surface."""
    from jno_b200 import _lib

    n = 6
    pf, cf, tets, p1 = _mesh(n, 1)
    rng = np.random.default_rng(11)
    nodal = rng.normal(0.0, 0.5, p1.shape[0]) if mode == "exp" else rng.uniform(0.5, 2.0, p1.shape[0])
    cmode = _lib.COEF_NODAL_EXP if mode == "exp" else _lib.COEF_NODAL_LINEAR
    plan = _plan(p1, tets, 1)
    pv = torch.as_tensor(nodal, device="cuda")
    vals, b = plan.assemble(pv, mode=cmode)
    ke = oe.nodal_coefficient(tets, nodal, mode)
    bnd = om.boundary_nodes(cf, 1)
    s = oa.assemble(pf, cf, 1, bnd, ke)
    assert np.abs(vals.cpu().numpy() - s.data).max() <= VAL_TOL * np.abs(s.data).max()
    xv = torch.as_tensor(rng.standard_normal(plan.n), device="cuda")
    ym = plan.spmv_matfree(pv, xv, mode=cmode).cpu().numpy()
    yo = s.csr() @ xv.cpu().numpy()
    assert np.abs(ym - yo).max() <= 1e-12 * np.abs(yo).max()
    # the jno surface: parameter(<P1 symbol>) is nodal
    import jno_b200 as jno

    d = jno.domain(jno.domain.equi_distant_box(nx=n, ny=n, nz=n), jitter=0.1, seed=0)
    u, v = d.fem_symbols()
    kf, _ = d.fem_symbols(names=("k", "kt"))
    xi, yi, zi = d.variable("interior", split=True)
    xb, yb, zb = d.variable("boundary", split=True)
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    k = jno.np.parameter(kf, name="k")
    coef = jno.np.exp(k) if mode == "exp" else k
    fem = jno.fem([coef * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi, u(xb, yb, zb) - 0.0])
    A, bb = fem.operator.evaluate({"k": nodal})
    x = jno.solve.cg(tol=1e-10)(A, bb, M=jno.precond.jacobi())
    xo = op.pcg(s.csr(), s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-10)[0]
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-8 * np.linalg.norm(xo)
    with pytest.raises(ValueError):
        fem.operator.evaluate({"k": np.zeros(len(tets))})  # P0-sized input for a nodal parameter


@pytest.mark.parametrize("mode", ["exp", "linear"])
def test_nodal_adjoint_matches_oracle_and_fd(mode):
    """dJ/dp for a nodal P1 parameter: oracle chain rule (1e-8) and central differences."""
    from jno_b200 import _lib
    from jno_b200.autograd import solve_nodal

    n = 5
    pf, cf, tets, p1 = _mesh(n, 1)
    rng = np.random.default_rng(13)
    vals = rng.normal(0.0, 0.4, p1.shape[0]) if mode == "exp" else rng.uniform(0.5, 2.0, p1.shape[0])
    cmode = _lib.COEF_NODAL_EXP if mode == "exp" else _lib.COEF_NODAL_LINEAR
    bnd = om.boundary_nodes(cf, 1)
    ustar, _, _ = oadj.solve(pf, cf, 1, bnd, om.logk_field(len(tets), 2001))
    mass = oadj.lumped_mass(pf, cf, 1)
    J_o, g_o = oadj.gradient_nodal(pf, cf, bnd, vals, mode, ustar, mass)
    plan = _plan(p1, tets, 1)
    m = plan.lumped_mass()
    us = torch.as_tensor(ustar, device="cuda")
    pv = torch.as_tensor(vals, device="cuda").requires_grad_(True)
    u = solve_nodal(plan, pv, cmode, tol=1e-13)
    J = 0.5 * torch.sum(m * (u - us) ** 2)
    J.backward()
    g = pv.grad.cpu().numpy()
    assert abs(J.item() - J_o) <= 1e-10 * abs(J_o)
    assert np.abs(g - g_o).max() <= 1e-8 * np.abs(g_o).max()

    def Jof(v):
        with torch.no_grad():
            uu = solve_nodal(plan, torch.as_tensor(v, device="cuda"), cmode, tol=1e-14)
            return (0.5 * torch.sum(m * (uu - us) ** 2)).item()

    interior = np.setdiff1d(np.arange(p1.shape[0]), bnd)
    for i in rng.choice(interior, 6, replace=False):
        e = np.zeros(p1.shape[0])
        e[i] = 1e-6
        fd = (Jof(vals + e) - Jof(vals - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * np.abs(g).max() + 1e-6 * abs(g[i])


def test_p2_surface_recovers_harmonic_quadratic():
    """Port of tests/test_fem_higher_order.py:133-150 onto the B200 path: P2 through jno.fem with
    u = xy + yz + xz on the boundary, f = 0, fem.solve() (Jacobi-BiCGStab) recovers it to 1e-9."""
    import jno_b200 as jno

    n = 3
    d = jno.domain(jno.domain.equi_distant_box(nx=n, ny=n, nz=n), jitter=0.1, seed=7)
    u, phi = d.fem_symbols(order=2)
    xi, yi, zi = d.variable("interior", split=True)
    cb = d.variable("boundary", split=True)
    ui, vi = u.bind(x=xi, y=yi, z=zi), phi.bind(x=xi, y=yi, z=zi)
    bc = u(cb[0], cb[1], cb[2]) - (cb[0] * cb[1] + cb[1] * cb[2] + cb[0] * cb[2])
    fem = jno.fem([ui.x * vi.x + ui.y * vi.y + ui.z * vi.z, bc])
    assert fem.dofs > (n + 1) ** 3  # vertices + edge nodes
    pts = fem.points.cpu().numpy()
    sol = fem.solve(linear=jno.solve.bicgstab(tol=1e-12)).cpu().numpy()
    exact = pts[:, 0] * pts[:, 1] + pts[:, 1] * pts[:, 2] + pts[:, 0] * pts[:, 2]
    assert np.linalg.norm(exact - sol) / np.linalg.norm(exact) < 1e-9


def test_p0_linearity_and_support_on_device():
    """Port of tests/test_topology_optimisation.py:210-237 onto the CUDA assembly: the operator is
    linear in the P0 values (sum of single-element assemblies) and an element's contribution stays
    on its own DOFs."""
    from jno_b200 import _lib

    n = 3
    pf, cf, tets, p1 = _mesh(n, 1)
    plan = _plan(p1, tets, 1)
    T = len(tets)
    ex = plan.export()
    dm = ex["dirichlet_mask"].cpu().numpy().astype(bool)
    ip, ind = ex["indptr"].cpu().numpy(), ex["indices"].cpu().numpy()
    rows = np.repeat(np.arange(plan.n), np.diff(ip))
    free = ~(dm[rows] | dm[ind])
    full, _ = plan.assemble(torch.ones(T, dtype=torch.float64, device="cuda"), mode=_lib.COEF_LINEAR)
    acc = torch.zeros_like(full)
    for j in range(T):
        e = torch.zeros(T, dtype=torch.float64, device="cuda")
        e[j] = 1.0
        vj, _ = plan.assemble(e, mode=_lib.COEF_LINEAR)
        acc += vj
        if j == 40:
            cell = set(tets[j].tolist())
            vjn = vj.cpu().numpy()
            off = np.array([(r not in cell or c not in cell) for r, c in zip(rows, ind)])
            assert np.abs(vjn[off & free]).max() == 0.0
    a, fl = acc.cpu().numpy(), full.cpu().numpy()
    assert np.abs(a[free] - fl[free]).max() <= 1e-12 * np.abs(fl).max()




@pytest.mark.parametrize("dim,n,order,opts", [(3, 12, 1, {}), (3, 12, 1, {"ring32": 0}),
                                              (3, 12, 1, {"solver_layout": 0}), (3, 4, 2, {}), (2, 64, 1, {})])
def test_mixed_single_reduction_loop(dim, n, order, opts):
    """The FP32 inner loop in single-reduction form on each of its SpMV kernels (bulk-copy ring,
    thread-per-row sliced ELL, canonical CSR; P2 rows wider than the ring; 2-D rows of 7): the FP64
    residual meets the 1e-8 stop rule, the solution agrees with a tight FP64 solve to 1e-7, the FP32
    iteration count is the oracle restatement's (oracle.pcg.mixed_pcg) within 10 % + 3, in both modes,
    and graph replay and direct launches of the same chunks give bit-identical iterates."""
    pf, cf, tets, p1 = _mesh(n, order) if dim == 3 else om.unit_square(n, order, seed=0)
    logk = om.logk_field(len(tets), 1011)
    s, _ = (_oracle_system(pf, cf, order, logk) if dim == 3 else
            (oa.assemble(pf, cf, order, om.boundary_nodes(cf, order, nv=3), np.exp(logk)), None))
    inv_o = oa.jacobi_inverse(oa.matrix_diagonal(s))
    sols = []
    vals = None
    for replay in (1, 0):
        plan = _plan(p1, tets, order, {**opts, "graph_replay": replay})
        if vals is None:  # one assembly for both plans (same pattern): FP64 atomics may round differently
            vals, b = plan.assemble(torch.as_tensor(logk, device="cuda"))
            inv = plan.jacobi(vals)
            ut, _, _, _ = plan.pcg(vals, b, inv_diag=inv, tol=1e-13)
        for mode in (0, 1):
            u, inner, outer, rel, st = plan.pcg_mixed(vals, b, inv, tol=1e-8, mode=mode)
            assert st == 0 and rel <= 1e-8 and outer >= 2
            r = b - plan.spmv(vals, u)
            assert (torch.linalg.norm(r) / torch.linalg.norm(b)).item() <= 1e-8
            assert (torch.linalg.norm(u - ut) / torch.linalg.norm(ut)).item() <= 1e-7
            # the device's reliable-update thresholds: 1e-4 (reliable), 1e-8 (restart); FP32 rounding
            # order alone moves the counts by several percent (the oracle's two arrangements differ so)
            _, ito, outo = op.mixed_pcg(s.csr(), s.b, inv_o, tol=1e-8, restart=mode == 1,
                                        delta2=1e-8 if mode == 1 else 1e-4)
            assert abs(inner - ito) <= 0.1 * ito + 3, (inner, ito)
            sols.append((mode, u, inner, outer))
    for (m0, u0, i0, o0), (m1, u1, i1, o1) in zip(sols[:2], sols[2:]):
        assert m0 == m1 and i0 == i1 and o0 == o1 and torch.equal(u0, u1)


@pytest.mark.parametrize("dim,n,order", [(3, 16, 1), (3, 6, 2), (2, 32, 1), (2, 12, 2)])
def test_assembly_is_bitwise_reproducible(dim, n, order):
    """The row-gather assembly adds each row's entries in one fixed order (its incidence list): two
    assemblies, and two plans of the same mesh, give the same bits for the values and the load; the
    load-only form (matrix-free use) gives the same load."""
    pf, cf, cells, p1 = om.kuhn_cube(n, order=order, seed=4) if dim == 3 else om.unit_square(n, order, seed=4)
    lk = torch.as_tensor(om.logk_field(len(cells), 1012), device="cuda")
    g = torch.as_tensor(np.cos(pf[:, 0]) + pf[:, 1], device="cuda")
    out = []
    for _ in range(2):
        plan = _plan(p1, cells, order)
        for _ in range(2):
            vals, b = plan.assemble(lk, g=g)
            out.append((vals, b))
        assert torch.equal(plan.load(lk, g=g), out[0][1])
    for vals, b in out[1:]:
        assert torch.equal(vals, out[0][0]) and torch.equal(b, out[0][1])
    s = oa.assemble(pf, cf, order, om.boundary_nodes(cf, order, nv=dim + 1), np.exp(lk.cpu().numpy()),
                    g=g.cpu().numpy())
    assert np.abs(out[0][0].cpu().numpy() - s.data).max() <= VAL_TOL * np.abs(s.data).max()
    assert np.abs(out[0][1].cpu().numpy() - s.b).max() <= VAL_TOL * np.abs(s.b).max()
