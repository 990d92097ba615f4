"""The C/OpenMP CPU restatement (oracle/femcpu.c, the benchmark's CPU baseline, P1 and P2 tets)
against the numpy oracle: the same CSR pattern, values and load to 1e-12, the same jax-cg iteration to one step and
solution to 1e-10, with several threads (row ownership makes the assembly independent of the count)."""

import numpy as np
import pytest

from oracle import assemble as oa
from oracle import build_cpu
from oracle import mesh as om
from oracle import pcg as op


@pytest.mark.parametrize("n,order,threads", [(5, 1, 1), (8, 1, 4), (3, 2, 1), (4, 2, 4)])
def test_femcpu_matches_numpy_oracle(n, order, threads):
    pf, cf, tets, p1 = om.kuhn_cube(n, order=order, seed=3)
    logk = om.logk_field(len(tets), 1000)
    bnd = om.boundary_nodes(cf, order)
    cpu = build_cpu.FemCpu(p1, cf, bnd, threads=threads)
    idx, inverse, nse = oa.compress_plan(cf)
    indptr, indices = oa.plan_to_csr(idx, pf.shape[0])
    assert np.array_equal(cpu.indptr, indptr) and np.array_equal(cpu.indices, indices)
    vals, b = cpu.assemble(logk)
    s = oa.assemble(pf, cf, order, bnd, np.exp(logk))
    assert np.abs(vals - s.data).max() <= 1e-12 * np.abs(s.data).max()
    assert np.abs(b - s.b).max() <= 1e-12 * np.abs(s.b).max()
    inv = cpu.jacobi()
    inv_o = oa.jacobi_inverse(oa.matrix_diagonal(s))
    assert np.abs(inv - inv_o).max() <= 1e-12 * np.abs(inv_o).max()
    x, it, rel = cpu.pcg(1e-8)
    xo, ito, _ = op.pcg(s.csr(), s.b, inv_o, tol=1e-8)
    assert abs(it - ito) <= 1 and rel <= 2e-8
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
    v1 = vals.copy()
    cpu.assemble(logk)
    assert np.array_equal(cpu.vals, v1)  # deterministic
