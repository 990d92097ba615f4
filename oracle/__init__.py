"""CPU oracle for the P1/P2 tetrahedral assembly -> Jacobi-PCG path (TEST INFRASTRUCTURE).

This package is a numpy/scipy FP64 restatement of jNO's algorithm for this path. It exists only to
check the CUDA product and to serve as the timed CPU baseline; it is imported by ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``
and by nothing else. The product (``jno_b200``) never imports it and has no CPU fallback.

Parity pinning
--------------
* Mesh construction, P2 node numbering, the boundary-facet node set and the compress-plan CSR
  pattern are pinned bit-exactly against fixtures produced by running the reference's own
  functions (``jno/domain/geometries.py:203-300``, ``jno/utils/solver/fem_utils.py:1979-2044`` and
  ``:4009-4057``, ``jno/_fem.py:2695``) on small meshes: ``tests/golden/make_golden.py``.
* Element matrices and the RHS follow ``jno/utils/solver/fem_native.py:1461-1497`` (affine map,
  ``meas = |det J|``, ``grad phi = dphi/dxi . J^-1``) with the weak form
  ``k * grad u . grad v - f * v``. The reference integrates with basix quadrature of degree 2 (P1)
  and 4 (P2); these integrands are polynomials of degree <= 2, so the closed forms used here are the
  same integrals (cross-checked against an independent Keast quadrature in the tests).
* The Jacobi-PCG loop restates ``jax.scipy.sparse.linalg.cg`` (jax 0.10.1, not vendored in the
  reference; called from ``jno/solve.py:191-206``). Its iterate-level output is not pinned by any
  reference test; converged solutions are (``tests/test_fem_solver_slots.py:68-80``).
"""
