"""Oracle: preconditioned CG with ``jax.scipy.sparse.linalg.cg`` semantics (test infrastructure).

``jno.solve.cg(tol=1e-8, atol=0.0, maxiter=20_000)`` (``jno/solve.py:191-206``) calls
``jax.scipy.sparse.linalg.cg(op.mv, b, x0, tol, atol, maxiter, M)`` from jax 0.10.1, a dependency
that is not vendored in the reference. Its published algorithm, restated here:

    x0 = 0 if None;  r = b - A x0;  z = M r;  p = z;  gamma = <r, z>
    bs = <b, b>;  atol2 = max(tol^2 * bs, atol^2)
    while (rs > atol2) and (k < maxiter):        # rs = <r, r> when M is given, else gamma
        q = A p;  alpha = gamma / <p, q>
        x += alpha p;  r -= alpha q;  z = M r
        gamma' = <r, z>;  beta = gamma' / gamma;  p = z + beta p;  gamma = gamma';  k += 1

The stop test uses the recurrence residual; the ``info`` output is discarded by jNO, which then
runs the eager residual guard ``_maybe_residual_check`` (``jno/utils/solver/solver_api.py:224-240``:
``||b - A x|| / (||b|| + 1e-30) > 1e-4`` raises).
"""

import numpy as np


def pcg(A, b, inv_diag=None, x0=None, tol=1e-8, atol=0.0, maxiter=20_000):
    """Returns (x, iterations, recurrence rs history list)."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)

    def M(v):
        return v if inv_diag is None else inv_diag * v

    r = b - A @ x
    z = M(r)
    p = z.copy()
    gamma = float(np.dot(r, z))
    atol2 = max(tol * tol * float(np.dot(b, b)), atol * atol)
    rs = gamma if inv_diag is None else float(np.dot(r, r))
    hist = [rs]
    k = 0
    while rs > atol2 and k < maxiter:
        q = A @ p
        alpha = gamma / float(np.dot(p, q))
        x += alpha * p
        r -= alpha * q
        z = M(r)
        gamma_new = float(np.dot(r, z))
        beta = gamma_new / gamma
        p = z + beta * p
        gamma = gamma_new
        rs = gamma if inv_diag is None else float(np.dot(r, r))
        hist.append(rs)
        k += 1
    return x, k, hist


def residual_check(A, b, x, rtol=1e-4):
    """Relative true residual; raises RuntimeError like ``_maybe_residual_check``."""
    rel = float(np.linalg.norm(b - A @ x) / (np.linalg.norm(b) + 1e-30))
    if not np.isfinite(rel) or rel > rtol:
        raise RuntimeError(f"jno.solve.cg did not solve the system (relative residual {rel:.1e})")
    return rel
