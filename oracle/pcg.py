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


def bicgstab(A, b, inv_diag=None, x0=None, tol=1e-8, atol=0.0, maxiter=20_000):
    """``jax.scipy.sparse.linalg.bicgstab`` (jax 0.10.1), called by ``jno.solve.bicgstab``
    (``jno/solve.py:209-213``) and by the ``fem.solve()`` steady default with the Jacobi
    preconditioner (``jno/_fem.py:110-116``). Its published algorithm, restated:

        r = b - A x0;  rhat = r;  rho = alpha = omega = 1;  p = q = r;  k = 0
        atol2 = max(tol^2 <b, b>, atol^2)
        while <r, r> > atol2 and k < maxiter and k >= 0:
            rho' = <rhat, r>;  beta = rho' / rho * alpha / omega
            p = r + beta (p - omega q);  phat = M p;  q = A phat
            alpha = rho' / <rhat, q>;  s = r - alpha q;  early = <s, s> < atol2
            shat = M s;  t = A shat;  omega = <t, s> / <t, t>
            x = x + alpha phat            if early else  x + (alpha phat + omega shat)
            r = s                         if early else  s - omega t
            k = -10 if rho' == 0 else (-11 if omega == 0 or alpha == 0 else k + 1);  rho = rho'

    Returns (x, k): k < 0 reports a breakdown (the loop ends there, x as it stands).
    """
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)

    def M(v):
        return v if inv_diag is None else inv_diag * v

    r = b - A @ x
    rhat = r.copy()
    p = r.copy()
    q = r.copy()
    rho = alpha = omega = 1.0
    atol2 = max(tol * tol * float(np.dot(b, b)), atol * atol)
    k = 0
    while float(np.dot(r, r)) > atol2 and k < maxiter and k >= 0:
        rho_ = float(np.dot(rhat, r))
        with np.errstate(divide="ignore", invalid="ignore"):
            beta = float(np.float64(rho_) / rho * alpha / omega)
        p = r + beta * (p - omega * q)
        phat = M(p)
        q = A @ phat
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha = float(np.float64(rho_) / np.dot(rhat, q))
        s = r - alpha * q
        early = float(np.dot(s, s)) < atol2
        shat = M(s)
        t = A @ shat
        with np.errstate(divide="ignore", invalid="ignore"):
            omega = float(np.dot(t, s) / np.dot(t, t))
        if early:
            x = x + alpha * phat
            r = s
        else:
            x = x + (alpha * phat + omega * shat)
            r = s - omega * t
        if rho_ == 0.0:
            k = -10
        elif omega == 0.0 or alpha == 0.0:
            k = -11
        else:
            k += 1
        rho = rho_
    return x, k


def _safe_normalize(v, thresh=None):
    """(v / ||v||, ||v||), or (0, 0) when ||v|| <= thresh (default: machine epsilon, absolute)."""
    nrm = float(np.linalg.norm(v))
    t = np.finfo(np.float64).eps if thresh is None else thresh
    if nrm > t:
        return v / nrm, nrm
    return np.zeros_like(v), 0.0


def gmres(A, b, inv_diag=None, x0=None, tol=1e-8, atol=0.0, restart=20, maxiter=None):
    """``jax.scipy.sparse.linalg.gmres`` with ``solve_method="batched"`` (jax 0.10.1), called by
    ``jno.solve.gmres`` (``jno/solve.py:216-221``, default ``restart=30``) and by the rescue of a
    failed theta step (``jno/utils/solver/backend_blocks.py:402-413``: ``restart=min(n, 40)``,
    ``tol=max(1e-10, 100 eps)``). Its published algorithm, restated (M = the preconditioner):

        m = min(restart, n);  maxiter = 10 n if None
        atol' = max(tol ||b||, atol);  ptol = ||M b|| min(1, atol' / ||b||)
        w, beta = normalize(M (b - A x0));  k = 0
        while beta > ptol and k < maxiter:                      # one restart cycle per pass
            V[:, 0] = w;  H = eye(m, m + 1)                   # row j of H = column j of the Hessenberg
            for j in 0 .. m-1 (until breakdown):
                v = M A V[:, j];  v0 = ||v||
                one classical Gram-Schmidt pass of v against V: h = V^T v;  v -= V h
                (jax's _iterative_classical_gram_schmidt with max_iterations=2 loops while
                k < max_iterations - 1, so it stops after its first pass)
                V[:, j+1], h[j+1] = normalize(v, threshold eps * v0);  H[j, :] = h
                breakdown = h[j+1] == 0
            y = solve(H H^T, H e1 beta) by Cholesky           # the normal equations of min ||H^T y - beta e1||
            x = x + V[:, :m] y;  w, beta = normalize(M (b - A x));  k += 1

    normalize(v, t) returns (v / ||v||, ||v||) when ||v|| > t (default t = eps), else (0, 0). The
    stop test is on the preconditioned residual, checked once per restart cycle. Returns
    (x, Arnoldi steps, restart cycles, final beta)."""
    import scipy.linalg as sla

    b = np.asarray(b, dtype=np.float64)
    n = b.shape[0]
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)

    def M(v):
        return v if inv_diag is None else inv_diag * v

    m = min(int(restart), n)
    maxiter = 10 * n if maxiter is None else int(maxiter)
    eps = np.finfo(np.float64).eps
    b_norm = float(np.linalg.norm(b))
    atol_ = max(tol * b_norm, atol)
    Mb_norm = float(np.linalg.norm(M(b)))
    ptol = Mb_norm * min(1.0, atol_ / b_norm) if b_norm > 0 else 0.0
    w, beta = _safe_normalize(M(b - A @ x))
    steps = cycles = 0
    while beta > ptol and cycles < maxiter:
        V = np.zeros((n, m + 1))
        V[:, 0] = w
        H = np.eye(m, m + 1)
        for j in range(m):
            v = M(A @ V[:, j])
            _, v0 = _safe_normalize(v)
            h = V.T @ v
            v = v - V @ h
            unit, h[j + 1] = _safe_normalize(v, eps * v0)
            V[:, j + 1] = unit
            H[j, :] = h
            steps += 1
            if h[j + 1] == 0.0:
                break
        e1 = np.zeros(m + 1)
        e1[0] = beta
        y = sla.cho_solve(sla.cho_factor(H @ H.T), H @ e1)
        x = x + V[:, :m] @ y
        w, beta = _safe_normalize(M(b - A @ x))
        cycles += 1
    return x, steps, cycles, beta


def residual_check(A, b, x, rtol=1e-4):
    """Relative true residual; raises RuntimeError like ``_maybe_residual_check``."""
    rel = float(np.linalg.norm(b - A @ x) / (np.linalg.norm(b) + 1e-30))
    if not np.isfinite(rel) or rel > rtol:
        raise RuntimeError(f"jno.solve.cg did not solve the system (relative residual {rel:.1e})")
    return rel


def mixed_pcg(A, b, inv_diag, tol=1e-8, atol=0.0, maxiter=20_000, delta2=1e-4, restart=False,
              single_reduction=True):
    """The mixed-precision Jacobi-PCG of ``femk_pcg_mixed`` (no reference counterpart): FP32 values
    and inner vectors, FP64 solution, FP64 true residual at reliable updates (when the FP32 <r, r>
    fell by ``delta2`` since the last update, met the stop test, or at the cap), stopping on the FP64
    residual with the stop rule of :func:`pcg`. ``restart`` starts a new direction at every update.

    ``single_reduction`` selects the device's arrangement: CG on A^ = S A S (S = D^-1/2, formed in
    FP64, rounded to FP32) -- Jacobi-PCG in split form, so z^ = r^ -- with w = A^ r and s = A^ p by
    recurrence, the products <p, s>, <r, s>, <r, r> taken after the vector update and <r, w> after
    the SpMV, and <p', A^ p'> = <r, w> + 2 beta <r, s> + beta^2 <p, s>. Steps alternate: the odd ones
    (counted from 0 after each refresh) form <r, D r> for the stop and drop tests and add two steps'
    worth of e, (alpha' + alpha beta) p' + alpha r; an owed term is paid at the update. Otherwise the
    textbook FP32 loop (q = A p, <p, q> and <r, z> in two reductions, z = D^-1 r). FP32 products are
    summed in FP64 here (the device sums FP32 per thread, then FP64), so iteration counts agree to a
    few. Returns (x, FP32 iterations, FP64 residual evaluations)."""
    import scipy.sparse as sp

    A64 = A.tocsr()
    f32 = np.float32
    b = np.asarray(b, dtype=np.float64)
    dinv = np.asarray(inv_diag, dtype=np.float64)
    n = b.size

    def dot(a, c):
        return float(np.dot(a.astype(np.float64), c.astype(np.float64)))

    x = np.zeros(n)
    e = np.zeros(n, f32)
    atol2 = max(tol * tol * float(b @ b), atol * atol)
    it, outer = 0, 1
    if not single_reduction:
        A32, d32 = A64.astype(f32), dinv.astype(f32)
        r64 = b - A64 @ x
        rr_since = float(r64 @ r64)
        if not rr_since > atol2 or maxiter <= 0:
            return x, 0, outer
        r = r64.astype(f32)
        u = d32 * r
        p = u.copy()
        gamma = dot(r, u)
        while True:
            q = A32 @ p
            alpha = gamma / dot(p, q)
            e = f32(alpha) * p + e
            r = -f32(alpha) * q + r
            u = d32 * r
            g2, rho = dot(r, u), dot(r, r)
            it += 1
            if rho <= atol2 or rho < delta2 * rr_since or it >= maxiter:
                x = x + e
                e[:] = 0
                r64 = b - A64 @ x
                rr_since = float(r64 @ r64)
                outer += 1
                if rr_since <= atol2 or it >= maxiter:
                    return x, it, outer
                r = r64.astype(f32)
                u = d32 * r
                g2 = dot(r, u)
                beta = 0.0 if restart else g2 / gamma
            else:
                beta = g2 / gamma
            gamma = g2
            p = f32(beta) * p + u
    sc64 = np.sqrt(dinv)
    Ah = (sp.diags(sc64) @ A64 @ sp.diags(sc64)).tocsr().astype(f32)
    dd = (1.0 / dinv).astype(f32)
    p = np.zeros(n, f32)
    s = np.zeros(n, f32)

    def replace():
        r64 = b - A64 @ x
        return (sc64 * r64).astype(f32), float(r64 @ r64)

    r, rr_since = replace()
    if not rr_since > atol2 or maxiter <= 0:
        return x, 0, outer
    gamma, alpha, beta = None, 1.0, 0.0
    w = Ah @ r  # the first direction: beta = 0
    g2, ps, rs = dot(r, r), 0.0, 0.0
    j, pend = 0, 0.0  # steps since the last refresh; alpha whose e += alpha p an even step owes
    refreshed = True
    while True:
        den = dot(r, w) + 2.0 * beta * rs + beta * beta * ps
        if not den > 0:
            if refreshed:
                raise ArithmeticError("mixed_pcg: <p, A p> <= 0 in FP32")
            # an untested even step left r = 0 (exact arithmetic): the FP64 residual decides
            x = x + sc64 * (f32(pend) * p + e).astype(np.float64)
            e[:] = 0
            pend, j = 0.0, 0
            r, rr_since = replace()
            outer += 1
            if rr_since <= atol2 or it >= maxiter:
                return x, it, outer
            g2, ps, rs = dot(r, r), dot(p, s), dot(r, s)
            w = Ah @ r
            beta = 0.0 if restart else g2 / gamma
            refreshed = True
            continue
        refreshed = False
        alpha, gamma = g2 / den, g2
        odd = j % 2 == 1  # odd steps pay e for two steps and read D for the tests
        p_prev, r_prev = p, r
        p = f32(beta) * p + r  # K_A
        s = f32(beta) * s + w
        if odd:  # alpha' p' + alpha p = (alpha' + alpha beta) p' + alpha r
            e = f32(pend + alpha * beta) * p_prev + (f32(alpha) * r_prev + e)
        r = -f32(alpha) * s + r
        ps, rs, g2 = dot(p, s), dot(r, s), dot(r, r)
        rho = dot(r * r, dd) if odd else None
        pend = 0.0 if odd else alpha
        w = Ah @ r  # K_B
        it += 1
        j += 1
        if (odd and (rho <= atol2 or rho < delta2 * rr_since)) or it >= maxiter:
            x = x + sc64 * (f32(pend) * p + e).astype(np.float64)
            e[:] = 0
            pend, j = 0.0, 0
            r, rr_since = replace()
            outer += 1
            if rr_since <= atol2 or it >= maxiter:
                return x, it, outer
            g2, ps, rs = dot(r, r), dot(p, s), dot(r, s)  # the refresh step's products
            w = Ah @ r
            beta = 0.0 if restart else g2 / gamma
            refreshed = True
        else:
            beta = g2 / gamma
