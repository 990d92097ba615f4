"""``jno.solve.cg`` on the B200 kernels (jno/solve.py:191-206, jno/utils/solver/solver_api.py:243-301).

``cg(tol=1e-8, atol=0.0, maxiter=20_000)`` returns a :class:`LinearSolver` called as
``solver(A, b, *, M=None, x0=None) -> x``. The iteration is ``jax.scipy.sparse.linalg.cg``'s
(jax 0.10.1): x0 = 0 by default, stop when <r, r> <= max(tol^2 <b, b>, atol^2) with a
preconditioner (<r, z> without one) or at maxiter. After the solve the eager residual guard of
``_maybe_residual_check`` (solver_api.py:224-240) raises ``RuntimeError`` when
``||b - A x|| / (||b|| + 1e-30) > 1e-4``.

``bicgstab(tol, atol, maxiter)`` is ``jax.scipy.sparse.linalg.bicgstab`` on the same operator, and
``gmres(tol, atol, maxiter=None, restart=30)`` is ``jax.scipy.sparse.linalg.gmres`` (restarted,
``solve_method="batched"``).

Extensions with no reference counterpart: ``precision="mixed"`` (FP32 inner CG with FP64 reliable
updates, ``refine="reliable"`` or classic restarted refinement ``refine="restart"``) and matrix-free
operators (:class:`~jno_b200.sparse.MatrixFreeOperator`). FP32 CG converges more slowly than FP64
as the condition number grows (rounding delays the Krylov convergence; on 2-D P1 512^2 Jacobi-PCG
the FP32 inner loop needs 3.4x the FP64 iterations), so a mixed solve that has not met the stop
rule after ``mixed_maxiter`` FP32 iterations (default ``maxiter``) continues in FP64 from its
iterate, and ``last_info.fallback`` records it.
"""

import math

import torch

from . import _lib
from .precond import JacobiApplier, PrecondContext
from .sparse import CsrMatrix, MatrixFreeOperator, _as_cuda


class LinearOperator:
    """Wrapper kept for signature parity with ``jno.solve.LinearOperator``; holds a device operator."""

    def __init__(self, A):
        self.A = A.A if isinstance(A, LinearOperator) else A

    def mv(self, v):
        return self.A @ v

    __matmul__ = mv

    def diag(self):
        return self.A.diag()


class SolveInfo:
    def __init__(self, iterations, relres, status, outer=None, fallback=0):
        self.iterations, self.relres, self.status, self.outer = iterations, relres, status, outer
        self.fallback = fallback  # FP64 iterations run after a mixed solve missed the stop rule

    def __repr__(self):
        return (f"SolveInfo(iterations={self.iterations}, relres={self.relres:.3e}, outer={self.outer}, "
                f"fallback={self.fallback})")


class LinearSolver:
    def __init__(self, tol, atol, maxiter, precision="fp64", refine="reliable", name="cg", mixed_maxiter=None):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if refine not in ("reliable", "restart"):
            raise ValueError("refine must be 'reliable' or 'restart'")
        self.tol, self.atol = float(tol), float(atol)
        self.maxiter = 20_000 if maxiter is None else int(maxiter)
        self.mixed_maxiter = self.maxiter if mixed_maxiter is None else int(mixed_maxiter)
        self.precision, self.refine, self.name = precision, refine, name
        self.direct = False
        self.key = (type(self), name, (self.tol, self.atol, self.maxiter, precision, refine, self.mixed_maxiter))
        self.last_info = None

    def __eq__(self, other):
        return isinstance(other, LinearSolver) and other.key == self.key

    def __hash__(self):
        return hash(self.key)

    def __call__(self, A, b, *, M=None, x0=None):
        """``x = solve(A, b)``. Differentiable (torch autograd) in ``b`` and in ``A``: through the
        assembly parameter when ``A`` is the unmodified output of ``FemLinearSystem.evaluate`` (or a
        matrix-free operator of a parameter that requires grad), else through ``A.data``; the
        backward pass is one more solve with the same solver on the transposed (= the same) system,
        as ``custom_linear_solve`` does in the reference (jno/solve.py:202-206)."""
        from . import autograd
        from .sparse import CompactCsrMatrix

        op = A.A if isinstance(A, LinearOperator) else A
        if not isinstance(op, (CsrMatrix, MatrixFreeOperator)):
            raise TypeError("the B200 CG takes an assembled CsrMatrix or a MatrixFreeOperator")
        plan = op.plan
        b = b if isinstance(b, torch.Tensor) and b.is_cuda and b.dtype == torch.float64 else _as_cuda(b, plan.device)
        b = b.reshape(-1)
        if M is not None and hasattr(M, "materialize"):
            M = M.materialize(PrecondContext(op))
        if M is not None and not isinstance(M, JacobiApplier):
            raise TypeError("the fused CG kernels apply the Jacobi preconditioner only (jno_b200.precond.jacobi())")
        inv = None if M is None else M.inv_diag.detach()
        x0 = None if x0 is None else _as_cuda(x0, plan.device).reshape(-1).detach()
        grad_a = False
        if torch.is_grad_enabled():
            if isinstance(op, MatrixFreeOperator):
                grad_a = isinstance(op.param, torch.Tensor) and op.param.requires_grad
            else:
                grad_a = op.data.requires_grad
                if grad_a and isinstance(op, CompactCsrMatrix):
                    raise NotImplementedError("gradients through a compacted (non-parametric) operator")
        if not (grad_a or (torch.is_grad_enabled() and b.requires_grad)):
            return self._run(op, None, b.detach(), inv, x0)
        first = [True]

        def solve(vals, rhs):
            x = self._run(op, vals, rhs, inv, x0 if first[0] else None)  # the adjoint solve starts at 0
            first[0] = False
            return x

        return autograd.linear_solve(op, b, solve)

    def _run(self, op, vals, b, inv, x0):
        """One solve on the device (no autograd): the forward, or the adjoint of a backward pass."""
        plan = op.plan
        if vals is None and isinstance(op, CsrMatrix):
            vals = op.solver_values
        x = torch.zeros_like(b) if x0 is None else x0.clone()
        if self.precision == "mixed":
            if not isinstance(op, CsrMatrix) or inv is None:
                raise ValueError("precision='mixed' needs an assembled CsrMatrix and M=jacobi()")
            mode = _lib.MIXED_RELIABLE if self.refine == "reliable" else _lib.MIXED_RESTART
            x, inner, outer, rel, st = plan.pcg_mixed(vals, b, inv, x, self.tol, self.atol, self.mixed_maxiter, mode)
            fb = 0
            if st == _lib.FEMK_NOT_CONVERGED:
                # FP32 rounding stalled the inner loop: finish in FP64 from the mixed iterate
                x, fb, rel, st = plan.pcg(vals, b, x, inv, self.tol, self.atol, self.maxiter)
            self.last_info = SolveInfo(inner, rel, st, outer, fb)
        elif self.name == "bicgstab":
            if not isinstance(op, CsrMatrix):
                raise TypeError("the B200 BiCGStab takes an assembled CsrMatrix")
            x, it, rel, st = plan.bicgstab(vals, b, x, inv, self.tol, self.atol, self.maxiter)
            self.last_info = SolveInfo(it, rel, st)
        elif self.name == "gmres":
            if not isinstance(op, CsrMatrix):
                raise TypeError("the B200 GMRES takes an assembled CsrMatrix")
            x, it, cyc, rel, st = plan.gmres(vals, b, x, inv, self.tol, self.atol, self.restart, self.gmres_maxiter)
            self.last_info = SolveInfo(it, rel, st, outer=cyc)
        elif isinstance(op, MatrixFreeOperator):
            x, it, rel, st = plan.pcg_matfree(op.param.detach(), b, x, inv, op.mode, op.scale, self.tol, self.atol,
                                              self.maxiter)
            self.last_info = SolveInfo(it, rel, st)
        else:
            x, it, rel, st = plan.pcg(vals, b, x, inv, self.tol, self.atol, self.maxiter)
            self.last_info = SolveInfo(it, rel, st)
        rel = self.last_info.relres
        if not math.isfinite(rel) or rel > 1e-4:
            raise RuntimeError(
                f"jno.solve.{self.name} did not solve the system (relative residual {rel:.1e}); the problem may be "
                "singular/ill-posed or need a preconditioner. Try jno.solve.lu(), a precond= spec, or your own solve_fn."
            )
        return x


def cg(*, tol=1e-8, atol=0.0, maxiter=20_000, precision="fp64", refine="reliable", mixed_maxiter=None):
    """Jacobi-preconditionable CG on the B200 kernels (``jax.scipy.sparse.linalg.cg`` semantics)."""
    return LinearSolver(tol, atol, maxiter, precision, refine, mixed_maxiter=mixed_maxiter)


GMRES_MAX_RESTART = 64  # restart lengths the library's GMRES accepts (femk_gmres)


def gmres(*, tol=1e-8, atol=0.0, maxiter=None, restart=30):
    """Restarted GMRES on the B200 kernels (``jax.scipy.sparse.linalg.gmres`` with
    ``solve_method="batched"``, jno/solve.py:216-221): ``maxiter`` counts restart cycles (None: jax's
    10 n); ``last_info.iterations`` = Arnoldi steps, ``last_info.outer`` = cycles."""
    if not 1 <= int(restart) <= GMRES_MAX_RESTART:
        raise ValueError(f"jno.solve.gmres: restart must be in [1, {GMRES_MAX_RESTART}] on the B200 path "
                         f"(the library keeps at most {GMRES_MAX_RESTART + 1} Krylov vectors), got {restart}")
    if maxiter is not None and int(maxiter) < 0:
        raise ValueError("jno.solve.gmres: maxiter must be >= 0 (or None for jax's 10 n restart cycles)")
    s = LinearSolver(tol, atol, 20_000, name="gmres")
    s.restart = int(restart)
    s.gmres_maxiter = None if maxiter is None else int(maxiter)
    s.key = s.key + (("gmres", s.restart, s.gmres_maxiter),)
    return s


def bicgstab(*, tol=1e-8, atol=0.0, maxiter=20_000):
    """BiCGStab on the B200 kernels (``jax.scipy.sparse.linalg.bicgstab`` semantics,
    jno/solve.py:209-213); with ``M=jno.precond.jacobi()`` it is the steady ``fem.solve()`` default
    (jno/_fem.py:110-116)."""
    return LinearSolver(tol, atol, maxiter, name="bicgstab")


class ThetaScheme:
    """``jno.solve.theta(theta)`` (jno/solve.py:1160-1170): the theta-method time scheme of a
    transient ``fem.solve(time=...)`` -- 1 backward Euler (the default), 1/2 Crank-Nicolson."""

    def __init__(self, theta=1.0):
        theta = float(theta)
        if not 0.0 < theta <= 1.0:
            raise NotImplementedError("theta must be in (0, 1] on the B200 path (theta = 0 leaves the Dirichlet rows empty)")
        self.theta = theta


def theta(theta=1.0):
    return ThetaScheme(theta)

