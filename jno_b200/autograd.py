"""``torch.autograd.Function`` bindings: gradients through the parametric assembly and the solves.

The reference differentiates ``loss(FemLinearSystem.evaluate({name: theta}))`` with ``jax.grad``
(tests/test_fem_native_lagrange.py:688-711): the reverse pass runs through ``segment_sum`` and the
per-cell ``jacfwd`` of the assembly (jno/utils/solver/fem_native.py:2318-2334) and, for
``jno.solve.cg``, through ``lax.custom_linear_solve`` (jno/solve.py:202-206), which differentiates
the solve implicitly. The same structure here, on the B200 kernels:

* :class:`_Assemble` -- ``(vals, b) = assemble(theta)``; its backward is ``femk_assemble_vjp``:
  per element ``dk_e/dtheta * (sum_ab gv[slot(e,a,b)] K_hat_ab - lift terms of gb)``.
* :class:`_LinearSolve` -- ``u = A(vals)^-1 b`` for any operator values; backward
  ``lambda = A^-T du`` (A is symmetric), ``grad_b = lambda``, ``grad_vals[(i, j)] = -lambda_i u_j``
  on the pattern.
* :class:`_SolveParam` -- the same solve when ``A`` is the assembly of a parameter: the backward
  contracts per element instead of materialising ``grad_vals`` (``femk_adjoint_grad``:
  ``-dk_e/dtheta (m o lambda)_e^T K_hat_e (m o u)_e``, m masking Dirichlet DOFs), which equals
  ``_LinearSolve`` followed by ``_Assemble``'s backward. ``grad_b = lambda`` still flows into ``b``'s
  own graph (the Dirichlet lift makes ``b`` depend on the parameter when ``g != 0``).

``solve_p0`` / ``solve_nodal`` are the fused assemble + solve of one call.
:func:`central_difference` evaluates the central finite-difference quotient of a lumped-mass misfit
without subtractive cancellation (for gradient checks).
"""

import numpy as np
import torch

from . import _lib


def _needs_param(mode):
    return mode != _lib.COEF_CONST


class _Assemble(torch.autograd.Function):
    @staticmethod
    def forward(ctx, param, plan, mode, scale, f, g):
        vals, b = plan.assemble(param.detach(), mode, scale, f, g)
        ctx.plan, ctx.mode, ctx.scale, ctx.g = plan, mode, scale, g
        ctx.save_for_backward(param)
        if g is None:
            ctx.mark_non_differentiable(b)  # the load does not depend on the coefficient without a lift
        return vals, b

    @staticmethod
    def backward(ctx, gv, gb):
        (param,) = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return None, None, None, None, None, None
        gv = None if gv is None else gv.contiguous().to(torch.float64)
        gb = None if (gb is None or ctx.g is None) else gb.contiguous().to(torch.float64)
        grad = ctx.plan.assemble_vjp(param.detach(), gv, gb, ctx.mode, ctx.scale, ctx.g)
        return grad, None, None, None, None, None


def assemble(plan, param, mode=_lib.COEF_EXP, scale=1.0, f=1.0, g=None):
    """(vals, b) with autograd from ``param`` when it requires grad (else a plain assembly)."""
    if _needs_param(mode) and isinstance(param, torch.Tensor) and param.requires_grad and torch.is_grad_enabled():
        return _Assemble.apply(param, plan, mode, scale, f, g)
    return plan.assemble(param if not isinstance(param, torch.Tensor) else param.detach(), mode, scale, f, g)


def _pattern_rows(plan):
    rows = getattr(plan, "_rows_cache", None)
    if rows is None:
        indptr, _ = plan.pattern()
        rows = torch.repeat_interleave(torch.arange(plan.n, device=plan.device), (indptr[1:] - indptr[:-1]).long())
        plan._rows_cache = rows
    return rows


class _LinearSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, b, plan, solve):
        u = solve(vals.detach(), b.detach())
        ctx.plan, ctx.solve = plan, solve
        ctx.save_for_backward(vals, u)
        return u

    @staticmethod
    def backward(ctx, gu):
        vals, u = ctx.saved_tensors
        lam = ctx.solve(vals.detach(), gu.contiguous().to(torch.float64))  # A^T = A
        gvals = None
        if ctx.needs_input_grad[0]:
            _, indices = ctx.plan.pattern()
            gvals = -lam[_pattern_rows(ctx.plan)] * u[indices.long()]
        gb = lam if ctx.needs_input_grad[1] else None
        return gvals, gb, None, None


class _SolveParam(torch.autograd.Function):
    @staticmethod
    def forward(ctx, param, b, plan, mode, scale, solve):
        u = solve(b.detach())
        ctx.plan, ctx.mode, ctx.scale, ctx.solve = plan, mode, scale, solve
        ctx.save_for_backward(param, u)
        return u

    @staticmethod
    def backward(ctx, gu):
        param, u = ctx.saved_tensors
        lam = ctx.solve(gu.contiguous().to(torch.float64))  # A^T = A
        gp = ctx.plan.adjoint_grad(param.detach(), u, lam, ctx.mode, ctx.scale) if ctx.needs_input_grad[0] else None
        gb = lam if ctx.needs_input_grad[1] else None
        return gp, gb, None, None, None, None


def linear_solve(A, b, solve):
    """``u = solve(A, b)`` with autograd: through the assembly parameter when ``A`` is the unmodified
    output of a differentiable assembly (or a matrix-free operator of a parameter), else through
    ``A``'s stored values. ``solve(vals, rhs)`` / ``solve(rhs)`` runs the forward and adjoint solves."""
    from .sparse import CsrMatrix, MatrixFreeOperator

    param = getattr(A, "param", None) if isinstance(A, MatrixFreeOperator) else None
    if isinstance(A, CsrMatrix) and A.assembly is not None and A.data is getattr(A, "_assembled_data", None):
        param = A.assembly[0]
    if isinstance(param, torch.Tensor) and param.requires_grad:
        mode, scale = (A.mode, A.scale) if isinstance(A, MatrixFreeOperator) else A.assembly[1:3]
        return _SolveParam.apply(param, b, A.plan, mode, scale, lambda rhs: solve(None, rhs))
    if isinstance(A, MatrixFreeOperator):
        return solve(None, b.detach())
    return _LinearSolve.apply(A.data, b, A.plan, solve)


class _SolveP0(torch.autograd.Function):
    @staticmethod
    def forward(ctx, param, plan, mode, scale, f, tol, maxiter, precision):
        vals, b = plan.assemble(param, mode, scale, f)
        inv = plan.jacobi(vals)
        if precision == "mixed":
            u, _, _, _, st = plan.pcg_mixed(vals, b, inv, tol=tol, maxiter=maxiter)
        else:
            u, _, _, st = plan.pcg(vals, b, inv_diag=inv, tol=tol, maxiter=maxiter, relres=False)
        ctx.plan, ctx.mode, ctx.scale, ctx.tol, ctx.maxiter, ctx.precision = plan, mode, scale, tol, maxiter, precision
        ctx.save_for_backward(param, vals, inv, u)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        param, vals, inv, u = ctx.saved_tensors
        plan = ctx.plan
        rhs = grad_u.contiguous().to(torch.float64)
        if ctx.precision == "mixed":
            lam, _, _, _, _ = plan.pcg_mixed(vals, rhs, inv, tol=ctx.tol, maxiter=ctx.maxiter)
        else:
            lam, _, _, _ = plan.pcg(vals, rhs, inv_diag=inv, tol=ctx.tol, maxiter=ctx.maxiter, relres=False)
        grad = plan.adjoint_grad(param, u, lam, ctx.mode, ctx.scale)
        return grad, None, None, None, None, None, None, None


def solve_p0(plan, param, mode=_lib.COEF_EXP, scale=1.0, f=1.0, tol=1e-8, maxiter=20_000, precision="fp64"):
    """Differentiable ``u(param)`` for ``scale * g(param_e) grad u . grad v - f v`` with u = 0 on the boundary."""
    return _SolveP0.apply(param, plan, mode, scale, f, tol, maxiter, precision)


def solve_nodal(plan, param, mode=_lib.COEF_NODAL_EXP, scale=1.0, f=1.0, tol=1e-8, maxiter=20_000,
                precision="fp64"):
    """The same for a nodal P1 parameter (one value per vertex): the backward pass spreads each
    element's dJ/dk_e onto its vertices by dk_e/dparam_i."""
    if mode not in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR):
        raise ValueError("solve_nodal takes FEMK_COEF_NODAL_EXP or FEMK_COEF_NODAL_LINEAR")
    return _SolveP0.apply(param, plan, mode, scale, f, tol, maxiter, precision)


def central_difference(plan, logk, ustar, mass, elements, eps=1e-6, f=1.0, tol=1e-13):
    """Central finite differences ``(J(theta + eps e_c) - J(theta - eps e_c)) / (2 eps)`` of
    ``J = 1/2 sum_i M_ii (u_i - u*_i)^2`` for P0 log-conductivities (k = exp(theta)), u = 0 on the
    boundary, at the listed elements, evaluated without subtractive cancellation.

    With A(+) u(+) = b = A(-) u(-) (the load does not depend on theta), the difference
    d = u(+) - u(-) solves A(+) d = (A(-) - A(+)) u(-), whose right-hand side is element c's
    stiffness alone: (k(-) - k(+)) P_c K_hat_c (m o u(-))_c (m masks Dirichlet DOFs). Then
    J(+) - J(-) = sum_i M_ii d_i (u(-)_i + d_i / 2 - u*_i) exactly, so the quotient carries the FP64
    solves' accuracy (tol) instead of the rounding of J divided by 2 eps. Returns f64[len(elements)]."""
    base = torch.as_tensor(logk, dtype=torch.float64, device=plan.device).reshape(-1)
    ustar = torch.as_tensor(ustar, dtype=torch.float64, device=plan.device)
    mass = torch.as_tensor(mass, dtype=torch.float64, device=plan.device)
    khat, _ = plan.element_matrices()
    ex = plan.export()
    cells = ex["cells"].long()
    free = (ex["dirichlet_mask"] == 0).to(torch.float64)
    out = np.zeros(len(elements))
    for j, c in enumerate(np.asarray(elements, dtype=np.int64).tolist()):
        lm, lp = base.clone(), base.clone()
        lm[c] -= eps
        lp[c] += eps
        vm, bm = plan.assemble(lm, f=f)
        um, _, _, _ = plan.pcg(vm, bm, inv_diag=plan.jacobi(vm), tol=tol, relres=False)
        vp, _ = plan.assemble(lp, f=f)
        dofs = cells[c]
        m = free[dofs]
        km, kp = torch.exp(lm[c]), torch.exp(lp[c])
        rhs = torch.zeros_like(um)
        rhs.index_add_(0, dofs, (km - kp) * m * (khat[c] @ (m * um[dofs])))
        d, _, _, _ = plan.pcg(vp, rhs, inv_diag=plan.jacobi(vp), tol=tol, relres=False)
        dJ = torch.sum(mass * d * (um + 0.5 * d - ustar)).item()
        out[j] = dJ / (2.0 * eps)
    return out
