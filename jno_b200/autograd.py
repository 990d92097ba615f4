"""``torch.autograd.Function`` binding: u = solve(A(logk), b) with a hand-written adjoint (P0 or
nodal P1 parameters).

Forward: fused assembly + Jacobi-PCG (FP64, or the mixed FP32/FP64 solver). Backward: one more
PCG on the same kernels for lambda = A^-T dJ/du (A is symmetric), then the per-element contraction
dJ/dlogk_c = -k_c (m o lambda)_e^T K_hat_e (m o u)_e (m masks Dirichlet DOFs; b does not depend on
k). This is the gradient ``jax.grad`` takes through ``lax.custom_linear_solve`` in the reference
(jno/solve.py:202-206): the solve is differentiated implicitly, the preconditioner does not enter.
"""

import torch

from . import _lib


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
