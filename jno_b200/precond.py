"""``jno.precond`` for the B200 path: the Jacobi preconditioner (jno/precond.py:98-112, :221).

``jacobi().materialize(ctx)`` returns ``inv = 1 / where(|d| > 1e-30, d, 1)`` computed on the
device from the operator's diagonal slots; the CG kernels apply it as ``z = inv * r``.
"""


class PrecondContext:
    def __init__(self, operator):
        self.operator = operator

    def diag(self):
        return self.operator.diag()


class _Jacobi:
    traceable = True
    key = ("jacobi",)

    def materialize(self, ctx):
        op = ctx.operator if isinstance(ctx, PrecondContext) else ctx
        return JacobiApplier(op.jacobi_inverse())

    def __eq__(self, other):
        return isinstance(other, _Jacobi)

    def __hash__(self):
        return hash(self.key)

    def __repr__(self):
        return "jno.precond.jacobi()"


class JacobiApplier:
    """``v -> inv * v`` with the inverse diagonal kept on the device for the fused CG kernels."""

    def __init__(self, inv_diag):
        self.inv_diag = inv_diag

    def __call__(self, v):
        return self.inv_diag * v


def jacobi():
    """Diagonal (Jacobi) preconditioner ``M^-1 v = v / diag(A)`` (zero diagonals left unscaled)."""
    return _Jacobi()
