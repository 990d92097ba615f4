"""``jno.fem`` for the B200 path: classify the terms, build the device plan, assemble on demand.

Mirrors jno/_fem.py:3742 (``fem``), :1132 (``class FEM``: ``.operator`` :1207, ``.solve`` :1294,
``.dofs`` :2575) and ``FemLinearSystem`` (jno/trace/__init__.py:3584-3690): a form with a P0
parameter returns a :class:`FemLinearSystem` re-assembled on each ``evaluate({name: value})``; a
form without one is assembled once into ``(A, b)`` with ``A`` compacted (exact zeros dropped).
The quadrature degree the reference infers (P1 -> 2, P2 -> 4, _fem.py:4551,4573) integrates
these forms exactly, as the closed-form element kernels do, so ``quad_degree`` is accepted for
signature parity and only validated.
"""

import numpy as np
import torch

from . import _lib
from .plan import FemPlan
from .precond import jacobi
from .solve import bicgstab, cg
from .sparse import CsrMatrix, MatrixFreeOperator
from .trace import classify_dirichlet, classify_volume, evaluate_on


class FemLinearSystem:
    """Parametric linear system: ``evaluate(args) -> (A, b)`` re-assembles on the device."""

    def __init__(self, fem_obj):
        self._fem = fem_obj
        self.is_parametric = True
        self.runtime_parameter_exprs = {fem_obj.form.param: None}
        self.metadata = {"nonaffine_operator": True}

    def evaluate(self, args=None):
        return self._fem._assemble(args or {})

    def operator(self, args=None):
        return self.evaluate(args)[0]

    def rhs(self, args=None):
        return self.evaluate(args)[1]

    def solve(self, args=None, linear=None, precond=None, x0=None):
        A, b = self.evaluate(args)
        return _solve(A, b, linear, precond, x0)

    @property
    def A(self):
        return self.evaluate({self._fem.form.param: 0.0})[0]

    @property
    def b(self):
        return self.evaluate({self._fem.form.param: 0.0})[1]


def _solve(A, b, linear, precond, x0, default=cg):
    solver = default() if linear is None else linear
    M = jacobi() if precond is None else precond
    return solver(A, b, M=M, x0=x0)


class FEM:
    """Result of :func:`fem`: plan + classified form."""

    def __init__(self, form, plan, g_values):
        self.form = form
        self.plan = plan
        self._g = g_values
        self.problem = None  # routed natively (the reference's marker for the native assembler)
        self.stats = {}
        self._eager = None

    @property
    def dofs(self):
        return self.plan.n

    @property
    def points(self):
        return self.plan.export()["points"]

    def _param_tensor(self, args):
        name = self.form.param
        if name is None:
            return None
        if name not in args:
            raise KeyError(f"missing runtime parameter {name!r}")
        v = args[name]
        if isinstance(v, (int, float)):
            nodal = self.form.mode in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR)
            size = self.plan.nvert if nodal else self.plan.ntet
            return torch.full((size,), float(v), dtype=torch.float64, device=self.plan.device)
        t = v if isinstance(v, torch.Tensor) else torch.as_tensor(np.asarray(v))
        t = t.to(device=self.plan.device, dtype=torch.float64).reshape(-1).contiguous()
        nodal = self.form.mode in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR)
        want, kind = (self.plan.nvert, "nodal P1") if nodal else (self.plan.ntet, "P0")
        if t.numel() != want:
            raise ValueError(f"parameter {name!r} is {kind}: it needs {want} values, got {t.numel()}")
        return t

    def _assemble(self, args):
        param = self._param_tensor(args)
        vals, b = self.plan.assemble(param, self.form.mode, self.form.scale, self.form.f, self._g)
        return CsrMatrix(self.plan, vals, (param, self.form.mode, self.form.scale)), b

    @property
    def operator(self):
        if self.form.param is not None:
            return FemLinearSystem(self)
        if self._eager is None:
            # linear non-parametric route: Dirichlet elimination, then compress_eager drops the exact
            # zeros (jno/utils/solver/fem_native.py:3371-3379)
            A, b = self._assemble({})
            self._eager = (A.compact(), b)
        return self._eager

    @property
    def A(self):
        return self.operator[0] if self.form.param is None else self.operator.A

    @property
    def b(self):
        return self.operator[1] if self.form.param is None else self.operator.b

    def matrix_free(self, args=None):
        """Matrix-free operator and RHS for the same form (``b`` from one assembly of the load)."""
        param = self._param_tensor(args or {})
        _, b = self._assemble(args or {})
        return MatrixFreeOperator(self.plan, param, self.form.mode, self.form.scale), b

    def solve(self, linear=None, precond=None, x0=None, args=None):
        if self.form.param is not None:
            return self.operator.solve(args, linear, precond, x0)
        A, b = self.operator
        # steady linear default of the reference: Jacobi-preconditioned BiCGStab (jno/_fem.py:110-116)
        return _solve(A, b, linear, precond, x0, default=bicgstab)


def fem(terms, quad_degree=None, element_type=None, chunk=None, dirichlet_mask=None):
    """Build the B200 FEM for ``[k grad u . grad v - f v, u(boundary) - g]``."""
    if not isinstance(terms, (list, tuple)) or not terms:
        raise ValueError("jno.fem takes a list of terms")
    vol, dirichlet = terms[0], list(terms[1:])
    form = classify_volume(vol)
    dim = getattr(form.domain, "dimension", 3)
    allowed = (None, "TET4", "TET10") if dim == 3 else (None, "TRI3", "TRI6")
    if element_type not in allowed:
        raise NotImplementedError(f"element_type={element_type!r} is outside the B200 path for a {dim}-D mesh")
    if element_type in ("TET10", "TRI6"):
        form.order = 2
    need = 2 * form.order
    if quad_degree is not None and int(quad_degree) < need:
        raise ValueError(f"quad_degree={quad_degree} under-integrates P{form.order} stiffness (needs {need})")
    if len(dirichlet) > 1:
        raise NotImplementedError("one Dirichlet condition on the whole boundary is supported")
    d = form.domain
    mesh = d.built_mesh
    plan = FemPlan(mesh.points[:, :dim], mesh.tets, form.order, dirichlet_mask)  # fem_native.py:250
    g_values = None
    if dirichlet:
        sym, gexpr = classify_dirichlet(dirichlet[0])
        gv = evaluate_on(gexpr, plan.export()["points"].cpu().numpy())
        if np.any(gv != 0.0):
            g_values = torch.as_tensor(gv, dtype=torch.float64, device=plan.device)
    else:
        raise NotImplementedError("a Dirichlet condition u(boundary) - g is required on the B200 path")
    return FEM(form, plan, g_values)
