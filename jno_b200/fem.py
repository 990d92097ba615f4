"""``jno.fem`` for the B200 path: classify the terms, build the device plan, assemble on demand.

Mirrors jno/_fem.py:3742 (``fem``), :1132 (``class FEM``: ``.operator`` :1207, ``.solve`` :1294,
``.dofs`` :2575) and ``FemLinearSystem`` (jno/trace/__init__.py:3584-3690): a form with a P0
parameter returns a :class:`FemLinearSystem` re-assembled on each ``evaluate({name: value})``; a
form without one is assembled once into ``(A, b)`` with ``A`` compacted (exact zeros dropped).
The quadrature degree the reference infers (P1 -> 2, P2 -> 4, _fem.py:4551,4573) integrates
these forms exactly, as the closed-form element kernels do, so ``quad_degree`` is accepted for
signature parity and only validated.

A form with a ``rho * ui.t * vi`` term on a domain with ``time=(t0, t1, n_steps)`` is the linear
first-order transient block (jno/utils/solver/fem_native.py:2846-3110): ``fem.solve()`` marches the
theta method over the domain's grid (``_default_transient_integrate``,
jno/utils/solver/backend_blocks.py:475-530; ``time=jno.solve.theta(theta)`` picks the scheme) and
returns the trajectory, state0 first. A form with a runtime parameter takes the reference's
parametric route (Dirichlet rows replaced, columns kept), one without takes the symmetric
elimination of ``_apply_dirichlet_transient`` (jno/utils/solver/fem_1d.py:939-949).
"""

import numpy as np
import torch

from . import _lib
from .plan import FemPlan
from .precond import JacobiApplier, _Jacobi, jacobi
from .solve import LinearSolver, ThetaScheme, bicgstab, cg
from .sparse import CsrMatrix, MatrixFreeOperator
from .trace import classify_condition, classify_volume, evaluate_on


class FemLinearSystem:
    """Parametric linear system: ``evaluate(args) -> (A, b)`` re-assembles on the device.

    ``evaluate`` is differentiable (torch autograd) in the parameter tensor: ``A.data`` and ``b`` carry
    the graph of the assembly (``femk_assemble_vjp`` in the backward pass), so a loss built from them
    -- a dense solve of ``A.todense()``, or ``jno.solve.cg(...)(A, b)`` -- has a gradient with respect
    to the parameter, as ``jax.grad`` gives in the reference (tests/test_fem_native_lagrange.py:688-711).
    """

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

    def solve(self, solve_fn=None, *, periodic=None):
        """Differentiable forward solve ``u = solve_fn(A(theta), b(theta))`` as a callable
        (jno/trace/__init__.py:3617-3669 returns the same as a lazy trace node): ``call(value)`` or
        ``call({name: value})`` evaluates it at the parameter value, and gradients flow back to the
        value through the assembly and ``solve_fn``. ``solve_fn`` is any ``(A, b) -> u``; the
        reference's default is its sparse direct solve, which this path does not have, so the
        default here is Jacobi-PCG at tol 1e-10 (``jno.solve.cg``, differentiable by its adjoint).
        Periodic reduction is outside this path."""
        if periodic is not None:
            raise NotImplementedError("periodic reduction is outside the B200 path")
        if solve_fn is None:
            cg10 = cg(tol=1e-10)

            def solve_fn(A, b):
                return cg10(A, b, M=jacobi())

        return FemSolveCall(self, solve_fn)

    def _solve_eager(self, args=None, linear=None, precond=None, x0=None):
        A, b = self.evaluate(args)
        return _solve(A, b, linear, precond, x0)

    @property
    def A(self):
        return self.evaluate({self._fem.form.param: 0.0})[0]

    @property
    def b(self):
        return self.evaluate({self._fem.form.param: 0.0})[1]


class FemSolveCall:
    """The value of ``FemLinearSystem.solve(solve_fn)``: ``call(value)``, ``call(*values)`` in the order
    of ``params``, or ``call({name: value})`` -> ``u`` (differentiable in the values)."""

    def __init__(self, system, solve_fn):
        self.system, self.solve_fn = system, solve_fn
        self.params = list(system.runtime_parameter_exprs)
        self.name = "fem_solve"

    def __call__(self, *values):
        if len(values) == 1 and isinstance(values[0], dict):
            args = values[0]
        else:
            if len(values) != len(self.params):
                raise TypeError(f"fem_solve takes {len(self.params)} parameter value(s) {self.params}")
            args = dict(zip(self.params, values))
        A, b = self.system.evaluate(args)
        return self.solve_fn(A, b.reshape(-1))


def _solve(A, b, linear, precond, x0, default=cg):
    solver = default() if linear is None else linear
    M = jacobi() if precond is None else precond
    return solver(A, b, M=M, x0=x0)


class TransientSolution:
    """Trajectory of a transient solve on the domain's time grid: ``fn()`` -> f64[n_steps, n] (CUDA),
    state0 first, like the reference's ``fem.solve().fn()``."""

    def __init__(self, traj, ts, iterations, step_residual):
        self.traj, self.ts, self.iterations, self.step_residual = traj, ts, iterations, step_residual

    def fn(self):
        return self.traj


class FEM:
    """Result of :func:`fem`: plan + classified form."""

    def __init__(self, form, plan, g_values, u0=None, time=None):
        self.form = form
        self.plan = plan
        self._g = g_values
        self._u0 = u0  # transient initial state at the DOFs
        self.time = time  # (t0, t1, n_steps) of a transient form
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
        """The parameter as an f64 CUDA tensor of one value per element (P0, or a scalar broadcast to
        every element) or per P1 vertex (nodal), keeping the caller's autograd graph."""
        name = self.form.param
        if name is None:
            return None
        if name not in args:
            raise KeyError(f"missing runtime parameter {name!r}")
        v = args[name]
        nodal = self.form.mode in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR)
        size = self.plan.nvert if nodal else self.plan.ntet
        if isinstance(v, (int, float)):
            return torch.full((size,), float(v), dtype=torch.float64, device=self.plan.device)
        t = v if isinstance(v, torch.Tensor) else torch.as_tensor(np.asarray(v))
        t = t.to(device=self.plan.device, dtype=torch.float64).reshape(-1)
        if self.form.scalar:
            if t.numel() != 1:
                raise ValueError(f"parameter {name!r} is a scalar: it needs 1 value, got {t.numel()}")
            return t.expand(size).contiguous()
        kind = "nodal P1" if nodal else "P0"
        if t.numel() != size:
            raise ValueError(f"parameter {name!r} is {kind}: it needs {size} values, got {t.numel()}")
        return t.contiguous()

    def _assemble(self, args):
        from . import autograd

        param = self._param_tensor(args)
        vals, b = autograd.assemble(self.plan, param, self.form.mode, self.form.scale, self.form.f, self._g)
        return CsrMatrix(self.plan, vals, (param, self.form.mode, self.form.scale)), b

    @property
    def operator(self):
        if self.is_transient:
            raise NotImplementedError(
                "a transient form has no single (A, b): use fem.solve() for the trajectory or "
                "fem.step_operators(args, theta) for the theta-step operators")
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
        b = self.plan.load(param.detach() if param is not None else None, self.form.mode, self.form.scale,
                           self.form.f, self._g)
        return MatrixFreeOperator(self.plan, param, self.form.mode, self.form.scale), b

    @property
    def is_transient(self):
        return self.form.mass is not None

    @property
    def dt(self):
        t0, t1, n_steps = self.time
        if n_steps <= 1:
            raise ValueError("a transient solve needs time=(t0, t1, n_steps) with n_steps >= 2")
        return (t1 - t0) / (n_steps - 1)

    def step_operators(self, args=None, theta=1.0):
        """(S, R, q) of the theta step as CUDA tensors: S = M' + theta dt A', R = M' - (1 - theta)
        dt A', q = dt (c' + f') on the canonical CSR (rhs = R u + q)."""
        param = self._param_tensor(args or {})
        rho = self.form.mass
        route = _lib.DIRICHLET_ROWS if self.form.param is not None else _lib.DIRICHLET_SYMMETRIC
        # rho M u' + A u = c + f is M u' + (A / rho) u = (c + f) / rho on the free rows
        return self.plan.assemble_theta(param, self.form.mode, self.form.scale / rho, self.form.f / rho, self._g,
                                        theta, self.dt, route)

    def _march(self, time=None, args=None, linear=None, precond=None):
        """The theta march. No slots: the default step solve of SemidiscreteTimeBlock.step
        (Jacobi-BiCGStab at tol 1e-10 plus the 1e-9 step check, backend_blocks.py:386-413). With a
        ``linear`` and/or ``precond`` slot: compose_transient_step_solvers (solver_api.py:911-945),
        i.e. the slot solver (``jno.solve.bicgstab()`` when only ``precond`` is given) at its own
        tolerance with the step operator's Jacobi preconditioner and no step check, the solver's
        residual guard applying per step."""
        if time is not None and not isinstance(time, ThetaScheme):
            raise NotImplementedError("time= takes jno.solve.theta(...) on the B200 path")
        if precond is not None and not isinstance(precond, (_Jacobi, JacobiApplier)):
            raise NotImplementedError("the transient step preconditioner is Jacobi on the B200 path")
        slots = linear is not None or precond is not None
        solver = linear if linear is not None else (bicgstab() if slots else None)
        if solver is not None and (not isinstance(solver, LinearSolver) or solver.name not in ("bicgstab", "cg")
                                   or solver.precision != "fp64"):
            raise NotImplementedError("the transient step solve is Jacobi-BiCGStab or Jacobi-CG on the B200 path")
        th = 1.0 if time is None else time.theta
        S, R, q = self.step_operators(args, th)
        t0, t1, n_steps = self.time
        traj = torch.empty((n_steps, self.plan.n), dtype=torch.float64, device=self.plan.device)
        traj[0] = self._u0
        u = self._u0.clone()
        if solver is None:  # the per-step default of backend_blocks.py:394-396
            _, iters, worst = self.plan.theta_march(S, R, q, u, n_steps - 1, 1e-10, 20_000, traj=traj[1:])
        elif solver.name == "bicgstab":
            _, iters, worst = self.plan.theta_march(S, R, q, u, n_steps - 1, solver.tol, solver.maxiter,
                                                    traj=traj[1:], step_check=0.0)
        else:
            inv = self.plan.jacobi(S)
            iters, worst = [], 0.0
            for k in range(1, n_steps):
                rhs = self.plan.spmv(R, u) + q
                _, it, rel, st = self.plan.pcg(S, rhs, u, inv, solver.tol, solver.atol, solver.maxiter)
                iters.append(it)
                worst = max(worst, rel)
                traj[k] = u
            iters = np.asarray(iters, dtype=np.int32)
        if slots and not worst <= 1e-4:  # the slot solver's eager residual guard (solver_api.py:224-240)
            raise RuntimeError(f"jno.solve.{solver.name} did not solve a transient step (relative residual {worst:.1e})")
        self.stats["transient"] = {"theta": th, "dt": self.dt, "iterations": iters, "step_residual": worst}
        ts = np.linspace(t0, t1, n_steps)
        return TransientSolution(traj, ts, iters, worst)

    def solve(self, linear=None, precond=None, x0=None, args=None, time=None):
        if self.is_transient:
            if x0 is not None:
                raise ValueError("fem.solve: x0 is not used by a transient solve (the initial condition sets state0)")
            return self._march(time, args, linear, precond)
        if time is not None:
            raise ValueError("fem.solve: time= needs a transient form (a ui.t * vi term)")
        if self.form.param is not None:
            return self.operator._solve_eager(args, linear, precond, x0)
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
    conds = [classify_condition(t) for t in dirichlet]
    bcs = [(s, g) for r, s, g in conds if r == "boundary"]
    ics = [(s, g) for r, s, g in conds if r == "initial"]
    if len(bcs) > 1 or len(ics) > 1:
        raise NotImplementedError("one Dirichlet condition on the whole boundary (and one initial condition) is supported")
    d = form.domain
    transient = form.mass is not None
    if ics and not transient:
        raise ValueError("an initial condition needs a transient form (a ui.t * vi term)")
    if transient and getattr(d, "time", None) is None:
        raise ValueError("a transient form needs a domain with time=(t0, t1, n_steps)")
    mesh = d.built_mesh
    plan = FemPlan(mesh.points[:, :dim], mesh.tets, form.order, dirichlet_mask)  # fem_native.py:250
    if not bcs:
        raise NotImplementedError("a Dirichlet condition u(boundary) - g is required on the B200 path")
    pts = plan.export()["points"].cpu().numpy()
    g_values = None
    gv = evaluate_on(bcs[0][1], pts)
    if np.any(gv != 0.0):
        g_values = torch.as_tensor(gv, dtype=torch.float64, device=plan.device)
    u0 = None
    if transient:
        # nodal interpolation of the initial condition at every DOF (exact for Lagrange; the
        # Dirichlet DOFs keep u0 too, fem_native.py:2883-2913); zeros without one
        u0v = evaluate_on(ics[0][1], pts) if ics else np.zeros(plan.n)
        u0 = torch.as_tensor(np.broadcast_to(u0v, (plan.n,)).copy(), dtype=torch.float64, device=plan.device)
    return FEM(form, plan, g_values, u0, getattr(d, "time", None) if transient else None)
