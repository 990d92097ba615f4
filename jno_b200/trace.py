"""A small symbolic front end that recognises the weak forms of the B200 path.

It mirrors the reference's DSL surface for this path only (``d.fem_symbols``, ``u.bind``, ``ui.x``,
``jno.np.exp``, ``jno.np.parameter``, ``u(xb, yb, zb) - g``; jno/trace/__init__.py,
jno/architectures/models.py:58-142) and classifies a form into the kernel arguments:

    [rho * ui.t * vi +] coef * (ui.x*vi.x + ui.y*vi.y [+ ui.z*vi.z]) - f * vi,
    coef in {c, c*p, c*exp(p)},  rho, c, f constants

with p a P0 parameter (one value per element) or, in P1 forms, a nodal P1 parameter (one value per
vertex). The optional ``ui.t * vi`` mass term makes the form the linear first-order transient block
``M u' + A u = c`` (jno/utils/solver/fem_native.py:2846-3110), with ``u(initial) - u0`` giving its
initial state. Anything else raises ``NotImplementedError``: other physics is outside this path.
"""

import numbers

import numpy as np


class Expr:
    def __add__(self, o):
        return Add(self, _wrap(o))

    def __radd__(self, o):
        return Add(_wrap(o), self)

    def __sub__(self, o):
        return Add(self, Mul(Const(-1.0), _wrap(o)))

    def __rsub__(self, o):
        return Add(_wrap(o), Mul(Const(-1.0), self))

    def __mul__(self, o):
        return Mul(self, _wrap(o))

    def __rmul__(self, o):
        return Mul(_wrap(o), self)

    def __neg__(self):
        return Mul(Const(-1.0), self)

    def __pow__(self, k):
        if not isinstance(k, numbers.Integral) or k < 1:
            raise NotImplementedError("only positive integer powers")
        out = self
        for _ in range(k - 1):
            out = Mul(out, self)
        return out


def _wrap(o):
    if isinstance(o, Expr):
        return o
    if isinstance(o, numbers.Number):
        return Const(float(o))
    raise TypeError(f"cannot use {type(o).__name__} in a weak form")


class Const(Expr):
    def __init__(self, v):
        self.v = float(v)


class Add(Expr):
    def __init__(self, a, b):
        self.a, self.b = a, b


class Mul(Expr):
    def __init__(self, a, b):
        self.a, self.b = a, b


class Exp(Expr):
    def __init__(self, a):
        self.a = a


class Sin(Expr):
    def __init__(self, a):
        self.a = a


class Cos(Expr):
    def __init__(self, a):
        self.a = a


class Coordinate(Expr):
    """A coordinate of a region: axis 0..dim-1, or "t" (the time variable of a transient domain)."""

    def __init__(self, region, axis):
        self.region, self.axis = region, axis


class FieldSymbol(Expr):
    """A trial/test symbol (``role``) of a Lagrange field or a P0 symbol (space='P0')."""

    def __init__(self, name, role, domain, order, space="P"):
        self.name, self.role, self.domain, self.order, self.space = name, role, domain, order, space

    def bind(self, **coords):
        return Bound(self)

    def __call__(self, *coords):
        regions = {getattr(c, "region", None) for c in coords}
        if regions == {"initial"}:
            return TraceOn(self, "initial")
        if regions != {"boundary"}:
            raise NotImplementedError("Dirichlet conditions are supported on the whole 'boundary' only")
        return TraceOn(self, "boundary")


class Bound(Expr):
    def __init__(self, sym):
        self.sym = sym

    @property
    def x(self):
        return Deriv(self.sym, 0)

    @property
    def y(self):
        return Deriv(self.sym, 1)

    @property
    def z(self):
        return Deriv(self.sym, 2)

    @property
    def t(self):
        return Deriv(self.sym, "t")


class Deriv(Expr):
    def __init__(self, sym, axis):
        self.sym, self.axis = sym, axis


class TraceOn(Expr):
    def __init__(self, sym, region):
        self.sym, self.region = sym, region


class Param(Expr):
    """``jno.np.parameter(<symbol>, name=...)`` (jno/architectures/models.py:85-117): one value per
    element for a P0 symbol, one value per P1 vertex (``nodal``) for a P1 symbol; or
    ``jno.np.parameter((1,), name=...)``, one value for the whole mesh (``scalar``)."""

    def __init__(self, sym, name, nodal=False, scalar=False):
        self.sym, self.name, self.nodal, self.scalar = sym, name, nodal, scalar


def parameter(sym, name="param", **_):
    if isinstance(sym, tuple) and tuple(sym) in ((), (1,)):
        return Param(None, name, scalar=True)  # a global scalar (tests/test_fem_native_lagrange.py:666)
    if not isinstance(sym, FieldSymbol):
        raise NotImplementedError("jno.np.parameter takes a field symbol or the shape (1,) on the B200 path")
    if sym.space == "P0":
        return Param(sym, name)
    if sym.order != 1:
        # the reference raises the same way for higher-order symbols (models.py:109-113)
        raise NotImplementedError("nodal field parameters support P1 (order=1) symbols only")
    return Param(sym, name, nodal=True)


def exp(a):
    a = _wrap(a)
    if isinstance(a, Const):
        return Const(float(np.exp(a.v)))
    return Exp(a)


def sin(a):
    """``jno.np.sin``: in initial and Dirichlet value expressions."""
    a = _wrap(a)
    return Const(float(np.sin(a.v))) if isinstance(a, Const) else Sin(a)


def cos(a):
    """``jno.np.cos``: in initial and Dirichlet value expressions."""
    a = _wrap(a)
    return Const(float(np.cos(a.v))) if isinstance(a, Const) else Cos(a)


# ------------------------------------------------------------------------------ classification
def _monomials(e):
    """Expand into a list of (scalar, [factors])."""
    if isinstance(e, Const):
        return [(e.v, [])]
    if isinstance(e, Add):
        return _monomials(e.a) + _monomials(e.b)
    if isinstance(e, Mul):
        out = []
        for ca, fa in _monomials(e.a):
            for cb, fb in _monomials(e.b):
                out.append((ca * cb, fa + fb))
        return out
    return [(1.0, [e])]


def _coef_key(factors):
    """Coefficient factors -> ('const',) | ('linear', name) | ('exp', name)."""
    params = [f for f in factors if isinstance(f, Param)]
    exps = [f for f in factors if isinstance(f, Exp)]
    other = [f for f in factors if not isinstance(f, (Param, Exp))]
    if other:
        raise NotImplementedError("a spatially varying coefficient is outside the B200 path (parameters only)")
    if not params and not exps:
        return ("const",)
    if len(params) == 1 and not exps:
        kind = "nodal_linear" if params[0].nodal else ("scalar_linear" if params[0].scalar else "linear")
        return (kind, params[0].name)
    if len(exps) == 1 and not params and isinstance(exps[0].a, Param):
        kind = "nodal_exp" if exps[0].a.nodal else ("scalar_exp" if exps[0].a.scalar else "exp")
        return (kind, exps[0].a.name)
    raise NotImplementedError("only c, c*p and c*exp(p) coefficients are on the B200 path")


class WeakForm:
    """Classified volume form: k_e = scale * g(param_e), source f, field order; ``mass`` is the
    constant coefficient of the ``ui.t * vi`` term of a transient form (None when steady);
    ``scalar`` when the parameter is one value for the whole mesh (broadcast to every element)."""

    def __init__(self, order, mode, scale, param, f, domain, mass=None, scalar=False):
        self.order, self.mode, self.scale, self.param, self.f, self.domain = order, mode, scale, param, f, domain
        self.mass, self.scalar = mass, scalar


def classify_volume(expr):
    stiff = {}  # axis -> (scale, key)
    source = 0.0
    mass = None
    order = None
    domain = None
    for c, factors in _monomials(expr):
        ders = [f for f in factors if isinstance(f, Deriv)]
        vals = [f for f in factors if isinstance(f, Bound)]
        rest = [f for f in factors if not isinstance(f, (Deriv, Bound))]
        if len(ders) == 1 and ders[0].axis == "t":
            if (len(vals) != 1 or rest or ders[0].sym.role != "trial" or vals[0].sym.role != "test"):
                raise NotImplementedError("the transient term must read rho * ui.t * vi with a constant rho")
            mass = (mass or 0.0) + c
            continue
        if any(d.axis == "t" for d in ders):
            raise NotImplementedError("only the first-order ui.t * vi term is on the B200 path")
        if len(ders) == 2 and not vals:
            roles = {d.sym.role for d in ders}
            if roles != {"trial", "test"} or ders[0].axis != ders[1].axis:
                raise NotImplementedError("only grad u . grad v stiffness terms are on the B200 path")
            ax = ders[0].axis
            if ax in stiff:
                raise NotImplementedError("repeated stiffness component")
            stiff[ax] = (c, _coef_key(rest))
            order = ders[0].sym.order
            domain = ders[0].sym.domain
        elif len(vals) == 1 and not ders and vals[0].sym.role == "test":
            if rest:
                raise NotImplementedError("only a constant source f is on the B200 path")
            source += -c
        elif not ders and not vals:
            continue
        else:
            raise NotImplementedError("this term is outside the B200 path (-div(k grad u) = f only)")
    dim = getattr(domain, "dimension", 3)
    if sorted(stiff) != list(range(dim)):
        raise NotImplementedError(
            "the form needs ui.x*vi.x + ui.y*vi.y" + (" + ui.z*vi.z" if dim == 3 else "") + f" on a {dim}-D domain")
    scales = {s for s, _ in stiff.values()}
    keys = {k for _, k in stiff.values()}
    if len(scales) != 1 or len(keys) != 1:
        raise NotImplementedError("an anisotropic coefficient is outside the B200 path")
    scale, key = scales.pop(), keys.pop()
    from . import _lib

    mode = {"const": _lib.COEF_CONST, "linear": _lib.COEF_LINEAR, "exp": _lib.COEF_EXP,
            "scalar_linear": _lib.COEF_LINEAR, "scalar_exp": _lib.COEF_EXP,
            "nodal_linear": _lib.COEF_NODAL_LINEAR, "nodal_exp": _lib.COEF_NODAL_EXP}[key[0]]
    if key[0].startswith("nodal") and order != 1:
        raise NotImplementedError("a nodal P1 parameter in a P2 form is outside the B200 path")
    if mass is not None and not mass > 0.0:
        raise NotImplementedError("the ui.t * vi coefficient must be a positive constant")
    return WeakForm(order, mode, scale, key[1] if len(key) > 1 else None, source, domain, mass,
                    scalar=key[0].startswith("scalar"))


def evaluate_on(expr, pts):
    """Evaluate a Dirichlet value expression (constants and boundary coordinates) at points f64[m, dim]."""
    if isinstance(expr, Const):
        return np.full(pts.shape[0], expr.v)
    if isinstance(expr, Coordinate):
        if expr.axis == "t":
            raise NotImplementedError("time-dependent boundary or initial values are outside the B200 path")
        return pts[:, expr.axis].copy()
    if isinstance(expr, Add):
        return evaluate_on(expr.a, pts) + evaluate_on(expr.b, pts)
    if isinstance(expr, Mul):
        return evaluate_on(expr.a, pts) * evaluate_on(expr.b, pts)
    if isinstance(expr, Exp):
        return np.exp(evaluate_on(expr.a, pts))
    if isinstance(expr, Sin):
        return np.sin(evaluate_on(expr.a, pts))
    if isinstance(expr, Cos):
        return np.cos(evaluate_on(expr.a, pts))
    raise NotImplementedError("boundary and initial values may use constants, coordinates, exp, sin and cos only")


def classify_condition(expr):
    """``u(boundary) - g`` or ``u(initial) - u0`` -> (region, symbol, value expression)."""
    sym, g = classify_dirichlet(expr, regions=("boundary", "initial"))
    return _condition_region(expr), sym, g


def _condition_region(expr):
    for _c, factors in _monomials(expr):
        for f in factors:
            if isinstance(f, TraceOn):
                return f.region
    return None


def classify_dirichlet(expr, regions=("boundary",)):
    """``u(boundary) - g`` -> (symbol, g expression)."""
    traces, rest = [], []
    for c, factors in _monomials(expr):
        tr = [f for f in factors if isinstance(f, TraceOn)]
        if any(t.region not in regions for t in tr):
            raise NotImplementedError(f"a condition on {tr[0].region!r} is outside the B200 path")
        if tr:
            if len(tr) != 1 or len(factors) != 1 or c != 1.0:
                raise NotImplementedError("Dirichlet terms must read u(boundary) - g")
            traces.append(tr[0])
        else:
            prod = Const(-c)
            for f in factors:
                prod = Mul(prod, f)
            rest.append(prod)
    if len(traces) != 1:
        raise NotImplementedError("exactly one u(boundary) per Dirichlet term")
    g = Const(0.0)
    for r in rest:
        g = Add(g, r)
    return traces[0].sym, g
