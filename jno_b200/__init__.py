"""jno_b200: jNO's P1/P2 tetrahedral (and triangular) assembly -> Jacobi-PCG path on B200 (sm_100a).

The public names mirror the reference's surface for this path (jno/__init__.py:11-19):
``jno_b200.fem``, ``jno_b200.solve.cg``, ``jno_b200.precond.jacobi``, ``jno_b200.np.exp`` /
``jno_b200.np.parameter``, ``jno_b200.domain``. Compute runs in hand-written CUDA kernels behind the C
ABI of ``include/femk.h`` (``libfemk.so``); there is no CPU fallback.
"""

from types import SimpleNamespace

from . import precond, solve  # noqa: F401
from . import trace as _trace
from .domain import domain, equi_distant_box, equi_distant_rect  # noqa: F401
from .fem import FEM, FemLinearSystem, fem  # noqa: F401
from .plan import FemPlan  # noqa: F401
from .sparse import CsrMatrix, MatrixFreeOperator  # noqa: F401

np = SimpleNamespace(exp=_trace.exp, sin=_trace.sin, cos=_trace.cos, parameter=_trace.parameter)

domain.equi_distant_box = staticmethod(equi_distant_box)
domain.equi_distant_rect = staticmethod(equi_distant_rect)

__all__ = ["fem", "solve", "precond", "np", "domain", "FEM", "FemLinearSystem", "FemPlan", "CsrMatrix",
           "MatrixFreeOperator"]
