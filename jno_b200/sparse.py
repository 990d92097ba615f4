"""The assembled operator: canonical CSR in HBM plus the views the reference's consumers expect.

The pattern is the reference's compress-plan unique set (jno/utils/solver/fem_utils.py:4049-4057);
values are FP64 with Dirichlet rows/columns stored as explicit zeros and a unit diagonal (the
parametric route, fem_native.py:3311-3339). ``to_bcoo(appended=True)`` rebuilds the reference's
exact BCOO layout (compressed triplets with the Dirichlet entries zeroed, then one ``(d, d, 1)``
triplet per Dirichlet DOF appended, fem_utils.py:3354-3359). ``compact()`` is the non-parametric
route's operator: the same entries with the exact zeros dropped (``compress_eager``,
fem_utils.py:4063-4091), computed on the device.
"""

import torch

from . import _lib


class CsrMatrix:
    """Device CSR operator bound to its :class:`~jno_b200.plan.FemPlan`."""

    def __init__(self, plan, data, assembly=None):
        self.plan = plan
        self.data = data
        self.indptr, self.indices = plan.pattern()
        self.shape = (plan.n, plan.n)
        # (param, mode, scale) of the values: matrix-free use, and the solves' gradient through the
        # parameter while `data` is still the assembly's own output
        self.assembly = assembly
        self._assembled_data = data if assembly is not None else None
        self._inv_diag = None

    @property
    def nnz(self):
        return int(self.data.numel())

    @property
    def solver_values(self):
        """Values on the plan's canonical pattern: what the SpMV and CG kernels stream (no autograd)."""
        return self.data.detach()

    def compact(self):
        """:class:`CompactCsrMatrix` of the entries with ``|v| > 0`` (``compress_eager``)."""
        return CompactCsrMatrix(self)

    def __matmul__(self, x):
        return self.plan.spmv(self.solver_values, _as_cuda(x, self.data.device))

    mv = __matmul__

    def diag(self):
        """Sum of the stored on-diagonal entries (``matrix_diagonal``, jno/utils/solver/linear.py:88-94)."""
        ex = self.plan.export()
        return self.solver_values[ex["diag_slot"].long()]

    def jacobi_inverse(self):
        if self._inv_diag is None:
            self._inv_diag = self.plan.jacobi(self.solver_values)
        return self._inv_diag

    def todense(self):
        """Dense copy (differentiable in ``data``)."""
        rows = torch.repeat_interleave(
            torch.arange(self.plan.n, device=self.data.device), (self.indptr[1:] - self.indptr[:-1]).long()
        )
        out = torch.zeros(self.shape, dtype=self.data.dtype, device=self.data.device)
        return out.index_put((rows, self.indices.long()), self.data)

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix(
            (self.data.detach().cpu().numpy(), self.indices.cpu().numpy(), self.indptr.cpu().numpy()), shape=self.shape
        )

    def to_bcoo(self, appended=False):
        """(indices i32[nse(+n_D), 2], data f64[nse(+n_D)]) in the reference's BCOO layout."""
        rows = torch.repeat_interleave(
            torch.arange(self.plan.n, device=self.data.device, dtype=torch.int32),
            (self.indptr[1:] - self.indptr[:-1]).long(),
        )
        idx = torch.stack([rows, self.indices], dim=1)
        data = self.data.detach().clone()
        if not appended:
            return idx, data
        ex = self.plan.export()
        dm = ex["dirichlet_mask"].bool()
        d = torch.nonzero(dm).flatten().to(torch.int32)
        data[ex["diag_slot"].long()[dm]] = 0.0
        idx = torch.cat([idx, torch.stack([d, d], dim=1)])
        data = torch.cat([data, torch.ones(d.numel(), dtype=data.dtype, device=data.device)])
        return idx, data


class CompactCsrMatrix(CsrMatrix):
    """The operator of the non-parametric route: ``indptr``/``indices``/``data`` hold only the
    entries with ``|v| > 0`` (rows ascending, columns ascending), as ``compress_eager`` leaves them.

    The solver kernels keep streaming the canonical-pattern values: the dropped entries are exact
    zeros (or NaN, which the residual guard reports either way), so products and solves equal those
    of the compact matrix.
    """

    def __init__(self, full):
        self.plan = full.plan
        self.shape = full.shape
        self.assembly = None  # the compact form comes from the non-parametric route
        self._assembled_data = None
        self._full = full.solver_values
        self.indptr, self.indices, self.data = full.plan.compact(self._full)
        self._inv_diag = None

    @property
    def solver_values(self):
        return self._full

    def compact(self):
        return self

    def to_bcoo(self, appended=False):
        """(indices i32[m, 2], data f64[m]); the compact form has no appended diagonal triplets."""
        rows = torch.repeat_interleave(
            torch.arange(self.plan.n, device=self.data.device, dtype=torch.int32),
            (self.indptr[1:] - self.indptr[:-1]).long(),
        )
        return torch.stack([rows, self.indices], dim=1), self.data.clone()


class MatrixFreeOperator:
    """y = A x recomputed per element from coordinates and k_e; never stores A."""

    def __init__(self, plan, param, mode=_lib.COEF_EXP, scale=1.0):
        self.plan = plan
        self.param = param
        self.mode = mode
        self.scale = scale
        self.shape = (plan.n, plan.n)
        self._inv_diag = None

    def __matmul__(self, x):
        return self.plan.spmv_matfree(self.param, _as_cuda(x, self.plan.device), self.mode, self.scale)

    mv = __matmul__

    def jacobi_inverse(self):
        if self._inv_diag is None:
            self._inv_diag = self.plan.jacobi_matfree(self.param, self.mode, self.scale)
        return self._inv_diag


def _as_cuda(x, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(x, dtype=torch.float64, device=device).contiguous()
