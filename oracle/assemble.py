"""Oracle: compress-plan CSR pattern, element scatter, Dirichlet elimination, Jacobi (test infrastructure).

Restates:
* the raw triplet order of the Jacobian pattern hoist -- ``jno/utils/solver/fem_native.py:2264-2268``:
  for cell c, test dof a, trial dof b: ``row = cells[c, a]``, ``col = cells[c, b]``;
* ``compress_plan`` -- ``jno/utils/solver/fem_utils.py:4049-4057``: ``np.unique`` of
  ``row * (max_col + 1) + col`` gives the unique, row-major sorted pattern U and the raw -> slot
  ``inverse`` map; values are ``segment_sum(K_e.ravel(), inverse)`` (``fem_native.py:2318-2329``);
* the parametric route's symmetric Dirichlet elimination -- ``_apply_dirichlet_symmetric``
  ``jno/utils/solver/fem_1d.py:667-686`` with ``bcoo_zero_rows_cols`` / ``bcoo_set_unit_diag``
  (``fem_utils.py:3332-3359``): ``b -= A e``; every stored entry of a Dirichlet row or column is
  zeroed (kept as an explicit zero); a ``(d, d, 1)`` triplet is appended, so the canonical CSR has
  ``A[d, d] = 1``; ``b[d] = g[d]``;
* ``compress_eager`` -- ``fem_utils.py:4063-4091`` (non-parametric route only): drop exact zeros;
* ``matrix_diagonal`` -- ``jno/utils/solver/linear.py:88-94`` and ``_Jacobi.materialize`` --
  ``jno/precond.py:106-111``: ``inv = 1 / where(|d| > 1e-30, d, 1)``.
"""

import numpy as np
import scipy.sparse as sp


def raw_pattern(cells):
    """Raw (row, col) int64 arrays in (c, a, b) order."""
    cells = np.asarray(cells, dtype=np.int64)
    T, nd = cells.shape
    rows = np.broadcast_to(cells[:, :, None], (T, nd, nd)).reshape(-1)
    cols = np.broadcast_to(cells[:, None, :], (T, nd, nd)).reshape(-1)
    return rows, cols


def compress_plan(cells):
    """(idx i32[nse,2], inverse i32[T*nd*nd], nse) exactly as the reference's ``np.unique`` plan."""
    rows, cols = raw_pattern(cells)
    stride = int(cols.max()) + 1
    uniq, inverse = np.unique(rows * stride + cols, return_inverse=True)
    idx = np.stack([uniq // stride, uniq % stride], axis=1).astype(np.int32)
    return idx, inverse.reshape(-1).astype(np.int32), int(uniq.shape[0])


def plan_to_csr(idx, n):
    """indptr i32[n+1], indices i32[nse] of a row-major sorted unique pattern."""
    counts = np.bincount(idx[:, 0], minlength=n)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=indptr[1:])
    return indptr.astype(np.int32), idx[:, 1].astype(np.int32)


def csr_pattern_fast(cells, n):
    """Same CSR pattern and slot map as :func:`compress_plan` for large meshes (scipy, no sort of keys).

    Returns (indptr i64[n+1], indices i32[nse], slot i64[T*nd*nd]).
    """
    rows, cols = raw_pattern(cells)
    A = sp.csr_matrix((np.ones(rows.size, dtype=np.float32), (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    indptr = A.indptr.astype(np.int64)
    indices = A.indices.astype(np.int32)
    # slot = indptr[row] + position of col within the row (rows are sorted)
    pos = np.empty(rows.size, dtype=np.int64)
    chunk = 1 << 24
    for s in range(0, rows.size, chunk):
        r = rows[s : s + chunk]
        c = cols[s : s + chunk]
        lo = indptr[r]
        hi = indptr[r + 1]
        # binary search of c within indices[lo:hi]
        while True:
            active = lo < hi
            if not active.any():
                break
            mid = (lo + hi) // 2
            go_right = active & (indices[np.minimum(mid, indices.size - 1)] < c)
            lo = np.where(go_right, mid + 1, lo)
            hi = np.where(active & ~go_right, mid, hi)
        pos[s : s + chunk] = lo
    return indptr, indices, pos


class System:
    """Assembled FP64 system in the canonical CSR of the compress plan."""

    def __init__(self, indptr, indices, data, b, dirichlet, n):
        self.indptr, self.indices, self.data, self.b = indptr, indices, data, b
        self.dirichlet, self.n = dirichlet, n

    def csr(self):
        return sp.csr_matrix((self.data, self.indices, self.indptr), shape=(self.n, self.n))


def assemble(points, cells, order, dirichlet, coef, f=1.0, g=None, plan=None, element=None):
    """Parametric-route assembly of ``coef_e * grad u . grad v - f v`` with Dirichlet ``u = g``.

    ``coef`` is the per-element coefficient k_e (already exponentiated), ``dirichlet`` the sorted
    Dirichlet node ids, ``g`` the per-node Dirichlet values (None = 0). ``plan`` may carry
    (indptr, indices, slot) to skip the pattern build. Returns a :class:`System`.
    """
    from .element import element_matrices, vertices

    points = np.asarray(points, dtype=np.float64)
    cells = np.asarray(cells, dtype=np.int64)
    n = points.shape[0]
    T, nd = cells.shape
    if plan is None:
        idx, inverse, nse = compress_plan(cells)
        indptr, indices = plan_to_csr(idx, n)
        slot = inverse.astype(np.int64)
    else:
        indptr, indices, slot = plan
        nse = indices.size
    if element is None:
        Khat, Fhat = element_matrices(vertices(points, cells), order)
    else:
        Khat, Fhat = element
    Ke = np.asarray(coef, dtype=np.float64)[:, None, None] * Khat
    data = np.bincount(slot, weights=Ke.reshape(-1), minlength=nse)
    b = np.bincount(cells.reshape(-1), weights=(f * Fhat).reshape(-1), minlength=n)
    isd = np.zeros(n, dtype=bool)
    isd[np.asarray(dirichlet, dtype=np.int64)] = True
    rows = np.repeat(np.arange(n), np.diff(np.asarray(indptr, dtype=np.int64)))
    cols = np.asarray(indices, dtype=np.int64)
    if g is not None:
        e = np.where(isd, np.asarray(g, dtype=np.float64), 0.0)
        b = b - sp.csr_matrix((data, indices, indptr), shape=(n, n)) @ e
    keep = ~(isd[rows] | isd[cols])
    data = np.where(keep, data, 0.0)
    data[(rows == cols) & isd[rows]] += 1.0  # the appended (d, d, 1) triplets, summed into the slot
    b = b.copy()
    b[isd] = 0.0 if g is None else np.asarray(g, dtype=np.float64)[isd]
    return System(np.asarray(indptr), np.asarray(indices), data, b, isd, n)


def compact_csr(indptr, indices, data):
    """``compress_eager``'s selection (jno/utils/solver/fem_utils.py:4083-4087) on a CSR in plan
    order: keep the entries with ``abs(data) > 0`` (exact zeros and NaN go), order unchanged."""
    indptr = np.asarray(indptr, dtype=np.int64)
    keep = np.abs(np.asarray(data)) > 0.0
    rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
    counts = np.bincount(rows[keep], minlength=indptr.size - 1)
    new_ptr = np.zeros(indptr.size, dtype=np.int64)
    np.cumsum(counts, out=new_ptr[1:])
    return new_ptr.astype(np.int32), np.asarray(indices)[keep].astype(np.int32), np.asarray(data)[keep]


def compact(system):
    """``compress_eager`` operator of an assembled system as a scipy CSR (non-parametric route)."""
    ip, ind, dat = compact_csr(system.indptr, system.indices, system.data)
    return sp.csr_matrix((dat, ind, ip), shape=(system.n, system.n))


def matrix_diagonal(system):
    """Sum of the on-diagonal stored entries per row."""
    rows = np.repeat(np.arange(system.n), np.diff(system.indptr))
    on = rows == system.indices
    return np.bincount(rows[on], weights=system.data[on], minlength=system.n)


def jacobi_inverse(d):
    """``1 / where(|d| > 1e-30, d, 1)``."""
    safe = np.where(np.abs(d) > 1e-30, d, 1.0)
    return 1.0 / safe
