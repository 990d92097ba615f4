"""Many independent P1 Poisson problems of uneven size, assembled and solved together.

The problems are concatenated into one disjoint mesh (vertex ids offset per problem), so one plan,
one assembly launch and one persistent batched-PCG launch (``femk_pcg_batched``) serve all of them.
The tile size and blocks per SM of that launch come from :mod:`jno_b200.tuner`.
No reference counterpart: jNO batches only by ``vmap`` over right-hand sides
(tests/test_fem_solver_slots.py:123-132).
"""

import numpy as np
import torch

from . import _lib
from .domain import box_points_tets, jitter_interior
from .plan import FemPlan


def batched_workload(count=256, seed=42, lo=8, hi=48, amp=0.1):
    """Synthetic batch: side n_i = round(exp(U(log lo, log hi))) from ``default_rng(seed)``; problem
    i is the unit-cube Kuhn mesh of side n_i with interior jitter seed 10000 + i and log k seed
    20000 + i (N(0, 0.5^2) per tet). Returns (sides, [(points, tets, logk)])."""
    rng = np.random.default_rng(seed)
    sides = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(int)
    probs = []
    for i, n in enumerate(sides):
        pts, tets = box_points_tets(n, n, n)
        pts = jitter_interior(pts, n, n, n, seed=10_000 + i, amp=amp)
        logk = np.random.default_rng(20_000 + i).normal(0.0, 0.5, len(tets))
        probs.append((pts, tets, logk))
    return sides, probs


class BatchedPoisson:
    """``k_e grad u . grad v - f v`` with u = 0 on each problem's boundary, for a list of P1 meshes."""

    def __init__(self, meshes, options=None):
        pts, tets, row_off, tet_off = [], [], [0], [0]
        for p, t in meshes:
            tets.append(np.asarray(t, dtype=np.int64) + row_off[-1])
            pts.append(np.asarray(p, dtype=np.float64))
            row_off.append(row_off[-1] + len(p))
            tet_off.append(tet_off[-1] + len(t))
        self.row_off = np.asarray(row_off, dtype=np.int64)
        self.tet_off = np.asarray(tet_off, dtype=np.int64)
        self.plan = FemPlan(np.concatenate(pts), np.concatenate(tets), 1, options=options)
        self.nprob = len(meshes)

    def assemble(self, logk):
        """logk: concatenated per-element values (or a list per problem)."""
        if isinstance(logk, (list, tuple)):
            logk = np.concatenate([np.asarray(v, dtype=np.float64) for v in logk])
        return self.plan.assemble(logk, mode=_lib.COEF_EXP)

    def solve(self, vals, b, tol=1e-8, maxiter=20_000, schedule=None, precision="fp64"):
        """All problems to the stop rule in one launch. Returns (x, iterations, relres).

        ``precision="mixed"``: FP32 inner CG with per-problem FP64 reliable updates
        (``femk_pcg_batched_mixed``); the iterations are then the FP32 ones and ``self.last_outer``
        holds each problem's FP64 residual evaluations."""
        from .tuner import batched_schedule

        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        inv = self.plan.jacobi(vals)
        sched = schedule or batched_schedule(self, vals, b, inv, tol)
        if precision == "mixed":
            x, it, outer, rel, stv, st = self.plan.pcg_batched_mixed(
                self.row_off, vals, b, inv, None, tol, 0.0, maxiter, sched["tile_rows"], sched["blocks_per_sm"])
            self.last_outer = outer
        else:
            x, it, rel, stv, st = self.plan.pcg_batched(self.row_off, vals, b, None, inv, tol, 0.0, maxiter,
                                                        sched["tile_rows"], sched["blocks_per_sm"])
        if st != 0:
            raise RuntimeError(f"batched CG: status {st}, per-problem status {np.unique(stv)}")
        return x, it, rel

    def split(self, x):
        xs = x.cpu().numpy()
        return [xs[self.row_off[k]:self.row_off[k + 1]] for k in range(self.nprob)]
