"""GPU: the batched persistent PCG against per-problem oracle solves (same iteration, jax cg
semantics per problem), and the schedule autotuner."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import assemble as oa  # noqa: E402
from oracle import mesh as om  # noqa: E402
from oracle import pcg as op  # noqa: E402


def _problems(sides):
    out = []
    for i, n in enumerate(sides):
        pts, tets = om.equi_distant_box(n, n, n)
        pts = om.jitter_interior(pts, n, n, n, seed=100 + i)
        out.append((pts, tets, om.logk_field(len(tets), 500 + i)))
    return out


@pytest.mark.parametrize("tile_rows,bps", [(32, 2), (64, 1), (2048, 2)])
def test_batched_matches_per_problem_oracle(tile_rows, bps):
    from jno_b200.batch import BatchedPoisson

    sides = [3, 5, 1, 8, 4, 6, 2, 12]
    probs = _problems(sides)
    batch = BatchedPoisson([(p, t) for p, t, _ in probs])
    vals, b = batch.assemble([lk for _, _, lk in probs])
    x, it, rel = batch.solve(vals, b, tol=1e-8, schedule={"tile_rows": tile_rows, "blocks_per_sm": bps})
    xs = batch.split(x)
    for k, (pts, tets, lk) in enumerate(probs):
        bnd = om.boundary_nodes(tets, 1)
        s = oa.assemble(pts, tets, 1, bnd, np.exp(lk))
        xo, ito, _ = op.pcg(s.csr(), s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-8)
        assert abs(int(it[k]) - ito) <= 1, (k, it[k], ito)
        nx = max(np.linalg.norm(xo), 1e-300)
        assert np.linalg.norm(xs[k] - xo) <= 1e-7 * nx + 1e-300, k
        if np.linalg.norm(s.b) > 0:
            assert rel[k] <= 2e-8
    assert it[2] == 0  # a single voxel has no interior DOF: b = 0, no iteration


def test_autotuner_caches_a_schedule(tmp_path, monkeypatch):
    from jno_b200 import tuner
    from jno_b200.batch import BatchedPoisson

    monkeypatch.setenv("JNO_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(tuner, "CANDIDATES", [(64, 1), (128, 2)])
    probs = _problems([4, 7, 3])
    batch = BatchedPoisson([(p, t) for p, t, _ in probs])
    vals, b = batch.assemble([lk for _, _, lk in probs])
    inv = batch.plan.jacobi(vals)
    sched = tuner.batched_schedule(batch, vals, b, inv, 1e-8)
    assert (sched["tile_rows"], sched["blocks_per_sm"]) in [(64, 1), (128, 2)]
    assert set(sched["tried"]) == {"64x1", "128x2"}
    assert tuner.batched_schedule(batch, vals, b, inv, 1e-8) == sched  # served from the cache


def test_batched_replay_is_bitwise_reproducible():
    """The second solve replays the captured graph; the reductions have a fixed order, so the
    result is bit-identical."""
    from jno_b200.batch import BatchedPoisson

    probs = _problems([5, 9, 3, 7])
    batch = BatchedPoisson([(p, t) for p, t, _ in probs])
    vals, b = batch.assemble([lk for _, _, lk in probs])
    sched = {"tile_rows": 64, "blocks_per_sm": 2}
    x1, it1, rel1 = batch.solve(vals, b, schedule=sched)
    x2, it2, rel2 = batch.solve(vals, b, schedule=sched)
    assert torch.equal(x1, x2) and np.array_equal(it1, it2) and np.array_equal(rel1, rel2)


@pytest.mark.parametrize("tile_rows,bps", [(32, 2), (64, 2), (2048, 1)])
def test_batched_mixed_reaches_the_fp64_stop_rule(tile_rows, bps):
    """The mixed-precision batched solve: every problem's FP64 residual meets the 1e-8 stop rule,
    each solution is within 1e-6 of the per-problem FP64 oracle, the large problems take FP64
    reliable updates, and the graph replay is bit-identical. Tiles of 32 and 64 rows run the FP32
    products and the update phase through the shared-memory rings; 2048-row tiles run direct loads."""
    from jno_b200.batch import BatchedPoisson

    sides = [3, 5, 1, 8, 4, 6, 2, 12, 16]
    probs = _problems(sides)
    batch = BatchedPoisson([(p, t) for p, t, _ in probs])
    vals, b = batch.assemble([lk for _, _, lk in probs])
    sched = {"tile_rows": tile_rows, "blocks_per_sm": bps}
    x, it, rel = batch.solve(vals, b, tol=1e-8, schedule=sched, precision="mixed")
    outer = batch.last_outer.copy()
    xs = batch.split(x)
    for k, (pts, tets, lk) in enumerate(probs):
        bnd = om.boundary_nodes(tets, 1)
        s = oa.assemble(pts, tets, 1, bnd, np.exp(lk))
        if np.linalg.norm(s.b) == 0:
            assert it[k] == 0 and np.all(xs[k] == 0)
            continue
        xo, ito, _ = op.pcg(s.csr(), s.b, oa.jacobi_inverse(oa.matrix_diagonal(s)), tol=1e-12)
        assert rel[k] <= 1e-8, (k, rel[k])
        assert np.linalg.norm(xs[k] - xo) <= 1e-6 * np.linalg.norm(xo), k
        assert outer[k] >= 1
    assert outer[-1] >= 2  # the 16^3 problem needs FP64 reliable updates to reach 1e-8
    x2, it2, rel2 = batch.solve(vals, b, tol=1e-8, schedule=sched, precision="mixed")
    assert torch.equal(x, x2) and np.array_equal(it, it2)


def test_grid_barrier_wait_runs_out_and_the_context_survives():
    """Failure detection without a GPU fault: with the plan option test_skip_arrival = 0, block 0 of
    the persistent batched launch does not arrive at its first grid barrier, so every other block
    waits out barrier_limit_ms (5 ms here), raises the barrier's timeout word and returns; the call
    reports FEMK_TIMEOUT within a bounded time. The same plan then solves with femk_pcg, and a plan of
    the same batch without the option solves the batch: the context is intact."""
    import time

    from jno_b200 import _lib
    from jno_b200.batch import BatchedPoisson

    probs = _problems([4, 4])
    meshes = [(p, t) for p, t, _ in probs]
    logk = [lk for _, _, lk in probs]
    bad = BatchedPoisson(meshes, options={"test_skip_arrival": 0, "barrier_limit_ms": 5.0})
    vals, b = bad.assemble(logk)
    inv = bad.plan.jacobi(vals)
    t0 = time.perf_counter()
    with pytest.raises(_lib.FemkError) as err:
        bad.plan.pcg_batched(bad.row_off, vals, b, None, inv, 1e-8, 0.0, 1000, 32, 1)
    assert err.value.status == _lib.FEMK_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    x, it, rel, st = bad.plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
    assert st == 0 and rel <= 2e-8
    good = BatchedPoisson(meshes)
    vg, bg = good.assemble(logk)
    xg, itg, relg = good.solve(vg, bg, tol=1e-8, schedule={"tile_rows": 32, "blocks_per_sm": 1})
    assert np.all(relg <= 2e-8)
    assert torch.linalg.norm(xg - x) <= 1e-7 * torch.linalg.norm(x)
