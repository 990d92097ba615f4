"""Autotuner for the batched persistent PCG schedule (tile size x blocks per SM).

Each candidate runs the real batched solve once as a warm-up and then ``reps`` (default 3) timed
times (CUDA events); the candidate with the smallest median is kept and cached in a JSON file
(``$JNO_B200_TUNE_CACHE``, default ``~/.cache/jno_b200/tune.json``) keyed by the device name, the
library version and the batch's size signature, so later runs skip the search.
"""

import json
import os
import statistics

import torch

from . import _lib

CANDIDATES = [(t, b) for t in (32, 64, 128, 256, 512) for b in (1, 2)]


def _cache_path():
    return os.environ.get("JNO_B200_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "jno_b200",
                                                              "tune.json"))


def _load():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def signature(batch):
    name = torch.cuda.get_device_name(batch.plan.device)
    version = _lib.load().femk_version()
    return f"{name}|femk {version}|nprob={batch.nprob}|n={batch.plan.n}|nnz={batch.plan.nnz}"


def tune(batch, vals, b, inv, tol, candidates=None, reps=3):
    """Time every candidate schedule (median of ``reps`` runs after a warm-up); returns
    (best, {candidate: median ms})."""
    candidates = CANDIDATES if candidates is None else candidates
    plan = batch.plan
    times = {}
    for tile_rows, bps in candidates:
        plan.pcg_batched(batch.row_off, vals, b, None, inv, tol, 0.0, 20_000, tile_rows, bps)  # warm-up
        runs = []
        for _ in range(max(1, reps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            plan.pcg_batched(batch.row_off, vals, b, None, inv, tol, 0.0, 20_000, tile_rows, bps)
            e1.record()
            torch.cuda.synchronize()
            runs.append(e0.elapsed_time(e1))
        times[(tile_rows, bps)] = statistics.median(runs)
    best = min(times, key=times.get)
    # leave the plan holding the chosen schedule's graph and tile tables (the last trial's otherwise),
    # so the caller's first solve does not rebuild them
    plan.pcg_batched(batch.row_off, vals, b, None, inv, tol, 0.0, 20_000, best[0], best[1])
    return {"tile_rows": best[0], "blocks_per_sm": best[1], "ms": times[best]}, times


def batched_schedule(batch, vals, b, inv, tol):
    """Cached schedule for this batch signature, tuning on first use."""
    cache = _load()
    key = signature(batch)
    if key in cache:
        return cache[key]
    best, times = tune(batch, vals, b, inv, tol)
    best["tried"] = {f"{t}x{bps}": ms for (t, bps), ms in times.items()}
    cache[key] = best
    _store(cache)
    return best
