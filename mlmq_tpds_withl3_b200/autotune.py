"""Autotuner for the queue configuration (delta, work blocks, warps per CTA).

The reference picks its queue type and delta with a fixed rule on degree and
weight statistics (core/include/adaptive.h:64-115) and disables it in the
timed path; this tuner instead measures: it times a few candidate
configurations on probe sources of the actual graph and keeps the fastest.
Every candidate gives the same exact distances (ordering changes only the
amount of work), so tuning never affects results.

Results are persisted per graph class (kind, log2 n, rounded average degree
and log2 average weight) in a JSON file, $MLMQ_TUNE_CACHE or
~/.cache/mlmq_b200/tune.json.
"""
import json
import math
import os
import time

import numpy as np

from ._lib import default_config
from .solver import Solver


def graph_class(hg, kind="graph"):
    info = hg.info()
    return (f"{kind}:n2^{int(round(math.log2(max(hg.n, 1))))}"
            f":deg{int(round(info.avg_nnz))}:w2^{int(round(math.log2(max(info.avg_weight, 1))))}")


def _cache_path():
    return os.environ.get("MLMQ_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "mlmq_b200", "tune.json"))


def load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store_cache(key, value):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache = load_cache()
        cache[key] = value
        with open(path + ".tmp", "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)
    except OSError:
        pass


def delta_candidates(hg, around=200000):
    """Bucket widths from a few multiples of the mean weight up to `around`."""
    avg_w = max(1.0, float(hg.info().avg_weight))
    cands = {int(around)}
    for k in (2, 4, 8, 16, 32, 64):
        cands.add(max(1, int(avg_w * k)))
    return sorted(c for c in cands if c <= 4 * around)


def _time_solve(solver, src, reps=2):
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        solver.solve(src)
        best = min(best, time.perf_counter() - t0)
    return best


def tune(dgraph, hg, probe_sources, kind="graph", around=200000, use_cache=True,
         extra=None):
    """Returns (config, report).  Candidates: delta from delta_candidates(),
    then warps per CTA in {8, 16, 24} at the best delta, then 1, 2 or 4
    relaxation rounds in flight, then vertex tiles on or off, then the L1
    run-ahead bound, then the light/heavy split with bucket sync, then L2
    claims of 16 slots (they pay with the split on R-MAT, 5.4 -> 4.7 ms, and
    cost narrow-frontier solves: kNN 10.5 -> 12.3 ms)."""
    key = graph_class(hg, kind)
    base = dict(extra or {})
    if use_cache:
        hit = load_cache().get(key)
        if hit:
            return default_config(**{**hit["config"], **base}), {"cached": key, **hit}
    probe = list(probe_sources)[:2]
    results = []

    def measure(over):
        s = Solver(dgraph, {**base, **over})
        try:
            s.solve(probe[0])  # warm-up
            t = sum(_time_solve(s, src) for src in probe)
        finally:
            s.close()
        results.append({"config": over, "seconds": t})
        return t

    best_d = min(delta_candidates(hg, around), key=lambda d: measure({"delta": d}))
    best = {"delta": best_d}
    best_t = min(r["seconds"] for r in results if r["config"] == best)
    for wpb in (8, 24):
        over = {"delta": best_d, "warps_per_block": wpb}
        t = measure(over)
        if t < best_t:
            best, best_t = over, t
    # Relaxation rounds in flight per warp (default 4), then the adjacency
    # layout (vertex tiles, default on) at the best shape.
    for extra_opt in ({"relax_unroll": 1}, {"relax_unroll": 2}, {"vertex_tiles": 0},
                      {"l1_ahead": 0}, {"l1_ahead": 16}):
        over = {**best, **extra_opt}
        t = measure(over)
        if t < best_t:
            best, best_t = over, t
    # The light/heavy split with bulk-synchronous buckets, at the best delta
    # and a quarter of it (the split pays where many arcs are heavy), on the
    # shape found so far and on the default one: the stages above are
    # greedy, and a shape picked without the split (more warps per CTA) can
    # be the wrong one with it.
    if best.get("vertex_tiles", 1):
        shapes = [best, {"delta": best["delta"]}]
        for shape in shapes[:1] if shapes[0] == shapes[1] else shapes:
            for dl in (shape["delta"], max(1, shape["delta"] // 4)):
                over = {**shape, "light_heavy": 1, "bucket_sync": 1, "delta": dl}
                t = measure(over)
                if t < best_t:
                    best, best_t = over, t
    over = {**best, "l2_batch": 16}
    t = measure(over)
    if t < best_t:
        best, best_t = over, t
    report = {"key": key, "config": best, "seconds": best_t, "trials": results}
    if use_cache:
        store_cache(key, {"config": best, "seconds": best_t})
    return default_config(**{**best, **base}), report


# Settings every batched or served candidate shares unless told otherwise.
BATCH_BASE = {"warps_per_block": 8, "l2_cap_log2": 20, "l2_batch": 16, "bucket_max": 2}


def tune_batch(queries, max_vertices, candidates=None, base=None):
    """Times one batched launch of `queries` ([(DeviceGraph, source)]) per
    candidate configuration (bucket width, L1 top-up, run-ahead bound,
    relaxation rounds, light/heavy split with bucket sync) and returns
    (config, report) for the fastest; `base` holds the settings every
    candidate shares (default: 8 worker warps per CTA, 2^20-slot rings per
    query -- smaller rings divert wide buckets to L3 -- and L2 claims of 16
    slots from a 2-bucket window: with every warp busy, a warp's top-up read
    is a chain of claim atomics and slot loads, and fewer, larger claims
    shorten it; 64 queries on a 4896^2 grid went 248 -> 213 ms).  A batch
    keeps every warp busy, so it is bound by records relaxed per warp
    iteration rather than by one query's chain of dependent hops, and its
    best setting differs from a single solve's (the L1 top-up, which fills a
    warp from L2 when its own L1 holds few records, pays off only here).
    Every candidate gives the same exact distances."""
    from .batch import BatchSolver
    base = dict(base or BATCH_BASE)
    if candidates is None:
        candidates = [{"delta": d, "relax_unroll": 2, "topup": t}
                      for d in (25000, 50000, 100000, 200000) for t in (16, 32)]
        candidates += [{"delta": 50000, "relax_unroll": 4, "topup": 16},
                       {"delta": 50000, "relax_unroll": 2, "topup": 16, "l1_ahead": 8}]
        candidates += [{"delta": d, "relax_unroll": 2, "topup": 32, "light_heavy": 1,
                        "bucket_sync": 1} for d in (25000, 50000, 100000)]
    results = []
    n_max = max(g.n for g, _ in queries)
    for over in candidates:
        # the light/heavy split needs n more vertex slots (heavy records)
        mv = max_vertices + (n_max if over.get("light_heavy", base.get("light_heavy", 0)) else 0)
        b = BatchSolver(len(queries), mv, {**base, **over})
        try:
            b.run(queries)  # warm-up
            t0 = time.perf_counter()
            b.run(queries)
            t = time.perf_counter() - t0
        finally:
            b.close()
        results.append({"config": over, "seconds": t})
    best = min(results, key=lambda r: r["seconds"])
    return default_config(**{**base, **best["config"]}), {"config": best["config"],
                                                          "seconds": best["seconds"],
                                                          "trials": results}


def median_ms(times):
    return float(np.median(np.asarray(times))) * 1e3
