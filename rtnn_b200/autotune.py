"""Autotuner for the search pipeline.

Replaces the reference's fixed rules for the same choices: the cell/radius ratio derived
from free GPU memory (calcCRRatio, util.cpp:551-676, used at util.cpp:680-688) and the
partition cost model that groups queries into batches (autoBatchingRange /
autoBatchingKNN, sort.cpp:221-320); here the choices are timed on the caller's data.

Picks the tuning knobs of a context (include/rtnn.h, rtnn_tuning) for one workload by
timing candidate settings on the GPU with the library's own event timers, one knob at a
time (coordinate descent) after timing a few whole cell-size presets: the cell edge
(points per cell for dense clouds, cell/radius ratio), the search kernels (tiles or one
warp per query, block size, run splitting, result-column slots), and -- for the learned
partition -- the width margin and the number of escalation passes. Choices are cached in a JSON file
keyed by a workload signature (sizes, cloud count, mode, r, K, flags, GPU name), so later
runs of the same kind of workload skip the search.

The cached file lives at $RTNN_AUTOTUNE_CACHE, else ~/.cache/rtnn_b200/autotune.json.
"""
import json
import math
import os

import numpy as np

import rtnn_b200

# knobs that change the grid (and so the learned model's input features)
CELL_KNOBS = [
    ("points_per_cell", [0.0, 0.125, 0.25, 1.0, 4.0, 16.0]),
    ("cell_ratio", [0.125, 0.25, 0.5, 1.0]),
]
# knobs of the search kernels only
SEARCH_KNOBS = [
    ("warps_per_block", [2, 4]),
    ("lane_walk_ratio", [0.0, 0.5, 1.0, 2.0]),
    ("gap_ratio", [0.0, 1.0, 2.0, 4.0]),
    ("pending_slots", [8, 16, 32, 64]),
    ("query_warps", [0, 1, 2, 3]),
]
GRID_KNOBS = CELL_KNOBS + SEARCH_KNOBS
# whole cell-size regimes tried as starting points: one knob at a time would not move from
# coarse cells with tiles to fine cells with per-query escalation passes
GRID_PRESETS = [
    {"cell_ratio": 0.5, "min_cell_ratio": 0.0625, "points_per_cell": 1.0, "query_warps": 0},
    {"cell_ratio": 0.25, "min_cell_ratio": 0.02, "points_per_cell": 0.25, "query_warps": 2},
    {"cell_ratio": 0.125, "min_cell_ratio": 0.01, "points_per_cell": 0.125, "query_warps": 2},
    {"cell_ratio": 1.0, "min_cell_ratio": 0.0625, "points_per_cell": 4.0, "query_warps": 0},
]
# the learned widths are per tile (the search's bucket), so the analytic partition's
# width buckets (buckets_per_halving) do not apply
LEARNED_KNOBS = [
    ("width_margin", [0.8, 0.9, 1.0, 1.05, 1.1, 1.15, 1.25]),
    ("fallback_passes", [2, 4, 6]),
    ("width_clip", [0, 2, 4, 8]),
]


def cache_path():
    p = os.environ.get("RTNN_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "rtnn_b200", "autotune.json")


def signature(n_points, n_queries, n_clouds, mode, radius, k, learned, partition):
    import torch
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    b = lambda x: int(math.log2(max(int(x), 1)))
    return (f"{dev}|p2^{b(n_points)}|q2^{b(n_queries)}|c2^{b(n_clouds)}|{mode}|r{radius:g}|k{k}"
            f"|{'learned' if learned else 'partition' if partition else 'plain'}")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(d):
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
    except OSError:
        pass


def time_plan(ctx, points, offsets, queries, qoffsets, out, repeats=2, **plan_kw):
    """Mean device time (ms) of a non-graph plan execution after one warm-up."""
    plan = ctx.plan(offsets, qoffsets, use_graph=False, **plan_kw)
    try:
        plan.execute(points, queries, out)
        ms = []
        for _ in range(repeats):
            st = rtnn_b200.Stats()
            plan.execute(points, queries, out, stats=st)
            ms.append(st.ms_total)
        return float(np.mean(ms))
    finally:
        plan.close()


def autotune(ctx, points, offsets, queries=None, qoffsets=None, mode="knn", radius=0.2, k=32,
             partition=False, learned=False, knobs=None, presets=None, use_cache=True, log=None):
    """Tunes `ctx` for this workload (CUDA tensors, host offset arrays). Returns the
    chosen tuning as a dict and leaves it set on the context. `presets` (partial tunings)
    are timed first and the best one is the starting point of the descent."""
    import torch
    offsets = np.asarray(offsets, dtype=np.uint64)
    n_clouds = len(offsets) - 1
    nq = int(offsets[-1]) if queries is None else int(np.asarray(qoffsets)[-1])
    sig = signature(int(offsets[-1]), nq, n_clouds, mode, radius, k, learned, partition)
    cache = _load() if use_cache else {}
    if sig in cache:
        ctx.set_tuning(**cache[sig]["tuning"])
        return cache[sig]["tuning"]
    knobs = knobs if knobs is not None else (GRID_KNOBS + (LEARNED_KNOBS if learned else []))
    out = torch.empty((nq, k), dtype=torch.int32, device=points.device)
    kw = dict(mode=mode, radius=radius, k=k, partition=partition, learned=learned)
    best = ctx.tuning().as_dict()
    best_ms = time_plan(ctx, points, offsets, queries, qoffsets, out, **kw)
    trials = [(dict(best), best_ms)]
    for pre in presets or []:
        cand = {**best, **pre}
        try:
            ctx.set_tuning(**cand)
        except rtnn_b200.RtnnError:
            continue
        ms = time_plan(ctx, points, offsets, queries, qoffsets, out, **kw)
        trials.append((dict(cand), ms))
        if log:
            log(f"autotune preset {pre}: {ms:.3f} ms (best {best_ms:.3f})")
        if ms < best_ms:
            best, best_ms = cand, ms
    ctx.set_tuning(**best)
    for name, values in knobs:
        for v in values:
            if best.get(name) == v:
                continue
            cand = dict(best)
            cand[name] = v
            try:
                ctx.set_tuning(**cand)
            except rtnn_b200.RtnnError:
                continue
            ms = time_plan(ctx, points, offsets, queries, qoffsets, out, **kw)
            trials.append((dict(cand), ms))
            if log:
                log(f"autotune {name}={v}: {ms:.3f} ms (best {best_ms:.3f})")
            if ms < best_ms:
                best, best_ms = cand, ms
        ctx.set_tuning(**best)
    cache[sig] = {"tuning": best, "ms": best_ms, "trials": len(trials)}
    if use_cache:
        _save(cache)
    return best


WIDTH_MODELS = [0, 1]   # rtnn_tuning.width_model: per query before the sort, per tile in the search
OFF = 2                 # rtnn_tuning.width_model: learned widths switched off (full radius)
MARGINS = [0.9, 1.0, 1.05, 1.1, 1.15, 1.25]
CLIPS = [0, 4, 8]


def autotune_learned(ctx, points, offsets, queries=None, qoffsets=None, mode="knn", radius=0.2,
                     k=32, train=None, presets=None, width_models=None, log=None):
    """Tuning for the learned partition. The width model's features depend on the grid and
    on the kind of bucket, so for every cell-size preset and both kinds (width_model 0: a
    width per query before the sort; 1: a width per 32-query tile inside the search) the
    model is trained at that setting (`train(ctx)` collects training data and trains; what
    it returns is handed back for the chosen setting) and the width margin and the width
    clip are tuned. The fastest setting keeps its model; then the search and learned knobs,
    which leave the grid alone, are tuned by descent. Last, that setting is timed against
    the widths switched off (width_model 2, the starting tuning: the plain search's) and the
    faster is kept. Returns (tuning, train's result for the chosen setting plus "widths":
    "on" or "off" and both times)."""
    import torch
    offsets = np.asarray(offsets, dtype=np.uint64)
    nq = int(offsets[-1]) if queries is None else int(np.asarray(qoffsets)[-1])
    out = torch.empty((nq, k), dtype=torch.int32, device=points.device)
    kw = dict(mode=mode, radius=radius, k=k, learned=True)
    start = ctx.tuning().as_dict()
    best = None
    for pre in presets if presets is not None else GRID_PRESETS:
        for kind in width_models if width_models is not None else WIDTH_MODELS:
            ctx.set_tuning(**{**start, **pre, "width_model": kind})
            info = train(ctx)
            # the margin and the width clip interact (a clip trades box size for escalations),
            # so both are tuned for every setting before the settings are compared
            tun = autotune(ctx, points, offsets, queries, qoffsets,
                           knobs=[("width_margin", MARGINS), ("width_clip", CLIPS)],
                           use_cache=False, log=log, **kw)
            ms = time_plan(ctx, points, offsets, queries, qoffsets, out, **kw)
            if log:
                log(f"autotune learned preset {pre} width_model {kind}: {ms:.3f} ms")
            if best is None or ms < best[0]:
                best = (ms, tun, ctx.get_model(), info)
    _, tun, model, info = best
    ctx.set_tuning(**tun)
    ctx.set_model(model)
    tun = autotune(ctx, points, offsets, queries, qoffsets, knobs=SEARCH_KNOBS + LEARNED_KNOBS,
                   use_cache=False, log=log, **kw)
    ms_on = time_plan(ctx, points, offsets, queries, qoffsets, out, **kw)
    # the widths switched off (width_model 2: every query at the full radius, the starting
    # tuning's grid and kernels) where narrowing cannot pay -- most K-th distances at r, or
    # a grid whose cells already fit the balls -- so the learned search never loses to the
    # plain one; the model stays loaded
    off = {**start, "width_model": OFF}
    ctx.set_tuning(**off)
    ms_off = time_plan(ctx, points, offsets, queries, qoffsets, out, **kw)
    if log:
        log(f"autotune learned widths on: {ms_on:.3f} ms, off: {ms_off:.3f} ms")
    if ms_off < ms_on:
        info = {**(info or {}), "widths": "off", "ms_on": ms_on, "ms_off": ms_off}
        return off, info
    ctx.set_tuning(**tun)
    info = {**(info or {}), "widths": "on", "ms_on": ms_on, "ms_off": ms_off}
    return tun, info


def grid_of(tuning):
    """The cell-size part of a tuning, as a preset (e.g. the plain search's tuned grid)."""
    keys = ("cell_ratio", "min_cell_ratio", "points_per_cell", "query_warps")
    return {n: tuning[n] for n in keys}
