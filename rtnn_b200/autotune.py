"""Autotuner for the search pipeline.

Picks the tuning knobs of a context (include/rtnn.h, rtnn_tuning) for one workload by
timing candidate settings on the GPU with the library's own event timers, one knob at a
time (coordinate descent): the cell edge (points per cell for dense clouds, cell/radius
ratio), the search block size (warps per block), and -- for the learned partition -- the
width margin and the number of doubling fallback passes. Choices are cached in a JSON file
keyed by a workload signature (sizes, cloud count, mode, r, K, flags, GPU name), so later
runs of the same kind of workload skip the search.

The cached file lives at $RTNN_AUTOTUNE_CACHE, else ~/.cache/rtnn_b200/autotune.json.
"""
import json
import math
import os

import numpy as np

import rtnn_b200

GRID_KNOBS = [
    ("points_per_cell", [0.0, 1.0, 4.0, 16.0]),
    ("cell_ratio", [0.5, 1.0]),
    ("warps_per_block", [2, 4]),
    ("lane_walk_ratio", [0.0, 0.5, 1.0, 2.0]),
    ("gap_ratio", [0.0, 1.0, 2.0, 4.0]),
    ("pending_slots", [8, 16, 32, 64]),
]
LEARNED_KNOBS = [
    ("width_margin", [1.0, 1.08, 1.15, 1.25, 1.4]),
    ("fallback_passes", [2, 4, 6]),
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
             partition=False, learned=False, knobs=None, use_cache=True, log=None):
    """Tunes `ctx` for this workload (CUDA tensors, host offset arrays). Returns the
    chosen tuning as a dict and leaves it set on the context."""
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
