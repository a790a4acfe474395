"""Full-size parity of the three large workloads -- needs a B200.

At full size the oracle cannot search every query in seconds, so each workload is checked
on a seeded subset of 1,000 queries, row for row (rows sorted by (FP32 distance, index))
against the oracle's brute force over the query's own cloud, and the same subset is run
through the reference's own check (check.cpp:20-101 KNN, :103-139 radius, compiled into
oracle/_ref/refcheck). Every workload runs on the plain grid and on the learned partition
(a width per query, and a width per tile) with the tuning the benchmark settles on for the
multi-cloud workload (fine cells, one warp per query for the escalation passes); all must
agree on every row.

  surfaces   10,000,000 surface points, queries = points, KNN K = 16, r = 2
  multicloud 4,096 clouds (54.8 M points), queries = own points, KNN K = 32, r = 0.2
  sph        52.5 M lattice + splash particles after one perturbation step, radius K = 64,
             r = 2
"""
import os

import numpy as np
import pytest

import oracle
import rtnn_b200
from rtnn_b200 import workloads as wl

pytestmark = pytest.mark.gpu

SUBSET = 1000
TUNED = dict(points_per_cell=0.125, cell_ratio=0.125, min_cell_ratio=0.01, width_margin=1.1,
             fallback_passes=2, gap_ratio=2.0, pending_slots=16, query_warps=2,
             buckets_per_halving=1.0)
THREADS = os.cpu_count() or 1


def _search_both(ctx, name, tp, offsets):
    """(plain rows, [learned rows per width model], learned stats) as CUDA tensors, rows
    sorted; the learned search runs with a width per query and with a width per tile."""
    import torch
    cfg = wl.CONFIGS[name]
    kw = dict(mode=cfg["mode"], radius=cfg["radius"], k=cfg["k"], sorted_rows=True)
    base = ctx.tuning().as_dict()
    plain = ctx.search_batched(tp, offsets, **kw)
    learned, st = [], None
    for kind in (0, 1):
        ctx.set_tuning(**{**base, **TUNED, "width_model": kind})
        wl.train_width_model(ctx, name, epochs=8,
                             count=4 if name != "knn_multicloud_4096" else 48)
        st = rtnn_b200.Stats()
        learned.append(ctx.search_batched(tp, offsets, learned=True, stats=st, **kw))
        torch.cuda.synchronize()
    ctx.set_tuning(**base)
    return plain, learned, st


def _check_subset(points, offsets, rows_sub, idx, name, refcheck_procs=THREADS):
    """rows_sub[i] = the row of query idx[i] (queries = points, global indices)."""
    cfg = wl.CONFIGS[name]
    mode, r, k = cfg["mode"], cfg["radius"], cfg["k"]
    cloud = np.searchsorted(offsets.astype(np.int64), idx, side="right") - 1
    for c in np.unique(cloud):
        sel = np.nonzero(cloud == c)[0]
        a, b = int(offsets[c]), int(offsets[c + 1])
        cp = points[a:b]
        cq = points[idx[sel]]
        exp = oracle.bruteforce(cp, cq, mode, r, k)
        exp = np.where(exp >= 0, exp + a, -1)
        got = rows_sub[sel]
        bad = np.nonzero((got != exp).any(1))[0]
        assert bad.size == 0, (f"cloud {c}: {bad.size} rows differ from the oracle, query "
                               f"{idx[sel][bad[0]]}: got {got[bad[0]].tolist()} "
                               f"exp {exp[bad[0]].tolist()}")
        local = np.where(got >= 0, got - a, -1)
        ok, log = oracle.refcheck(cp, cq, local, mode, r, k,
                                  procs=refcheck_procs if len(offsets) == 2 else 1)
        assert ok, f"reference check rejected cloud {c}: {log[-500:]}"


def _run(ctx, name, points, offsets):
    import torch
    tp = torch.from_numpy(points).cuda()
    plain, learned, st = _search_both(ctx, name, tp, offsets)
    for kind, rows in enumerate(learned):
        assert torch.equal(plain, rows), f"plain and learned rows differ (width model {kind})"
    assert st.n_queries == points.shape[0]
    idx = np.sort(np.random.default_rng(12345).choice(points.shape[0], SUBSET, replace=False))
    sub = plain[torch.from_numpy(idx).cuda()].cpu().numpy()
    del plain, learned
    torch.cuda.empty_cache()
    _check_subset(points, offsets, sub, idx, name)
    return st


def test_surfaces_1e7_full_size(ctx):
    p = wl.surfaces(seed=2)
    st = _run(ctx, "knn_surface_1e7", p, np.array([0, len(p)], np.uint64))
    assert st.n_fallback < p.shape[0]


def test_multicloud_4096_full_size(ctx):
    p, off = wl.multicloud(seed=3)
    st = _run(ctx, "knn_multicloud_4096", p, off)
    assert st.n_clouds == 4096


def test_sph_lattice_5e7_full_size(ctx):
    p = wl.sph_step(wl.sph_lattice(seed=4), seed=5)
    _run(ctx, "sph_lattice_5e7", p, np.array([0, len(p)], np.uint64))
