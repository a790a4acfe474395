"""Learned partition: the hand-written MLP kernels against the FP64 oracle, training on
the GPU, and exactness / gain of learned widths -- needs a B200."""
import numpy as np
import pytest

import oracle
import rtnn_b200
from oracle import mlp as omlp
from rtnn_b200 import workloads as wl

pytestmark = pytest.mark.gpu

F, H, NORM = omlp.F, omlp.H, omlp.NORM


def _params(seed):
    rng = np.random.default_rng(seed)
    n = NORM + H * F + H + H * H + H + H + 1
    P = np.zeros(n, np.float32)
    P[:F] = rng.normal(0, 1, F)
    P[F:2 * F] = rng.uniform(0.5, 2.0, F)
    P[2 * F] = rng.normal()
    P[2 * F + 1] = rng.uniform(0.5, 2.0)
    P[NORM:] = rng.normal(0, 0.3, n - NORM)
    return P


def _batch(seed, n):
    rng = np.random.default_rng(seed + 100)
    X = rng.normal(0, 1.5, (n, F)).astype(np.float32)
    t = rng.normal(0, 1.0, n).astype(np.float32)
    return X, t


def test_model_size(ctx):
    assert ctx.model_size() == NORM + H * F + H + H * H + H + H + 1


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_gradient_matches_fp64_oracle(ctx, seed):
    import torch
    P = _params(seed)
    X, t = _batch(seed, 3000)
    g, loss = ctx.mlp_loss_grad(torch.from_numpy(P).cuda(), torch.from_numpy(X).cuda(),
                                torch.from_numpy(t).cuda())
    l_ref, g_ref = omlp.loss_grad(P, X, t)
    g = g.cpu().numpy().astype(np.float64)
    # FP32 accumulation over 3000 samples: relative error against the gradient scale
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 2e-4 * scale, np.abs(g - g_ref).max() / scale
    assert abs(float(loss.item()) - l_ref) <= 1e-4 * abs(l_ref)


def test_forward_matches_fp64_oracle(ctx):
    import torch
    P = _params(3)
    X, _ = _batch(3, 5000)
    y = ctx.mlp_forward(torch.from_numpy(P).cuda(), torch.from_numpy(X).cuda()).cpu().numpy()
    y_ref = omlp.forward(P, X)
    assert np.abs(y - y_ref).max() <= 1e-4 * max(1.0, np.abs(y_ref).max())


def test_adam_step_matches_oracle(ctx):
    import torch
    P = _params(4)
    X, t = _batch(4, 500)
    _, g_ref = omlp.loss_grad(P, X, t)
    nt = g_ref.size
    tP = torch.from_numpy(P.copy()).cuda()
    tg = torch.from_numpy(g_ref.astype(np.float32)).cuda()
    m = torch.zeros(nt, device="cuda")
    v = torch.zeros(nt, device="cuda")
    Pr, mr, vr = P.astype(np.float64), np.zeros(nt), np.zeros(nt)
    for step in (1, 2, 3):
        ctx.mlp_adam_step(tP, tg, m, v, 1e-2, step, 1.0 / 500)
        Pr, mr, vr = omlp.adam(Pr, g_ref.astype(np.float32), mr, vr, 1e-2, step, 1.0 / 500)
    assert np.abs(tP.cpu().numpy() - Pr).max() <= 1e-5
    assert np.array_equal(tP.cpu().numpy()[:NORM], P[:NORM])  # normalisation is not trained


def _cloud(seed, n=200_000):
    """Surface cloud dense enough that most queries have K = 16 neighbors within r = 2."""
    return wl.surfaces(n=n, n_spheres=4, n_quads=4, box=100.0, seed=seed)


@pytest.fixture(params=[0, 1], ids=["per_query", "per_tile"])
def kind(request, ctx):
    """The width model's bucket: 0 a width per query before the sort, 1 a width per tile
    inside the search (rtnn_tuning.width_model); restored after the test."""
    base = ctx.tuning().as_dict()
    ctx.set_tuning(**{**base, "width_model": request.param})
    yield request.param
    ctx.set_tuning(**base)


def _train(ctx, mode="knn", r=2.0, k=16, seeds=range(20, 26), epochs=15, n=200_000):
    import torch
    fs, ts = [], []
    for s in seeds:
        p = torch.from_numpy(_cloud(s, n)).cuda()
        f, t = ctx.collect_training(p, None, mode, r, k)
        fs.append(f)
        ts.append(t)
    f = torch.cat(fs)
    t = torch.cat(ts)
    perm = torch.randperm(f.shape[0], device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
    return ctx.train_model(f[perm].contiguous(), t[perm].contiguous(), epochs=epochs,
                           batch=8192 if ctx.tuning().width_model == 0 else 1024, lr=3e-3, seed=1)


def test_training_reduces_loss_and_learned_search_is_exact(ctx, kind):
    import torch
    losses = _train(ctx, epochs=15 if kind == 0 else 40)
    # normalised targets: predicting their mean scores 0.5; training must beat it and improve
    # (the per-tile target, the largest K-th distance of 32 queries, is the noisier one)
    assert losses[-1] < losses[0] and losses[-1] < (0.45 if kind == 0 else 0.49), losses
    P = ctx.get_model()
    assert np.isfinite(P).all()
    p = _cloud(2, 60_000)
    exp = oracle.grid_search(p, None, "knn", 2.0, 16)
    st = rtnn_b200.Stats()
    got = ctx.search(p, None, "knn", 2.0, 16, learned=True, sorted_rows=True, stats=st)
    assert np.array_equal(got, exp)
    assert st.n_fallback < 0.5 * p.shape[0]
    # the loaded model round-trips through the C ABI
    ctx.set_model(P)
    assert np.array_equal(ctx.get_model(), P)


def test_escalating_fallback_stays_exact(ctx, kind):
    """Widths far too small force queries through every doubling pass and the final
    full-radius pass; rows stay identical to the oracle."""
    import torch
    _train(ctx, epochs=4)
    base = ctx.tuning().as_dict()
    try:
        for margin, passes in ((0.05, 4), (0.2, 1), (0.2, 0), (3.0, 6)):
            ctx.set_tuning(**{**base, "width_margin": margin, "fallback_passes": passes})
            p, q = wl.gmm(scale=0.02, seed=11)
            st = rtnn_b200.Stats()
            got = ctx.search(p, q, "knn", 10.0, 5, learned=True, sorted_rows=True, stats=st)
            assert np.array_equal(got, oracle.grid_search(p, q, "knn", 10.0, 5)), (margin, passes)
            if margin < 1:
                assert st.n_fallback > 0
    finally:
        ctx.set_tuning(**base)


def test_learned_widths_are_tighter_than_analytic(ctx):
    """What the trained network gains over the analytic rule: on held-out clouds its
    widths enclose a smaller search volume, with few queries needing the fallback."""
    import torch
    _train(ctx)
    p = torch.from_numpy(_cloud(3)).cuda()
    wa = ctx.query_widths(p, None, "knn", 2.0, 16, learned=False)
    wlrn = ctx.query_widths(p, None, "knn", 2.0, 16, learned=True)
    vol_a = float((wa.double() ** 3).mean())
    vol_l = float((wlrn.double() ** 3).mean())
    st = rtnn_b200.Stats()
    ctx.search(p, None, "knn", 2.0, 16, learned=True, stats=st)
    fb_rate = st.n_fallback / p.shape[0]
    print(f"mean search volume analytic {vol_a:.3f} learned {vol_l:.3f}, fallback {fb_rate:.3%}")
    assert vol_l < vol_a
    assert fb_rate < 0.25


def test_width_features_match_oracle_box_counts(ctx):
    """The per-query model's shell-count features (N_0..N_2 box counts around a query's
    cell) equal the oracle's counts on the same grid (cell and origin from the search)."""
    import torch
    p = wl.uniform_cube(20000, 30.0, seed=12)
    tp = torch.from_numpy(p).cuda()
    st = rtnn_b200.Stats()
    ctx.search(tp, None, "knn", 2.0, 16, partition=True, stats=st)
    f, _ = ctx.collect_training(tp, None, "knn", 2.0, 16)
    f = f.cpu().numpy()
    assert f.shape == (p.shape[0], rtnn_b200.MODEL_FEATURES)
    cell = np.float32(st.cell_size)
    dims = np.array(list(st.grid_dims))
    o = p.min(0).astype(np.float32)
    inv = np.float32(1) / cell
    ci = np.clip(np.floor((p - o) * inv), 0, dims - 1).astype(np.int64)
    counts = np.zeros(dims[::-1], dtype=np.uint32)
    np.add.at(counts, (ci[:, 2], ci[:, 1], ci[:, 0]), 1)
    for i in range(0, p.shape[0], 37):
        N = oracle.box_counts(counts, *ci[i], shells=3).astype(np.float64)
        exp = np.log1p([N[0], N[1] - N[0], N[2] - N[1]])
        assert np.allclose(f[i, [0, 1, 2]], exp, atol=1e-5), (i, f[i], N)
        assert abs(f[i, 3] - (np.log(17.0) - np.log1p(N[2]))) <= 1e-5


def test_tile_features_and_targets_match_the_oracle(ctx):
    """One training sample per 32-query tile of the plain search: the shell-count features
    (N_0..N_2 box counts around the cell of the tile box's centre) equal the oracle's counts
    on the same grid (cell and origin from the search), the extent and cell features follow
    the tile's box, and the target is log(largest K-th neighbor distance / cell) from the
    oracle's rows."""
    import torch
    n, k, r = 20000, 16, 2.0
    p = wl.uniform_cube(n, 30.0, seed=12)
    tp = torch.from_numpy(p).cuda()
    st = rtnn_b200.Stats()
    ctx.search(tp, None, "knn", r, k, stats=st)
    base = ctx.tuning().as_dict()
    ctx.set_tuning(**{**base, "width_model": 1})
    try:
        f, t = ctx.collect_training(tp, None, "knn", r, k)
    finally:
        ctx.set_tuning(**base)
    _, qo = ctx.layout(n, n)   # the sorted order of that plain search: tile t = rows 32t..
    f, t = f.cpu().numpy(), t.cpu().numpy()
    assert f.shape == ((n + 31) // 32, rtnn_b200.MODEL_FEATURES) and t.shape == (f.shape[0],)
    cell = np.float32(st.cell_size)
    dims = np.array(list(st.grid_dims))
    o = p.min(0).astype(np.float32)
    inv = np.float32(1) / cell
    ci = np.clip(np.floor((p - o) * inv), 0, dims - 1).astype(np.int64)
    counts = np.zeros(dims[::-1], dtype=np.uint32)
    np.add.at(counts, (ci[:, 2], ci[:, 1], ci[:, 0]), 1)
    rows = oracle.grid_search(p, None, "knn", r, k)
    for tile in range(0, f.shape[0], 23):
        q = p[qo[32 * tile:32 * tile + 32].astype(np.int64)]
        lo, hi = q.min(0), q.max(0)
        centre = (np.float32(0.5) * (lo + hi)).astype(np.float32)
        c = np.clip(np.floor((centre - o) * inv), 0, dims - 1).astype(np.int64)
        N = oracle.box_counts(counts, *c, shells=3).astype(np.float64)
        exp = np.log1p([N[0], N[1] - N[0], N[2] - N[1]])
        assert np.allclose(f[tile, [0, 1, 2]], exp, atol=1e-5), (tile, f[tile], N)
        assert abs(f[tile, 3] - (np.log(k + 1.0) - np.log1p(N[2]))) <= 1e-5
        assert abs(f[tile, 4] - np.log(float(cell) / r)) <= 1e-5
        ext = float((hi - lo).max()) * float(inv)
        assert abs(f[tile, 5] - np.log1p(ext)) <= 1e-4
        qi = qo[32 * tile:32 * tile + 32].astype(np.int64)
        last = rows[qi, k - 1]
        have = last >= 0
        if have.any():
            d = np.sqrt(((p[qi[have]] - p[last[have]]) ** 2).sum(1)).max()
            assert abs(t[tile] - np.log(d / float(cell))) <= 1e-4, (tile, t[tile])
        else:
            assert abs(t[tile] - np.log(1.5 * r / float(cell))) <= 1e-5


def test_learned_tile_widths_cover_most_queries(ctx):
    """With per-tile widths the search uses one width per tile (bucket): every query of a
    tile gets the same width, below r where the data is dense (clouds four times denser
    than the other tests', about 0.8 r for the 16th neighbor), and the share of queries
    that need the wider fallback stays small."""
    import torch
    base = ctx.tuning().as_dict()
    ctx.set_tuning(**{**base, "width_model": 1})
    try:
        _tile_widths_check(ctx, torch)
    finally:
        ctx.set_tuning(**base)


def _tile_widths_check(ctx, torch):
    _train(ctx, epochs=40, n=800_000, seeds=range(20, 23))
    p = torch.from_numpy(_cloud(4, 800_000)).cuda()
    w = ctx.query_widths(p, None, "knn", 2.0, 16, learned=True).cpu().numpy()
    _, qo = ctx.layout(p.shape[0], p.shape[0])
    ws = w[qo.astype(np.int64)]
    tiles = ws[: (ws.size // 32) * 32].reshape(-1, 32)
    assert (tiles == tiles[:, :1]).all()
    assert np.median(ws) < 2.0
    # the search's warp-wide MLP gives the width the inference kernel predicts from the
    # same tile's features (the plain search forms the same tiles)
    f, _ = ctx.collect_training(p, None, "knn", 2.0, 16)
    st0 = rtnn_b200.Stats()
    ctx.search(p, None, "knn", 2.0, 16, stats=st0)
    y = ctx.mlp_forward(torch.from_numpy(ctx.get_model()).cuda(), f.contiguous()).cpu().numpy()
    margin = ctx.tuning().width_margin
    exp_w = np.minimum(margin * st0.cell_size * np.exp(np.minimum(y, 30.0)), 2.0)
    got_w = ws[0::32][: exp_w.size]
    assert np.allclose(got_w, exp_w[: got_w.size], rtol=1e-4, atol=1e-6)
    st = rtnn_b200.Stats()
    ctx.search(p, None, "knn", 2.0, 16, learned=True, stats=st)
    assert st.n_fallback < 0.25 * p.shape[0]


def test_widths_off_is_the_plain_search(ctx):
    """width_model 2 switches the learned widths off: a learned search (a model loaded)
    takes every query at the full radius -- no escalation, the plain search's rows and its
    launch count -- and the widths the learned search reports are all r."""
    import torch
    base = ctx.tuning().as_dict()
    try:
        ctx.set_tuning(**{**base, "width_model": 0})
        _train(ctx, epochs=2, seeds=range(20, 22), n=50_000)
        ctx.set_tuning(**{**base, "width_model": 2})
        p = _cloud(3, 60_000)
        exp = oracle.grid_search(p, None, "knn", 2.0, 16)
        st, sp = rtnn_b200.Stats(), rtnn_b200.Stats()
        got = ctx.search(p, None, "knn", 2.0, 16, learned=True, sorted_rows=True, stats=st)
        assert np.array_equal(got, exp)
        ctx.search(p, None, "knn", 2.0, 16, sorted_rows=True, stats=sp)
        assert st.n_fallback == 0 and st.n_launches == sp.n_launches
        w = ctx.query_widths(torch.from_numpy(p).cuda(), None, "knn", 2.0, 16, learned=True)
        assert bool((w.cpu() == 2.0).all())
    finally:
        ctx.set_tuning(**base)


@pytest.mark.parametrize("clip", [2, 8, 16])
def test_width_clip_stays_exact(ctx, clip):
    """rtnn_tuning.width_clip: the widest per-query widths of a tile run are clipped to the
    next widest; a clipped query that finds fewer than K is escalated, so the rows equal the
    oracle's, and no fewer queries are escalated than without the clip."""
    base = ctx.tuning().as_dict()
    try:
        ctx.set_tuning(**{**base, "width_model": 0, "width_clip": 0})
        _train(ctx, epochs=3, seeds=range(20, 23), n=60_000)
        p = _cloud(4, 80_000)
        exp = oracle.grid_search(p, None, "knn", 2.0, 16)
        st0, st = rtnn_b200.Stats(), rtnn_b200.Stats()
        ctx.search(p, None, "knn", 2.0, 16, learned=True, stats=st0)
        ctx.set_tuning(**{**base, "width_model": 0, "width_clip": clip})
        for kw in ({"learned": True}, {"partition": True}):
            got = ctx.search(p, None, "knn", 2.0, 16, sorted_rows=True, stats=st, **kw)
            assert np.array_equal(got, exp)
        got = ctx.search(p, None, "knn", 2.0, 16, learned=True, stats=st)
        assert_sets = np.sort(np.where(got < 0, 1 << 30, got), 1)
        assert np.array_equal(assert_sets, np.sort(np.where(exp < 0, 1 << 30, exp), 1))
        assert st.n_fallback >= st0.n_fallback
        # the radius mode and the multi-cloud path with the clip
        r_exp = oracle.grid_search(p, None, "radius", 1.5, 32)
        assert np.array_equal(ctx.search(p, None, "radius", 1.5, 32, partition=True,
                                         sorted_rows=True), r_exp)
        q, off = wl.multicloud(n_clouds=12, lo=64, hi=3000, seed=9)
        got = ctx.search_batched(q, off, mode="knn", radius=0.2, k=32, sorted_rows=True,
                                 partition=True)
        assert np.array_equal(got, oracle.grid_search_batched(q, off, mode="knn", r=0.2, k=32))
    finally:
        ctx.set_tuning(**base)
