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


def _train(ctx, mode="knn", r=2.0, k=16, seeds=range(20, 26), epochs=15):
    import torch
    fs, ts = [], []
    for s in seeds:
        p = torch.from_numpy(_cloud(s)).cuda()
        f, t = ctx.collect_training(p, None, mode, r, k)
        fs.append(f)
        ts.append(t)
    f = torch.cat(fs)
    t = torch.cat(ts)
    perm = torch.randperm(f.shape[0], device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
    return ctx.train_model(f[perm].contiguous(), t[perm].contiguous(), epochs=epochs,
                           batch=8192, lr=3e-3, seed=1)


def test_training_reduces_loss_and_learned_search_is_exact(ctx):
    import torch
    losses = _train(ctx)
    # normalised targets: predicting their mean scores 0.5; training must beat it and improve
    assert losses[-1] < losses[0] and losses[-1] < 0.45, losses
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


def test_escalating_fallback_stays_exact(ctx):
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
    """The shell-count features of the width model (N_0..N_2 box counts around a query's
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
