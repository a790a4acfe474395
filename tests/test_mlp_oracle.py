"""The FP64 MLP oracle against central differences (CPU only)."""
import numpy as np

from oracle import mlp as omlp


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    n = omlp.NORM + omlp.H * omlp.F + omlp.H + omlp.H * omlp.H + omlp.H + omlp.H + 1
    P = np.zeros(n)
    P[:omlp.F] = rng.normal(0, 1, omlp.F)
    P[omlp.F:2 * omlp.F] = rng.uniform(0.5, 2.0, omlp.F)
    P[2 * omlp.F] = 0.3
    P[2 * omlp.F + 1] = 1.7
    P[omlp.NORM:] = rng.normal(0, 0.3, n - omlp.NORM)
    X = rng.normal(0, 1.5, (64, omlp.F))
    t = rng.normal(0, 1.0, 64)
    _, g = omlp.loss_grad(P, X, t)
    for i in rng.choice(g.size, 40, replace=False):
        e = np.zeros_like(P)
        e[omlp.NORM + i] = 1e-6
        num = (omlp.loss_grad(P + e, X, t)[0] - omlp.loss_grad(P - e, X, t)[0]) / 2e-6
        assert abs(num - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, num, g[i])


def test_adam_first_step_moves_by_lr():
    P = np.zeros(omlp.NORM + 4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    P2, m, v = omlp.adam(P, g, np.zeros(4), np.zeros(4), 0.1, 1, 1.0)
    # bias-corrected first step: -lr * sign(g) (g != 0)
    assert np.allclose(P2[omlp.NORM:], [-0.1, 0.1, -0.1, 0.0], atol=1e-6)
