"""FP64 numpy restatement of the width MLP -- TEST INFRASTRUCTURE ONLY.

Checks the hand-written CUDA forward / backward / Adam kernels of the learned
partition (6 -> 16 -> 16 -> 1, ReLU; parameter layout of include/rtnn_learn.h). The
reference has no learned model (its widths come from calcSearchSize, grid.cu:84-211), so
this restatement is pinned against finite differences instead of reference outputs.
"""
import numpy as np

F = 6
H = 16
NORM = 2 * F + 2


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    in_mean, in_std = P[:F], P[F:2 * F]
    out_mean, out_std = P[2 * F], P[2 * F + 1]
    T = P[NORM:]
    o = 0
    W1 = T[o:o + H * F].reshape(H, F); o += H * F
    b1 = T[o:o + H]; o += H
    W2 = T[o:o + H * H].reshape(H, H); o += H * H
    b2 = T[o:o + H]; o += H
    W3 = T[o:o + H]; o += H
    b3 = T[o]
    return in_mean, in_std, out_mean, out_std, W1, b1, W2, b2, W3, b3


def forward_norm(P, X):
    in_mean, in_std, _, _, W1, b1, W2, b2, W3, b3 = unpack(P)
    xn = (np.asarray(X, np.float64) - in_mean) / in_std
    a1 = xn @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    o = h2 @ W3 + b3
    return o, (xn, a1, h1, a2, h2)


def forward(P, X):
    _, _, out_mean, out_std = unpack(P)[:4]
    return forward_norm(P, X)[0] * out_std + out_mean


def loss_grad(P, X, t):
    """Sum over samples of 0.5 * (o - t_n)^2 and its gradient w.r.t. the trained
    parameters (same layout and order as the CUDA kernel)."""
    in_mean, in_std, out_mean, out_std, W1, b1, W2, b2, W3, b3 = unpack(P)
    o, (xn, a1, h1, a2, h2) = forward_norm(P, X)
    tn = (np.asarray(t, np.float64) - out_mean) / out_std
    err = o - tn
    loss = 0.5 * float((err ** 2).sum())
    gb3 = err.sum()
    gW3 = (err[:, None] * h2).sum(0)
    dh2 = err[:, None] * W3[None, :] * (a2 > 0)
    gb2 = dh2.sum(0)
    gW2 = dh2.T @ h1
    dh1 = (dh2 @ W2) * (a1 > 0)
    gb1 = dh1.sum(0)
    gW1 = dh1.T @ xn
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, grad


def adam(P, g, m, v, lr, step, scale, b1=0.9, b2=0.999, eps=1e-8):
    P = np.array(P, np.float64)
    g = np.asarray(g, np.float64) * scale
    m = b1 * np.asarray(m, np.float64) + (1 - b1) * g
    v = b2 * np.asarray(v, np.float64) + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    P[NORM:] -= lr * mh / (np.sqrt(vh) + eps)
    return P, m, v
