"""numpy float64 restatement of the learned criterion's MLP (8 -> 64 -> 64 ->
1, ReLU) and of its pinball-loss gradient: the checker of the training and
inference kernels. Parameter layout of FLN_MLP_PARAMS in include/fln.h."""
import numpy as np

from fastlinkingnumbers_b200 import _native as N

IN, H = 8, 64
W1, B1 = 0, IN * H
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H


def _unpack(p):
    p = p.astype(np.float64)
    return (p[W1:B1].reshape(IN, H), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3])


def mlp_loss_grad(p, X, T, q):
    """Mean pinball loss at quantile q and its gradient, float64."""
    w1, b1, w2, b2, w3, b3 = _unpack(p)
    X = X.astype(np.float64)
    T = T.astype(np.float64)
    a1 = X @ w1 + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w2 + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ w3 + b3
    e = T - y
    n = len(T)
    loss = np.mean(np.where(e >= 0, q * e, (q - 1) * e))
    dy = np.where(e > 0, -q, 1 - q) / n
    g = np.zeros(N.MLP_PARAMS)
    g[W3:B3] = h2.T @ dy
    g[B3] = dy.sum()
    d2 = (a2 > 0) * (dy[:, None] * w3[None, :])
    g[W2:B2] = (h1.T @ d2).ravel()
    g[B2:W3] = d2.sum(0)
    d1 = (a1 > 0) * (d2 @ w2.T)
    g[W1:B1] = (X.T @ d1).ravel()
    g[B1:W2] = d1.sum(0)
    return loss, g


def mlp_forward(p, X):
    w1, b1, w2, b2, w3, b3 = _unpack(p)
    h1 = np.maximum(X.astype(np.float64) @ w1 + b1, 0)
    h2 = np.maximum(h1 @ w2 + b2, 0)
    return h2 @ w3 + b3


def _init(rng):
    p = np.zeros(N.MLP_PARAMS, dtype=np.float32)
    p[W1:B1] = rng.normal(0, np.sqrt(2 / IN), IN * H)
    p[B1:W2] = rng.normal(0, 0.1, H)
    p[W2:B2] = rng.normal(0, np.sqrt(2 / H), H * H)
    p[B2:W3] = rng.normal(0, 0.1, H)
    p[W3:B3] = rng.normal(0, np.sqrt(1 / H), H)
    p[B3] = -4.0
    return p


def _features(rng, n):
    """Random rows in the ranges of the real features (s, radius ratio, two
    scaled logs, four moment ratios)."""
    # Ranges of the real features: s, radius ratio, two scaled logs, four ratios.
    X = np.stack([rng.uniform(0.8, 2.6, n), rng.uniform(0, 1, n), rng.uniform(-3, 0, n),
                  rng.uniform(-4, -1, n), rng.uniform(0, 2, n), rng.uniform(0, 2, n),
                  rng.uniform(0, 4, n), rng.uniform(0, 4, n)], axis=1)
    return X.astype(np.float32)
