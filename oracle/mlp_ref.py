"""FP64 CPU reference of the learned bucket scheduler's network.

Test infrastructure only: the GPU forward / backward / Adam kernels of the
engine (vine_b200/csrc/mlp.cu) are checked against these functions.  Nothing
in the product imports this module.

Network: x[16] -> ReLU(W1 x + b1)[64] -> ReLU(W2 h1 + b2)[64] -> W3 h2 + b3[2].
Flat parameter layout (the one the engine uses): W1[64][16] b1[64]
W2[64][64] b2[64] W3[2][64] b3[2].  Loss over n rows: (1/n) * sum over rows
and both outputs of (y - t)^2.  Adam (Kingma & Ba, 2015) with bias
correction, beta1 = 0.9, beta2 = 0.999, eps = 1e-8.

The reference has no learned scheduler (its bucket width follows a fixed
AR rule, algorithm/cspp.hpp); this network is the B200 engine's own
addition, so its oracle is the mathematics above rather than reference code.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 16, 64, 2
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
         ("W3", (OUT, HID)), ("b3", (OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    p = np.asarray(p, np.float64)
    assert p.size == N_PARAMS
    out, off = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = p[off:off + k].reshape(shape)
        off += k
    return out


def forward(p, x):
    """Returns (y, cache) for rows x[n, 16]."""
    w = unpack(p)
    x = np.asarray(x, np.float64).reshape(-1, IN)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w["W3"].T + w["b3"]
    return y, (x, z1, h1, z2, h2)


def loss_grad(p, x, t):
    """Mean (over rows) summed-squared error and its gradient (flat layout)."""
    w = unpack(p)
    y, (x, z1, h1, z2, h2) = forward(p, x)
    t = np.asarray(t, np.float64).reshape(-1, OUT)
    n = x.shape[0]
    e = y - t
    loss = float((e * e).sum() / n)
    dy = 2.0 * e / n
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ w["W3"]) * (z2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ w["W2"]) * (z1 > 0)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def adam_step(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update; returns (p, m, v).  `step` counts from 1."""
    p, m, v, g = (np.asarray(a, np.float64) for a in (p, m, v, g))
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    p = p - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return p, m, v
