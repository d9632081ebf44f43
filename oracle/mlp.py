"""CPU restatement of the learned cost model's network, in float64 numpy.

TEST INFRASTRUCTURE ONLY.  Imported by tests/ as the checker of the K7
kernels (hs_mlp_*); the product never imports it.  The reference has no
learned model, so this restates the textbook algorithms the kernels follow:
a ReLU multilayer perceptron in -> 64 -> 64 -> 64 -> 1, its mean-squared-error
gradient by backpropagation, and Adam (Kingma & Ba 2015, Algorithm 1, with the
bias-corrected step).  It is pinned by finite differences
(tests/test_oracle.py) rather than by reference vectors.

Flat parameter layout (matches include/hisv.h): W1 (64 x in) b1 W2 b2 W3 b3
W4 (64) b4, weights row-major W[out][in].
"""
from __future__ import annotations

import numpy as np

H = 64


def num_params(d: int) -> int:
    return H * d + H + 2 * (H * H + H) + H + 1


def unpack(p: np.ndarray, d: int):
    p = np.asarray(p, dtype=np.float64)
    o = 0

    def take(n, shape):
        nonlocal o
        v = p[o:o + n].reshape(shape)
        o += n
        return v

    w1 = take(H * d, (H, d)); b1 = take(H, (H,))
    w2 = take(H * H, (H, H)); b2 = take(H, (H,))
    w3 = take(H * H, (H, H)); b3 = take(H, (H,))
    w4 = take(H, (H,)); b4 = take(1, (1,))
    assert o == p.size
    return w1, b1, w2, b2, w3, b3, w4, b4


def forward(p, x, d=None):
    x = np.asarray(x, dtype=np.float64)
    d = x.shape[1] if d is None else d
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(p, d)
    h1 = np.maximum(x @ w1.T + b1, 0)
    h2 = np.maximum(h1 @ w2.T + b2, 0)
    h3 = np.maximum(h2 @ w3.T + b3, 0)
    return h3 @ w4 + b4[0], (x, h1, h2, h3)


def loss_and_grad(p, x, y):
    """Mean squared error (1/n) sum (f(x_i) - y_i)^2 and its gradient."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n, d = x.shape
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(p, d)
    f, (x, h1, h2, h3) = forward(p, x, d)
    r = f - y
    loss = float(np.mean(r * r))
    df = 2.0 * r / n
    gw4 = h3.T @ df
    gb4 = np.array([df.sum()])
    dz3 = np.outer(df, w4) * (h3 > 0)
    gw3 = dz3.T @ h2
    gb3 = dz3.sum(0)
    dz2 = (dz3 @ w3) * (h2 > 0)
    gw2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ w2) * (h1 > 0)
    gw1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3.ravel(), gb3, gw4, gb4])
    return loss, g


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (in place on p, m, v); step counts from 1."""
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    p -= lr * mh / (np.sqrt(vh) + eps)
    return p
