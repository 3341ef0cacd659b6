"""CPU oracle of the autotuner's cost model (test infrastructure only).

A float64 numpy restatement of the perceptron that libtcs.so trains on the GPU
(threadcoarsenedstencilgenerator_b200/csrc/tcs_mlp.cu): three linear layers n_in -> H -> H -> 1
with ReLU after the first two, mean-squared-error loss, and Adam (Kingma & Ba, "Adam: A Method
for Stochastic Optimization", 2015) with bias correction.  The parameter packing is the library's:
W1 [n_in x H], b1 [H], W2 [H x H], b2 [H], W3 [H], b3.  The reference project has no learned
component; this module is the checker of the engine's own kernels.
"""

from __future__ import annotations

import numpy as np


def param_count(n_in: int, hidden: int) -> int:
    return n_in * hidden + hidden + hidden * hidden + hidden + hidden + 1


def unpack(p: np.ndarray, n_in: int, hidden: int):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + n_in * hidden].reshape(n_in, hidden); o += n_in * hidden
    b1 = p[o:o + hidden]; o += hidden
    W2 = p[o:o + hidden * hidden].reshape(hidden, hidden); o += hidden * hidden
    b2 = p[o:o + hidden]; o += hidden
    W3 = p[o:o + hidden]; o += hidden
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def forward(p, x, n_in: int, hidden: int) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(p, n_in, hidden)
    x = np.asarray(x, dtype=np.float64)
    a1 = np.maximum(x @ W1 + b1, 0.0)
    a2 = np.maximum(a1 @ W2 + b2, 0.0)
    return a2 @ W3 + b3


def gradient(p, x, t, n_in: int, hidden: int):
    """(loss, packed gradient) of mean((forward(x) - t)^2)."""
    W1, b1, W2, b2, W3, b3 = unpack(p, n_in, hidden)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    n = x.shape[0]
    a1 = np.maximum(x @ W1 + b1, 0.0)
    a2 = np.maximum(a1 @ W2 + b2, 0.0)
    y = a2 @ W3 + b3
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    gW3 = a2.T @ dy
    gb3 = dy.sum()
    d2 = np.outer(dy, W3) * (a2 > 0)
    gW2 = a1.T @ d2
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2.T) * (a1 > 0)
    gW1 = x.T @ d1
    gb1 = d1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g


def adam(p, g, m, v, step: int, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One bias-corrected Adam update; returns (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
