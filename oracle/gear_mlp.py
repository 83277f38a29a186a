"""CPU oracle of the learned gear controller network (test infrastructure).

16 -> 64 -> 64 -> 4 MLP, ReLU hidden, loss (1/B) sum mask (y - t)^2,
forward / backward written out by hand in numpy (float64), plus a
central-difference gradient check.  No reference counterpart exists (the
reference's gear logic is thresholds + hysteresis); this pins the CUDA
kernels' arithmetic.
"""
from __future__ import annotations

import numpy as np

IN, H, OUT = 16, 64, 4
SIZES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (OUT, H)), ("b3", (OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shp in SIZES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SIZES])


def forward(p, x):
    P = unpack(p)
    a1 = x @ P["W1"].T + P["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ P["W2"].T + P["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ P["W3"].T + P["b3"]
    return y, (h1, h2)


def loss(p, x, t, mask=None):
    y, _ = forward(p, x)
    m = np.ones_like(t) if mask is None else mask
    return float((m * (y - t) ** 2).sum() / x.shape[0])


def backward(p, x, t, mask=None):
    P = unpack(p)
    B = x.shape[0]
    y, (h1, h2) = forward(p, x)
    m = np.ones_like(t) if mask is None else mask
    dy = 2.0 * m * (y - t) / B
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dh2 = (dy @ P["W3"]) * (h2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ P["W2"]) * (h1 > 0)
    g["W1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return pack(g)


def numeric_grad(p, x, t, mask=None, idx=None, eps=1e-6):
    idx = range(len(p)) if idx is None else idx
    g = np.zeros(len(p))
    for i in idx:
        q = np.array(p, dtype=np.float64)
        q[i] += eps
        lp = loss(q, x, t, mask)
        q[i] -= 2 * eps
        lm = loss(q, x, t, mask)
        g[i] = (lp - lm) / (2 * eps)
    return g


def init(seed=0):
    rng = np.random.default_rng(seed)
    d = {"W1": rng.standard_normal((H, IN)) * np.sqrt(2 / IN), "b1": np.zeros(H),
         "W2": rng.standard_normal((H, H)) * np.sqrt(2 / H), "b2": np.zeros(H),
         "W3": rng.standard_normal((OUT, H)) * np.sqrt(1 / H), "b3": np.zeros(OUT)}
    return pack(d)
