"""ORACLE -- test infrastructure only.

Float64 restatement of the cost model's network and loss, to check the CUDA
kernels' forward pass and gradients (tempi_mlp_predict, tempi_mlp_grad):
12 -> 64 -> 64 -> 23 with ReLU, masked mean squared error.  Parameter layout
per member: W1[64][12] b1[64] W2[64][64] b2[64] W3[23][64] b3[23].
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 12, 64, 23
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (OUT, HID)), ("b3", (OUT,))]
P = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(p):
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[off: off + n], np.float64).reshape(shape)
        off += n
    return out


def flatten(d):
    return np.concatenate([d[name].ravel() for name, _ in SHAPES])


def forward(p, x):
    w = unflatten(p)
    x = np.asarray(x, np.float64)
    a1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(a2, 0)
    o = h2 @ w["W3"].T + w["b3"]
    return o, (x, h1, h2)


def loss_and_grad(p, x, y, mask=None):
    """Masked mean squared error and its gradient (flat, float64)."""
    w = unflatten(p)
    o, (x, h1, h2) = forward(p, x)
    y = np.asarray(y, np.float64)
    m = np.ones_like(y) if mask is None else np.asarray(mask, np.float64)
    cnt = m.sum()
    inv = 1.0 / cnt if cnt > 0 else 0.0
    d = o - y
    loss = float((m * d * d).sum() * inv)
    do = 2.0 * m * d * inv
    g = {"W3": do.T @ h2, "b3": do.sum(0)}
    d2 = (do @ w["W3"]) * (h2 > 0)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ w["W2"]) * (h1 > 0)
    g["W1"] = d1.T @ x
    g["b1"] = d1.sum(0)
    return loss, flatten(g)


def init(seed=0):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            r = 1.0 / np.sqrt(shape[1])
            d[name] = rng.uniform(-r, r, shape)
        else:
            d[name] = np.zeros(shape)
    return flatten(d)
