"""ORACLE — test infrastructure only. A float64 numpy restatement of the
closure MLP's training arithmetic (flowcraft_b200/csrc/mlp_train.cu):
5 -> 32 -> 32 -> 1 with ReLU and a linear output, mean-squared-error loss
and its gradient with respect to the flat parameter vector
(w1[5*32], b1[32], w2[32*32], b2[32], w3[32], b3). Checked against finite
differences by the tests before it checks the CUDA gradients."""
from __future__ import annotations

import numpy as np

N_IN, H = 5, 32
SIZES = [("w1", N_IN * H), ("b1", H), ("w2", H * H), ("b2", H), ("w3", H), ("b3", 1)]
N_PARAMS = sum(n for _, n in SIZES)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, o = {}, 0
    for name, n in SIZES:
        out[name] = p[o:o + n]
        o += n
    out["w1"] = out["w1"].reshape(N_IN, H)
    out["w2"] = out["w2"].reshape(H, H)
    return out


def forward(p, x):
    q = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ q["w1"] + q["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ q["w2"] + q["b2"]
    h2 = np.maximum(z2, 0)
    return h2 @ q["w3"] + q["b3"][0], (z1, h1, z2, h2)


def loss_grad(p, x, y):
    """(mean squared error, gradient) in float64."""
    q = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    out, (z1, h1, z2, h2) = forward(p, x)
    n = len(x)
    e = out - y
    d = 2.0 * e / n
    g3 = h2.T @ d
    gb3 = d.sum()
    dz2 = np.outer(d, q["w3"]) * (z2 > 0)
    g2 = h1.T @ dz2
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ q["w2"].T) * (z1 > 0)
    g1 = x.T @ dz1
    gb1 = dz1.sum(0)
    grad = np.concatenate([g1.ravel(), gb1, g2.ravel(), gb2, g3, [gb3]])
    return float((e * e).mean()), grad
