"""CPU oracle of the warm-start MLP (TEST INFRASTRUCTURE ONLY).

A float64 numpy restatement of accelgraph_b200/csrc/ag_mlp.cu: the same
parameter layout (W1[64][8] b1[64] W2[64][64] b2[64] w3[64] b3), the forward
pass on the bfloat16 rounding of the binary32 masters (round to nearest
even), ReLU, mean squared error against the targets, and the gradient with
respect to the (bfloat16) weights.  Used only to check the GPU kernels.
"""
from __future__ import annotations

import numpy as np

IN, H = 8, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1


def bf16_round(w: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(params, X):
    W1, b1, W2, b2, w3, b3 = unpack(bf16_round(params))
    X = np.asarray(X, np.float64)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    return h2 @ w3 + b3, (X, a1, h1, a2, h2)


def gradients(params, X, T):
    W1, b1, W2, b2, w3, b3 = unpack(bf16_round(params))
    y, (X, a1, h1, a2, h2) = forward(params, X)
    n = X.shape[0]
    r = y - np.asarray(T, np.float64)
    loss = float(np.mean(r * r))
    d3 = 2.0 * r / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = h2.T @ d3
    g[OFF_B3] = d3.sum()
    dh2 = np.outer(d3, w3) * (a2 > 0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    g[OFF_W1:OFF_B1] = (dh1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    return g, loss
