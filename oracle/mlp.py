"""ORACLE — test infrastructure only (the checker, never the product).

The learned deflection network (2 -> 64 -> 64 -> 1, tanh) in numpy FP64:
forward pass and the gradient of the mean squared error by hand-written
backpropagation, for checking the device training kernels.  Parameter
layout: W1[64][2], b1[64], W2[64][64], b2[64], W3[64], b3 (4417 values).
"""
from __future__ import annotations

import numpy as np

H = 64
N_PARAMS = 4417


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[0:128].reshape(H, 2)
    b1 = p[128:192]
    W2 = p[192:192 + H * H].reshape(H, H)
    b2 = p[4288:4352]
    W3 = p[4352:4416]
    b3 = p[4416]
    return W1, b1, W2, b2, W3, b3


def forward(p: np.ndarray, x: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64).reshape(-1, 2)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3 + b3


def loss_and_grad(p: np.ndarray, x: np.ndarray, y: np.ndarray) -> tuple[float, np.ndarray]:
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64).reshape(-1, 2)
    y = np.asarray(y, dtype=np.float64)
    n = x.shape[0]
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    out = h2 @ W3 + b3
    e = out - y
    loss = float(np.mean(e * e))
    dout = 2.0 * e / n
    g = np.zeros(N_PARAMS)
    g[4352:4416] = dout @ h2
    g[4416] = dout.sum()
    d2 = np.outer(dout, W3) * (1.0 - h2 * h2)
    g[192:192 + H * H] = (d2.T @ h1).ravel()
    g[4288:4352] = d2.sum(axis=0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    g[0:128] = (d1.T @ x).ravel()
    g[128:192] = d1.sum(axis=0)
    return loss, g
