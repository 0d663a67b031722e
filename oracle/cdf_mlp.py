"""CPU restatement of the learned-splitter CDF network (TEST INFRASTRUCTURE ONLY).

The network and its loss are this project's (the reference has no learned
path); this module restates them in float64 numpy so that the GPU training
kernel's gradients can be checked against an independent implementation.

    u(z) = sigmoid(w3 . tanh(W2 tanh(W1 z + b1) + b2) + b3),  hidden width 32
    loss = sum over valid samples (u(z) - target)^2 / n_valid

Parameter vector layout (1153 floats): W1[32], b1[32], W2[32*32] (row = output
unit), b2[32], w3[32], b3.
"""
from __future__ import annotations

import numpy as np

H = 32
P = 4 * H + H * H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[0:H]
    b1 = p[H:2 * H]
    W2 = p[2 * H:2 * H + H * H].reshape(H, H)
    b2 = p[2 * H + H * H:3 * H + H * H]
    w3 = p[3 * H + H * H:4 * H + H * H]
    b3 = p[4 * H + H * H]
    return W1, b1, W2, b2, w3, b3


def forward(p, z):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    z = np.asarray(z, dtype=np.float64)
    h1 = np.tanh(np.outer(z, W1) + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return 1.0 / (1.0 + np.exp(-(h2 @ w3 + b3)))


def loss_and_grad(p, z, u):
    """Loss and gradient; samples with u < 0 are ignored (mask)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    z = np.asarray(z, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    valid = u >= 0
    nv = max(1, int(valid.sum()))
    a1 = np.outer(z, W1) + b1
    h1 = np.tanh(a1)
    a2 = h1 @ W2.T + b2
    h2 = np.tanh(a2)
    o = h2 @ w3 + b3
    uh = 1.0 / (1.0 + np.exp(-o))
    diff = np.where(valid, uh - u, 0.0)
    loss = float((diff ** 2).sum())
    g = 2.0 * diff * uh * (1.0 - uh) / nv          # dL/do (mean over valid)
    dw3 = h2.T @ g
    db3 = g.sum()
    da2 = np.outer(g, w3) * (1.0 - h2 ** 2)
    dW2 = da2.T @ h1
    db2 = da2.sum(axis=0)
    da1 = (da2 @ W2) * (1.0 - h1 ** 2)
    dW1 = da1.T @ z
    db1 = da1.sum(axis=0)
    grad = np.concatenate([dW1, db1, dW2.ravel(), db2, dw3, [db3]])
    return loss, grad


def mse(p, z, u):
    valid = np.asarray(u) >= 0
    nv = max(1, int(valid.sum()))
    d = np.where(valid, forward(p, z) - u, 0.0)
    return float((d ** 2).sum()) / nv
