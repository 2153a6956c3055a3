"""Float64 CPU reference of the cost-model MLP (TEST INFRASTRUCTURE ONLY).

Same parameter blob as the device kernels in csrc/costmodel.cu:
[mean 4][std 4][W1 64x4][b1 64][W2 64x64][b2 64][W3 kx64][b3 k], every W
row-major (output, input).  loss = mean over masked entries of (y - t)^2.
Used by tests/ to check the device gradients and predictions.
"""
from __future__ import annotations

import numpy as np

F, H = 4, 64


def unpack(p: np.ndarray, k: int):
    p = np.asarray(p, np.float64)
    o = 0

    def take(n, shape=None):
        nonlocal o
        v = p[o:o + n]
        o += n
        return v.reshape(shape) if shape else v

    mean, std = take(F), take(F)
    W1, b1 = take(H * F, (H, F)), take(H)
    W2, b2 = take(H * H, (H, H)), take(H)
    W3, b3 = take(k * H, (k, H)), take(k)
    assert o == len(p)
    return mean, std, W1, b1, W2, b2, W3, b3


def param_count(k: int) -> int:
    return 2 * F + H * F + H + H * H + H + k * H + k


def forward(p, k, X):
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(p, k)
    x = (np.asarray(X, np.float64) - mean) / std
    z1 = x @ W1.T + b1
    a1 = np.maximum(z1, 0)
    z2 = a1 @ W2.T + b2
    a2 = np.maximum(z2, 0)
    y = a2 @ W3.T + b3
    return y, (x, z1, a1, z2, a2)


def loss_and_grad(p, k, X, T, M):
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(p, k)
    y, (x, z1, a1, z2, a2) = forward(p, k, X)
    m = (np.asarray(M) != 0).astype(np.float64)
    cnt = m.sum()
    diff = (y - np.asarray(T, np.float64)) * m
    loss = (diff ** 2).sum() / cnt
    dy = 2 * diff / cnt
    gW3 = dy.T @ a2
    gb3 = dy.sum(0)
    dz2 = (dy @ W3) * (z2 > 0)
    gW2 = dz2.T @ a1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([np.zeros(2 * F), gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
