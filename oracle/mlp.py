"""CPU reference of the learned switch's network (test infrastructure only):
an 8 -> 32 -> 32 -> 3 MLP with ReLU and softmax cross-entropy over the packed
parameter layout of libxbfs (mean 8, std 8, W1 32x8, b1 32, W2 32x32, b2 32,
W3 3x32, b3 3). Used to check the device forward pass and the gradients of
xbfs_mlp_grad. Double precision, written from the definitions.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT = 8, 32, 3


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0

    def take(n, shape=None):
        nonlocal o
        a = w[o:o + n]
        o += n
        return a.reshape(shape) if shape else a

    mean, std = take(N_IN), take(N_IN)
    W1, b1 = take(N_H * N_IN, (N_H, N_IN)), take(N_H)
    W2, b2 = take(N_H * N_H, (N_H, N_H)), take(N_H)
    W3, b3 = take(N_OUT * N_H, (N_OUT, N_H)), take(N_OUT)
    return mean, std, W1, b1, W2, b2, W3, b3


def forward(w, feats):
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(w)
    x = (np.asarray(feats, dtype=np.float64) - mean) / std
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    out = h2 @ W3.T + b3
    return x, z1, h1, z2, h2, out


def loss_and_grad(w, feats, labels):
    """Mean cross-entropy and its gradient w.r.t. the trainable parameters
    (everything after the 16 normalisation constants), in packed order."""
    mean, std, W1, b1, W2, b2, W3, b3 = unpack(w)
    x, z1, h1, z2, h2, out = forward(w, feats)
    n = len(labels)
    m = out.max(axis=1, keepdims=True)
    e = np.exp(out - m)
    p = e / e.sum(axis=1, keepdims=True)
    y = np.asarray(labels)
    loss = -np.log(np.maximum(p[np.arange(n), y], 1e-30)).mean()
    d = p.copy()
    d[np.arange(n), y] -= 1.0
    d /= n
    gW3 = d.T @ h2
    gb3 = d.sum(axis=0)
    dh2 = (d @ W3) * (z2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(axis=0)
    dh1 = (dh2 @ W2) * (z1 > 0)
    gW1 = dh1.T @ x
    gb1 = dh1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
