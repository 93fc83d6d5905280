"""Test infrastructure: a NumPy restatement of the coupling predictor's
perceptron (fribois2d_b200/csrc/mlp.cu) used to check the CUDA kernels'
outputs and gradients.

Parameter layout: [W1 (64 x n_in) b1 (64) W2 (64 x 64) b2 (64) W3 (n_out x 64)
b3 (n_out)], W[out][in] row-major; tanh hidden layers; loss = mean over the
samples of the summed squared output errors.  Computed in float64 here; the
device computes in float32.
"""
from __future__ import annotations

import numpy as np

H = 64


def unpack(p: np.ndarray, n_in: int, n_out: int):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * n_in].reshape(H, n_in); o += H * n_in
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + n_out * H].reshape(n_out, H); o += n_out * H
    b3 = p[o:o + n_out]; o += n_out
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward(p, x, n_out):
    x = np.asarray(x, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p, x.shape[1], n_out)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h1, h2, h2 @ W3.T + b3


def loss_and_grad(p, x, t):
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    n_out = t.shape[1]
    W1, b1, W2, b2, W3, b3 = unpack(p, x.shape[1], n_out)
    h1, h2, y = forward(p, x, n_out)
    B = x.shape[0]
    e = y - t
    loss = float(np.sum(e * e) / B)
    dy = 2.0 * e / B
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ W3) * (1.0 - h2 * h2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
