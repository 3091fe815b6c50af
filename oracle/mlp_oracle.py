"""TEST INFRASTRUCTURE ONLY: CPU restatement (numpy, float64) of the sensor
MLP of libacfd_gpu -- forward pass, weighted binary cross-entropy, its
gradient by back-propagation, and the Adam update -- used to check the
library's training kernels.  Parameter layout: W1[32][10], b1[32], W2[32][32],
b2[32], w3[32], b3."""
from __future__ import annotations

import numpy as np

N_IN, N_H = 10, 32


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + N_H * N_IN].reshape(N_H, N_IN); o += N_H * N_IN
    b1 = p[o:o + N_H]; o += N_H
    W2 = p[o:o + N_H * N_H].reshape(N_H, N_H); o += N_H * N_H
    b2 = p[o:o + N_H]; o += N_H
    w3 = p[o:o + N_H]; o += N_H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    z = h2 @ w3 + b3
    return z, (X, z1, h1, z2, h2)


def forward_f16(p, X):
    """The arithmetic of the library's tensor-core flag pass: features, W1,
    W2 and the layer-1 activations rounded to IEEE half precision (round to
    nearest even), products accumulated without further rounding, biases and
    the output layer in full precision.  Returns the logits and, per sample,
    sum|w3*h2| + |b3|, the scale of the logit's rounding error."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    h = lambda a: np.asarray(a, dtype=np.float64).astype(np.float16).astype(np.float64)  # noqa: E731
    X = h(X)
    h1 = h(np.maximum(X @ h(W1).T + b1, 0))
    h2 = np.maximum(h1 @ h(W2).T + b2, 0)
    z = h2 @ w3 + b3
    return z, np.abs(h2) @ np.abs(w3) + abs(b3)


def loss_and_grad(p, X, y, pos_weight):
    """Summed weighted BCE and its gradient (same layout as p)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    z, (X, z1, h1, z2, h2) = forward(p, X)
    y = np.asarray(y, dtype=np.float64)
    w = np.where(y > 0.5, pos_weight, 1.0)
    sp = np.logaddexp(0.0, z)
    loss = np.sum(w * (sp - y * z))
    dz = w * (1.0 / (1.0 + np.exp(-z)) - y)
    gw3 = h2.T @ dz
    gb3 = dz.sum()
    d2 = np.outer(dz, w3) * (z2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (z1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g


def adam(p, g, m, v, step, lr, scale, b1=0.9, b2=0.999, eps=1e-8):
    g = g * scale
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
