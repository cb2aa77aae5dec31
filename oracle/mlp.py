"""TEST INFRASTRUCTURE ONLY: a numpy restatement of the learned ranking's network, its
features and its training step, the checker of the library's jk_mlp_* kernels.

The network has no counterpart in the reference.  Layout of the FP32 parameter vector:
W1 [64][7] row-major, b1 [64], W2 [64][64], b2 [64], W3 [64], b3.  Weights enter the
arithmetic rounded to BF16 (round to nearest even), biases as they are; everything here
is computed in float64.
"""
from __future__ import annotations

import numpy as np

NF = 7
H = 64


def bf16(x):
    """Round float32 values to the nearest BF16 value (ties to even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, np.float32)
    o = 0
    W1 = P[o:o + H * NF].reshape(H, NF); o += H * NF
    b1 = P[o:o + H]; o += H
    W2 = P[o:o + H * H].reshape(H, H); o += H * H
    b2 = P[o:o + H]; o += H
    W3 = P[o:o + H]; o += H
    b3 = P[o]
    return W1, b1, W2, b2, W3, b3


def features(A, J, step):
    """Features of every hyperbolic pair, (+ index, - index) order (see jk_mlp_features)."""
    A = np.asarray(A, np.float64)
    n = A.shape[0]
    J = np.asarray(J)
    plus = np.nonzero(J == 1)[0]
    minus = np.nonzero(J == -1)[0]
    X = np.zeros((len(plus) * len(minus), NF), np.float32)

    def lg(x):
        a = abs(x)
        return np.float32((np.log2(a) if a > 0 else -1074.0) / 64.0)

    k = 0
    for a in plus:
        for b in minus:
            p, q = (a, b) if a < b else (b, a)
            X[k] = [lg(A[p, q]), lg(A[q, p]), lg(A[p, p]), lg(A[q, q]), float(J[p]), float(J[q]),
                    min(np.float32(step) / np.float32(10.0 * n), np.float32(4.0))]
            k += 1
    return X


def forward(X, P):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    X = np.asarray(X, np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    return h2 @ W3 + float(b3), (X, z1, h1, z2, h2)


def loss_grad(X, T, P):
    """Mean squared error and its gradient with respect to the parameter vector
    (straight through the BF16 rounding of the weights)."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    y, (X, z1, h1, z2, h2) = forward(X, P)
    T = np.asarray(T, np.float64)
    m = len(T)
    r = y - T
    loss = float(np.mean(r * r))
    dy = 2.0 * r / m
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dh2 = np.outer(dy, bf16(W3)) * (z2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ bf16(W2)) * (z1 > 0)
    gW1 = dh1.T @ X
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g


def adam(P, G, M, V, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (float64), returns (P, M, V)."""
    P, G, M, V = (np.asarray(x, np.float64) for x in (P, G, M, V))
    M = b1 * M + (1 - b1) * G
    V = b2 * V + (1 - b2) * G * G
    P = P - lr * (M / (1 - b1 ** t)) / (np.sqrt(V / (1 - b2 ** t)) + eps)
    return P, M, V
