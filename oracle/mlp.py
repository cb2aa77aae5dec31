"""TEST INFRASTRUCTURE ONLY: a numpy restatement of the learned ranking's network, its
features and its training step, the checker of the library's jk_mlp_* kernels.

The network has no counterpart in the reference.  Layout of the FP32 parameter vector:
W1 [64][8] row-major, b1 [64], W2 [64][64], b2 [64], W3 [64], b3.  Inputs, weights and the
first layer's activations enter the arithmetic rounded to BF16 (round to nearest even),
biases as they are; everything else here is computed in float64.  The features are the
Gram quantities of a scanned hyperbolic pair (see features()).
"""
from __future__ import annotations

import numpy as np

NF = 8
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


def _lg64(x):
    a = abs(float(x))
    return np.float32((np.log2(a) if a > 0 else -1074.0) / 64.0)


def features(A, J, step):
    """Features and w_gram of every hyperbolic pair, (+ index, - index) order (see
    jk_mlp_features): for a pair (p, q) that needs the column scan, with x = A(:,p), y = A(:,q)
    without rows p, q and Z2 the pair's 2x2 right transformation,
      w_gram = d0 + nx (1 - Z11^2 - Z12^2) + ny (1 - Z21^2 - Z22^2) - 2 (Z11 Z21 + Z12 Z22) g,
    nx = x.x, ny = y.y, g = x.y, d0 the two leading terms of ABODNDF2; the features are the
    BF16 roundings of log2/64 of |w_gram|, nx, ny, |g|, |d0|, |Z12| + |Z21|, sign(w_gram) and
    min(S / (10 N), 4).  Other pairs: zero features and w_gram NaN.  Returns (X, w_gram).
    A complex A (jk_zmlp_features, ZMAGF2H / ABODNZF2): nx = x^H x, ny = y^H y, g = x^H y,
    d0 over the real and imaginary parts of the two leading terms and
      w_gram = d0 + nx (1 - |Z11|^2 - |Z12|^2) + ny (1 - |Z21|^2 - |Z22|^2)
               - 2 Re((conj(Z11) Z21 + conj(Z12) Z22) g)."""
    import oracle
    cplx = np.iscomplexobj(A)
    A = np.asarray(A, np.complex128 if cplx else np.float64)
    n = A.shape[0]
    J = np.asarray(J)
    plus = np.nonzero(J == 1)[0]
    minus = np.nonzero(J == -1)[0]
    X = np.zeros((len(plus) * len(minus), NF), np.float64)
    Wg = np.full(len(plus) * len(minus), np.nan)
    A0 = A.copy()
    np.fill_diagonal(A0, 0.0)
    k = -1
    for a in plus:
        for b in minus:
            k += 1
            p, q = (a, b) if a < b else (b, a)
            jp = 1 if a < b else -1
            app, aqp, apq, aqq = A[p, p], A[q, p], A[p, q], A[q, q]
            if cplx:
                may = aqp != 0 or apq != 0 or app.imag != 0 or aqq.imag != 0 or np.signbit(app.real) or \
                    np.signbit(aqq.real)
            else:
                may = aqp != 0 or apq != 0 or np.signbit(app) or np.signbit(aqq)
            if not may:
                continue
            A2, U2, Z2, info = oracle.hsvd2(np.array([[app, apq], [aqp, aqq]]), [jp, -jp])
            if info < 0 or not (info & 1) or not (info & 4):
                continue
            a1 = A2[1, 0] if info & 8 else 0.0
            a2 = A2[0, 1] if info & 8 else 0.0
            z11, z21, z12, z22 = Z2[0, 0], Z2[1, 0], Z2[0, 1], Z2[1, 1]
            x, y = A0[:, p].copy(), A0[:, q].copy()
            x[q] = 0.0
            y[p] = 0.0
            if cplx:
                d = 0.0
                for u, v in ((aqp.real, a1.real), (aqp.imag, a1.imag), (apq.real, a2.real), (apq.imag, a2.imag)):
                    d += (u - v) * (u + v)
                nx, ny = float(np.vdot(x, x).real), float(np.vdot(y, y).real)
                g = complex(np.vdot(x, y))
                c1 = (1.0 - z11.real) * (1.0 + z11.real) - z11.imag ** 2 - abs(z12) ** 2
                c2 = (1.0 - z22.real) * (1.0 + z22.real) - z22.imag ** 2 - abs(z21) ** 2
                c3 = np.conj(z11) * z21 + np.conj(z12) * z22
                w = d + (nx * c1 + ny * c2 - 2.0 * (c3 * g).real)
            else:
                d = (aqp - a1) * (aqp + a1) + (apq - a2) * (apq + a2)
                nx, ny, g = float(x @ x), float(y @ y), float(x @ y)
                c1 = (1.0 - z11) * (1.0 + z11) - z12 * z12
                c2 = (1.0 - z22) * (1.0 + z22) - z21 * z21
                c3 = z11 * z21 + z12 * z22
                w = d + (nx * c1 + ny * c2 - 2.0 * c3 * g)
            Wg[k] = w
            X[k] = bf16([_lg64(w), -1.0 if w < 0 else 1.0, _lg64(nx), _lg64(ny), _lg64(abs(g)), _lg64(d),
                         _lg64(abs(z12) + abs(z21)), min(np.float32(step) / np.float32(10.0 * n), np.float32(4.0))])
    return X.astype(np.float32), Wg


def forward(X, P):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    X = bf16(np.asarray(X, np.float32))
    z1 = X @ W1.T + b1
    h1 = bf16(np.maximum(z1, 0.0).astype(np.float32))
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    return h2 @ W3 + float(b3), (X, z1, h1, z2, h2)


def loss_grad(X, T, P):
    """Mean squared error and its gradient with respect to the parameter vector
    (straight through the BF16 rounding of the weights and of the first layer's outputs)."""
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
