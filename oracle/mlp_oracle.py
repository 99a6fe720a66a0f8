"""TEST INFRASTRUCTURE ONLY: FP64 reference of the proposal MLP.

Forward pass, weighted binary cross-entropy loss and its gradient for the
16 -> 64 -> 64 -> 1 network (parameter layout W1[16][64], b1[64], W2[64][64],
b2[64], W3[64], b3), in float64 numpy.  With bf16=True every operand the GPU
kernels feed to the tensor cores (features, weights, hidden activations, the
back-propagated hidden gradients and the output gradient dz, which the
kernels multiply with the hidden activations to get dW3 and sum into the bias
gradients on the tensor cores) is first rounded to BF16
(round-to-nearest-even), so the only remaining difference from the kernels
is FP32 versus FP64 accumulation.
"""
from __future__ import annotations

import numpy as np

IN, HID = 16, 64


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + IN * HID].reshape(IN, HID); o += IN * HID
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + HID]; o += HID
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def bf16(x):
    """Round to BF16 (nearest even) and back, in float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(params, X, bf=False):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    Xb = r(X)
    pre1 = Xb @ r(W1) + b1
    h1 = r(np.maximum(pre1, 0))
    pre2 = h1 @ r(W2) + b2
    h2 = r(np.maximum(pre2, 0))
    z = h2 @ r(W3) + b3
    q = 1.0 / (1.0 + np.exp(-z))
    return q, (Xb, pre1, h1, pre2, h2, z)


def loss_and_grad(params, X, t, w=None, bf=False):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    n = X.shape[0]
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    ws = w / w.sum()
    q, (Xb, pre1, h1, pre2, h2, z) = forward(params, X, bf)
    t = np.asarray(t, dtype=np.float64)
    qc = np.clip(q, 1e-7, 1 - 1e-7)
    loss = float(-(ws * (t * np.log(qc) + (1 - t) * np.log(1 - qc))).sum())
    dz = ws * (q - t)
    gW3 = h2.T @ r(dz)
    gb3 = dz.sum()
    dh2 = r((pre2 > 0) * np.outer(dz, W3))
    gb2 = dh2.sum(axis=0)
    gW2 = h1.T @ dh2
    dh1 = r((pre1 > 0) * (dh2 @ r(W2).T))
    gb1 = dh1.sum(axis=0)
    gW1 = Xb.T @ dh1
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
