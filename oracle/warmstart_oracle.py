"""ORACLE — test infrastructure only.  NumPy restatement of the learned
warm-start network (per-node 2-layer MLP), its rotation-invariant projector
loss and Adam, used by tests/ to check the CUDA forward, backward and Adam
kernels.  The product never imports this file.

There is no counterpart in the reference (it starts HOOI from random or
hoevd/hosvd factors, src/tucker.cpp:25-36, src/sparse/spsymtensor.cpp:339-383),
so the analytic gradients here are pinned by central finite differences
(tests/test_warmstart.py).

Parameter layout (one flat vector): W1 (H x F), b1 (H), W2 (O x H), b2 (O).
"""
import numpy as np


def split(w, F, H, O):
    o = 0
    W1 = w[o:o + H * F].reshape(H, F); o += H * F
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + O * H].reshape(O, H); o += O * H
    b2 = w[o:o + O]
    return W1, b1, W2, b2


def bf16_round(w):
    """round-to-nearest-even to bfloat16, returned as float64"""
    a = np.asarray(w, dtype=np.float32).copy()
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(X, w, F, H, O):
    W1, b1, W2, b2 = split(w, F, H, O)
    Z1 = X @ W1.T + b1
    Hh = np.maximum(Z1, 0.0)
    return Z1, Hh @ W2.T + b2


def projector_loss(Out, Ut):
    """L = r - tr(P_Ut P_Out), P_Out = Out (Out^T Out)^-1 Out^T; returns (L, dL/dOut)"""
    r = Out.shape[1]
    A = Ut.T @ Out
    G = Out.T @ Out
    Gi = np.linalg.inv(G)
    f = np.trace(Gi @ A.T @ A)
    M1 = A @ Gi
    M2 = Gi @ A.T @ A @ Gi
    grad = -2.0 * (Ut @ M1 - Out @ M2)
    return r - f, grad


def backward(X, w, Z1, gOut, F, H, O):
    W1, b1, W2, b2 = split(w, F, H, O)
    Hh = np.maximum(Z1, 0.0)
    gW2 = gOut.T @ Hh
    gb2 = gOut.sum(axis=0)
    dH = gOut @ W2
    dZ = dH * (Z1 > 0)
    gW1 = dZ.T @ X
    gb1 = dZ.sum(axis=0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2])


def loss_of_weights(X, w, Ut, F, H, O):
    _, Out = forward(X, w, F, H, O)
    return projector_loss(Out, Ut)[0]


def adam(w, m, v, g, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return w - lr * mh / (np.sqrt(vh) + eps), m, v
