"""CPU tests: the warm-start oracle's analytic gradients agree with central
finite differences (this pins the oracle used by the GPU gradient checks)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import warmstart_oracle as wo  # noqa: E402


def test_projector_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n, r = 40, 3
    Ut, _ = np.linalg.qr(rng.standard_normal((n, r)))
    Out = rng.standard_normal((n, r))
    L, g = wo.projector_loss(Out, Ut)
    assert 0 <= L <= r
    eps = 1e-6
    for (i, j) in [(0, 0), (5, 2), (17, 1), (39, 0)]:
        P = Out.copy(); P[i, j] += eps
        M = Out.copy(); M[i, j] -= eps
        fd = (wo.projector_loss(P, Ut)[0] - wo.projector_loss(M, Ut)[0]) / (2 * eps)
        assert abs(fd - g[i, j]) < 1e-6 * max(1.0, abs(fd))
    # rotation invariance: Out -> Out Q leaves the loss unchanged
    Q, _ = np.linalg.qr(rng.standard_normal((r, r)))
    assert abs(wo.projector_loss(Out @ Q, Ut)[0] - L) < 1e-12


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n, R, H = 30, 3, 8
    F = R + 2
    X = rng.standard_normal((n, F))
    Ut, _ = np.linalg.qr(rng.standard_normal((n, R)))
    P = H * F + H + R * H + R
    w = rng.standard_normal(P) * 0.3
    Z1, Out = wo.forward(X, w, F, H, R)
    _, gOut = wo.projector_loss(Out, Ut)
    g = wo.backward(X, w, Z1, gOut, F, H, R)
    eps = 1e-6
    for p in [0, 7, H * F + 2, H * F + H + 5, P - 1]:
        wp = w.copy(); wp[p] += eps
        wm = w.copy(); wm[p] -= eps
        fd = (wo.loss_of_weights(X, wp, Ut, F, H, R) - wo.loss_of_weights(X, wm, Ut, F, H, R)) / (2 * eps)
        assert abs(fd - g[p]) < 1e-5 * max(1.0, abs(fd)), (p, fd, g[p])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0])
    r = wo.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # ties to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
