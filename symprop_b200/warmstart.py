"""Learned warm start: training and use of the per-node MLP that proposes
HOOI's initial factor (north of the reference, which starts from random or
hoevd/hosvd factors, src/tucker.cpp:25-36, src/sparse/spsymtensor.cpp:339-383).

Every numeric step runs in this package's CUDA kernels through the C ABI
(include/symprop.h: symprop_ws_features, symprop_mlp_forward,
symprop_mlp_backward, symprop_projector_loss, symprop_adam_step,
symprop_ws_predict); torch only allocates device buffers.  Labels are the
converged factors of this package's own FP64 GPU HOOI on seeded synthetic
tensors; plain random-start HOOI stays the fallback and the reference point.
"""
from __future__ import annotations

import ctypes
import os
import time
from dataclasses import dataclass

import numpy as np

from . import SpSymtensor, _check, lib, synth

_P = ctypes.c_void_p
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_r8.npz")


def _bind():
    L = lib()
    U32, U64, F32, I = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float, ctypes.c_int
    sig = {
        "symprop_ws_features": (I, [_P, U32, U64, _P, _P]),
        "symprop_mlp_forward": (I, [_P, U32, U32, U32, U32, _P, _P, _P, _P]),
        "symprop_mlp_backward": (I, [_P, U32, U32, U32, U32, _P, _P, _P, _P, _P]),
        "symprop_projector_loss": (I, [_P, _P, U32, U32, _P, ctypes.POINTER(ctypes.c_double), _P]),
        "symprop_adam_step": (I, [_P, _P, _P, _P, U32, F32, F32, F32, F32, U32, _P, _P]),
        "symprop_ws_predict": (I, [_P, U32, U64, U32, _P, _P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def nparams(R: int, H: int) -> int:
    F = R + 2
    return H * F + H + R * H + R


class WarmStartModel:
    """FP32 master weights [W1 (H x F), b1, W2 (R x H), b2], F = R + 2."""

    def __init__(self, R: int = 8, H: int = 64, seed: int = 0, w: np.ndarray | None = None):
        self.R, self.H, self.F = R, H, R + 2
        if w is None:
            rng = np.random.default_rng(seed)
            F = self.F
            W1 = rng.standard_normal((H, F)) * np.sqrt(2.0 / F)
            W2 = rng.standard_normal((R, H)) * np.sqrt(1.0 / H)
            w = np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(R)])
        self.w = np.asarray(w, dtype=np.float32).copy()
        assert self.w.size == nparams(R, H)

    def save(self, path: str) -> None:
        np.savez(path, w=self.w, R=self.R, H=self.H)

    @staticmethod
    def load(path: str = DEFAULT_WEIGHTS) -> "WarmStartModel":
        d = np.load(path)
        return WarmStartModel(int(d["R"]), int(d["H"]), w=d["w"])

    def predict(self, X: SpSymtensor, seed: int = 0) -> np.ndarray:
        L = _bind()
        U = np.zeros((X.dim(), self.R))
        _check(L.symprop_ws_predict(X.handle, self.R, seed, self.H, _P(self.w.ctypes.data),
                                    _P(U.ctypes.data)))
        return U


@dataclass
class Sample:
    X: object       # torch.cuda FloatTensor n x F (features)
    Ut: object      # torch.cuda DoubleTensor n x R (converged factor)
    n: int
    hooi_iters: int


def features(X: SpSymtensor, R: int, seed: int = 0):
    import torch
    L = _bind()
    out = torch.empty((X.dim(), R + 2), dtype=torch.float32, device="cuda")
    _check(L.symprop_ws_features(X.handle, R, seed, _P(out.data_ptr()), None))
    torch.cuda.synchronize()
    return out


def random_tensor(seed: int, small: bool = True, family: str = "community"):
    """A seeded training tensor.

    family "community": order in {3,4,5,6}, planted communities with
    Zipf(1.2) degrees (small=True shrinks n and nnz for quick training).
    family "powerlaw": order 5, power-law degree weights (exponent 2.1) with
    16 planted communities, 80% of the tuples inside one community, n in
    [2000, 8000], 20k-200k tuples; a small version of the order-5 rank-16
    learned-start workload."""
    rng = np.random.default_rng(10_000 + seed)
    if family == "powerlaw":
        n = int(rng.integers(2000, 8_001))
        nnz = int(rng.integers(20_000, 200_001))
        t = synth.powerlaw_communities(5, n, nnz, 2.1, 16, 0.8, 20_000 + seed)
        return 5, n, t, np.ones(t.shape[0])
    order = int(rng.integers(3, 7))
    if small:
        n = int(rng.integers(1000, 4000))
        nnz = int(rng.integers(10_000, 40_000))
    else:
        n = int(rng.integers(1000, 20_001))
        nnz = int(rng.integers(10_000, 500_001))
    k = int(rng.integers(4, 17))
    t = synth.community_zipf(order, n, nnz, k, 1.2, seed)
    return order, n, t, np.ones(t.shape[0])


def make_samples(seeds, R: int = 8, delta: float = 1.0, small: bool = True, log=print,
                 family: str = "community"):
    import torch
    out = []
    for s in seeds:
        order, n, t, v = random_tensor(s, small, family)
        X = SpSymtensor(n, order, t, v)
        d = X.TuckerHOOI(rank=R, max_iter=200, rel_tol=1e-10, delta=delta, seed=s)
        Ut = torch.from_numpy(np.ascontiguousarray(d.factor)).cuda()
        out.append(Sample(features(X, R, seed=s), Ut, n, d.iterations))
        if log:
            log(f"sample {s}: order {order} n {n} nnz {t.shape[0]} HOOI iters {d.iterations} err {d.error:.6f}")
        X.close()
    return out


def train(model: WarmStartModel, samples, epochs: int = 20, lr: float = 1e-3, seed: int = 0, log=print):
    """Adam on the projector loss, one sample per step, all on the GPU."""
    import torch
    L = _bind()
    R, H, F = model.R, model.H, model.F
    P = nparams(R, H)
    w = torch.from_numpy(model.w.copy()).cuda()
    m = torch.zeros(P, dtype=torch.float32, device="cuda")
    v = torch.zeros_like(m)
    g = torch.zeros_like(m)
    wb = w.to(torch.bfloat16)
    rng = np.random.default_rng(seed)
    step = 0
    hist = []
    for ep in range(epochs):
        tot = 0.0
        for i in rng.permutation(len(samples)):
            s = samples[i]
            Z1 = torch.empty((s.n, H), dtype=torch.float32, device="cuda")
            Out = torch.empty((s.n, R), dtype=torch.float32, device="cuda")
            gOut = torch.empty_like(Out)
            _check(L.symprop_mlp_forward(_P(s.X.data_ptr()), s.n, F, H, R, _P(wb.data_ptr()),
                                         _P(Z1.data_ptr()), _P(Out.data_ptr()), None))
            loss = ctypes.c_double(0)
            _check(L.symprop_projector_loss(_P(Out.data_ptr()), _P(s.Ut.data_ptr()), s.n, R,
                                            _P(gOut.data_ptr()), ctypes.byref(loss), None))
            _check(L.symprop_mlp_backward(_P(s.X.data_ptr()), s.n, F, H, R, _P(wb.data_ptr()),
                                          _P(Z1.data_ptr()), _P(gOut.data_ptr()), _P(g.data_ptr()), None))
            step += 1
            _check(L.symprop_adam_step(_P(w.data_ptr()), _P(m.data_ptr()), _P(v.data_ptr()),
                                       _P(g.data_ptr()), P, lr, 0.9, 0.999, 1e-8, step,
                                       _P(wb.data_ptr()), None))
            tot += loss.value
        torch.cuda.synchronize()
        hist.append(tot / max(len(samples), 1))
        if log:
            log(f"epoch {ep}: mean projector loss {hist[-1]:.5f}")
    model.w = w.cpu().numpy()
    return hist


def compare(model: WarmStartModel, seeds, R: int = 8, delta: float = 1.0, tol: float = 1e-6,
            small: bool = True, precision: int = 0, family: str = "community"):
    """Random-start vs learned-start HOOI on held-out tensors: iterations,
    final errors and device time."""
    rows = []
    for s in seeds:
        order, n, t, v = random_tensor(s, small, family)
        X = SpSymtensor(n, order, t, v)
        base = X.TuckerHOOI(rank=R, max_iter=200, rel_tol=tol, delta=delta, seed=s, precision=precision)
        t0 = time.perf_counter()
        U0 = model.predict(X, seed=s)
        pred_ms = (time.perf_counter() - t0) * 1e3
        lrn = X.TuckerHOOI(rank=R, max_iter=200, rel_tol=tol, delta=delta, seed=s, init="user",
                           init_factor=U0, precision=precision)
        rows.append({"seed": s, "order": order, "n": n, "nnz": int(t.shape[0]),
                     "random_iters": base.iterations, "learned_iters": lrn.iterations,
                     "random_error": base.error, "learned_error": lrn.error,
                     "random_ms": base.time_ms, "learned_ms": lrn.time_ms + pred_ms})
        X.close()
    return rows
