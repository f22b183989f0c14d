"""Mixed-precision HOOI and HOQRI against the FP64 GPU path (the drop-in).

Mixed precision: FP32 S3TTMc with compensated accumulation, the dense
products (Gram, Y V, Y D C^T) on the tcgen05 tensor cores with split-BF16
operands and FP32 accumulation, FP64 eigen solve, QR and objective.  The
tensors here have n > m, so the m x m tensor-core Gram is the one HOOI
uses (n <= m takes the n x n form, covered by the reference-config test in
test_tucker_gpu.py).

Bars (north star: the final objective within 1e-6 of the FP64 path's):
  * objective: |e_mixed - e_fp64| <= 1e-6 e_fp64 at tolerance 1e-6;
  * ||C||^2: the relative error that objective bar allows,
    |d||C||^2| / ||C||^2 = 2 e |de| / (1 - e^2) <= 2e-6 e^2 / (1 - e^2);
  * factor: run to tolerance 1e-10, the mixed driver hands over to FP64
    iterations once its own resolution is reached, so both paths must end at
    the same fixed point: largest principal angle <= 1e-6 rad.
"""
import numpy as np
import pytest

from symprop_b200 import synth

pytestmark = pytest.mark.gpu


def planted_order4(sp):
    t = synth.community_zipf(4, 3000, 60_000, 8, 1.2, 3)
    return sp.SpSymtensor(3000, 4, t, np.ones(t.shape[0])), 8  # m = C(10,3) = 120 < n


def powerlaw_order5(sp):
    order, n, t, v = synth.workload("learned_order5_powerlaw", scale=0.1)  # n = 20k, 2M tuples
    return sp.SpSymtensor(n, order, t, v), 16  # m = C(19,4) = 3876 < n


def angle(U1, U2):
    s = np.linalg.svd(U1.T @ U2, compute_uv=False)
    return float(np.arccos(np.clip(s.min(), -1.0, 1.0)))


@pytest.mark.parametrize("make", [planted_order4, powerlaw_order5], ids=["order4_n3000_r8", "order5_n20k_r16"])
@pytest.mark.parametrize("alg", ["HOOI", "HOQRI"])
def test_mixed_reaches_fp64_objective(gpu, make, alg):
    X, R = make(gpu)
    assert X.dim() > gpu.symtens_size(R, X.order() - 1)
    fn = X.TuckerHOOI if alg == "HOOI" else X.TuckerHOQRI
    kw = dict(rank=R, max_iter=100, rel_tol=1e-6, delta=1.0, seed=0)
    d64 = fn(**kw)
    dmx = fn(precision=gpu.PREC_MIXED, **kw)
    e = d64.error
    gap = abs(dmx.error - e) / e
    cn = abs(dmx.core_norm ** 2 - d64.core_norm ** 2) / d64.core_norm ** 2
    msg = (f"{alg}: fp64 {e:.12f} ({d64.iterations} it), mixed {dmx.error:.12f} ({dmx.iterations} it), "
           f"gap {gap:.2e}, ||C||^2 {cn:.2e}, angle {angle(d64.factor, dmx.factor):.2e}")
    print(msg)
    assert gap <= 1e-6, msg
    assert cn <= 2e-6 * e * e / (1 - e * e), msg


@pytest.mark.parametrize("alg", ["HOOI", "HOQRI"])
def test_mixed_ends_at_fp64_fixed_point(gpu, alg):
    X, R = planted_order4(gpu)
    fn = X.TuckerHOOI if alg == "HOOI" else X.TuckerHOQRI
    kw = dict(rank=R, max_iter=400, rel_tol=1e-10, delta=1.0, seed=0)
    d64 = fn(**kw)
    dmx = fn(precision=gpu.PREC_MIXED, **kw)
    th = angle(d64.factor, dmx.factor)
    msg = (f"{alg}: fp64 {d64.error:.14f} ({d64.iterations} it), mixed {dmx.error:.14f} "
           f"({dmx.iterations} it), angle {th:.2e}")
    print(msg)
    assert th <= 1e-6, msg
    assert abs(dmx.error - d64.error) <= 1e-9 * d64.error, msg
