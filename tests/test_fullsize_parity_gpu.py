"""S3TTMc parity at the configured sizes, on sampled rows.

The three S3TTMc workloads run whole on the GPU:
  * order 4, n = 100,000, 5M Zipf(1.1) tuples, R = 16 (Y n x 816);
  * order 6, n = 50,000, 2M planted-partition tuples, R = 10 (Y n x 2002);
  * order 5, n = 200,000, 20M power-law tuples, R = 16 (Y n x 3876).
At these sizes the hub rows are cut into hundreds of slices whose partial
rows the combine step adds, and the order-5 team kernel runs two leaves per
pipeline step, none of which the small parity cases reach.  The oracle
(orc_s3ttmc_rows in oracle/s3ttmc_oracle.c, the owners of
src/compressed_dtree.cpp:482-510 restricted to the listed rows) computes the
packed Y of 500 rows: the 50 rows with the most owners and 450 drawn at
random.  On each of the two row sets the FP64 path must match within 1e-12
and the FP32 path within 1e-5 relative Frobenius error, both through the
device-pointer call and through the host-pointer call (row bands)."""
import numpy as np
import pytest

import oracle_lib as orc
from symprop_b200 import synth

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5
WORKLOADS = [("s3ttmc_order4_zipf", 16), ("mixed_order6_planted", 10), ("learned_order5_powerlaw", 16)]


def sample_rows(t, n, seed):
    owners = np.bincount(t.ravel().astype(np.int64) - 1, minlength=n)
    hubs = np.argsort(-owners, kind="stable")[:50]
    rest = np.setdiff1d(np.arange(n), hubs)
    rnd = np.random.default_rng(seed).choice(rest, size=450, replace=False)
    return hubs.astype(np.uint32), np.sort(rnd).astype(np.uint32), owners


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name,R", WORKLOADS)
def test_fullsize_rows_match_oracle(gpu, name, R):
    import torch
    order, n, t, v = synth.workload(name)
    X = gpu.SpSymtensor(n, order, t, v)
    g = np.random.default_rng(7)
    U, _ = np.linalg.qr(g.standard_normal((n, R)))
    hubs, rnd, owners = sample_rows(t, n, 11)
    assert owners[hubs].min() > 256  # every hub row is cut into slices
    rows = np.concatenate([hubs, rnd])
    Yo = orc.s3ttmc_rows(order, n, t, v, U, R, rows)
    Yo_h, Yo_r = Yo[:50], Yo[50:]
    m = Yo.shape[1]
    sel = torch.from_numpy(rows.astype(np.int64)).cuda()
    results = {}
    for prec, dt in ((gpu.FP64, torch.float64), (gpu.FP32, torch.float32)):
        dU = torch.from_numpy(U).to(dt).cuda().contiguous()
        dY = torch.empty((n, m), dtype=dt, device="cuda")
        X.s3ttmc_device(dU.data_ptr(), R, dY.data_ptr(), True, prec)
        torch.cuda.synchronize()
        results[("device", prec)] = dY.index_select(0, sel).double().cpu().numpy()
        del dY
        Yh = X.S3TTMc(U.astype(np.float64 if prec == gpu.FP64 else np.float32), R, True, precision=prec)
        results[("host", prec)] = Yh[rows].astype(np.float64)
        del Yh
    X.close()
    for (path, prec), Yg in results.items():
        tol = FP64_TOL if prec == gpu.FP64 else FP32_TOL
        eh, er = rel(Yg[:50], Yo_h), rel(Yg[50:], Yo_r)
        label = f"{name} {path} {'fp64' if prec == gpu.FP64 else 'fp32'}"
        assert eh <= tol, f"{label}: hub rows rel. Frobenius {eh:.3e} (owners {owners[hubs].sum()})"
        assert er <= tol, f"{label}: random rows rel. Frobenius {er:.3e}"
    # the host-pointer call only reorders the work: bit for bit the device call
    for prec in (gpu.FP64, gpu.FP32):
        assert np.array_equal(results[("host", prec)], results[("device", prec)])
