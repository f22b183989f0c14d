"""GPU parity tests of S3TTMc through the C ABI against the reference's own
outputs (golden fixtures) and the C oracle.  Tolerances: FP64 path 1e-12
relative Frobenius error, FP32 path 1e-5 (the bars of the reference-parity
contract)."""
import os

import numpy as np
import pytest

import oracle_lib as orc
from symprop_b200 import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-12
FP32_TOL = 1e-5

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_golden_outputs_fp64_and_fp32(gpu):
    g = np.load(os.path.join(GOLD, "s3ttmc.npz"))
    ncase = len([k for k in g.files if k.endswith("_meta")])
    for ci in range(ncase):
        order, n, nnz, seed, R = (int(x) for x in g[f"c{ci}_meta"])
        X = gpu.SpSymtensor(n, order, g[f"c{ci}_inds"], g[f"c{ci}_vals"])
        U = g[f"c{ci}_U"]
        Yp = X.S3TTMc(U, R, True)
        Yu = X.S3TTMc(U, R, False)
        assert rel(Yp, g[f"c{ci}_Yp"]) < FP64_TOL, (ci, rel(Yp, g[f"c{ci}_Yp"]))
        assert rel(Yu, g[f"c{ci}_Yu"]) < FP64_TOL
        Y32 = X.S3TTMc(U.astype(np.float32), R, True, precision=gpu.FP32)
        assert rel(Y32.astype(np.float64), g[f"c{ci}_Yp"]) < FP32_TOL, (ci, rel(Y32, g[f"c{ci}_Yp"]))


@pytest.fixture(params=[1, 2, 3, 4], ids=["rows", "tiled", "warp", "chain"])
def schedule(request, gpu):
    assert gpu.lib().symprop_s3ttmc_schedule(request.param) == 0
    yield request.param
    gpu.lib().symprop_s3ttmc_schedule(0)


def run_or_skip(gpu, schedule, fn):
    """Schedules 2, 3 and 4 reject shapes they do not cover with ERR_SIZE."""
    try:
        return fn()
    except gpu.SympropError as e:
        if schedule in (2, 3, 4) and e.status == gpu.ERR_SIZE:
            pytest.skip("shape not covered by this schedule")
        raise


@pytest.mark.parametrize("order,n,nnz,R,s", [
    (3, 200, 3000, 8, 1.2), (4, 500, 20000, 16, 1.1), (5, 250, 10000, 8, 1.2),
    (6, 60, 4000, 4, 1.3), (7, 20, 500, 3, 1.2), (4, 50, 30000, 5, 1.5),
    (5, 120, 6000, 16, 1.1), (6, 200, 3000, 10, 1.1), (4, 300, 8000, 13, 1.2),
])
def test_against_oracle(gpu, schedule, order, n, nnz, R, s):
    t = synth.zipf_tuples(order, n, nnz, s, 100 + order)
    v = synth.uniform_values(nnz, 5)
    U = np.random.default_rng(order).standard_normal((n, R))
    X = gpu.SpSymtensor(n, order, t, v)
    Yo = orc.s3ttmc(order, n, t, v, U, R, True)
    Y = run_or_skip(gpu, schedule, lambda: X.S3TTMc(U, R, True))
    assert rel(Y, Yo) < FP64_TOL
    Y32 = X.S3TTMc(U.astype(np.float32), R, True, precision=gpu.FP32)
    assert rel(Y32.astype(np.float64), Yo) < FP32_TOL
    assert X.norm() == pytest.approx(orc.norm(order, t, v), rel=1e-13)


def test_hub_row_split_is_deterministic(gpu, schedule):
    # one id in every tuple: its row is cut into many slices whose partials
    # are combined in a fixed order
    rng = np.random.default_rng(7)
    n, nnz = 400, 20000
    t = np.sort(np.concatenate([np.ones((nnz, 1), np.uint32),
                                rng.integers(1, n + 1, (nnz, 3)).astype(np.uint32)], axis=1), axis=1)
    t = np.unique(t, axis=0)
    v = np.ones(t.shape[0])
    U = rng.standard_normal((n, 6))
    X = gpu.SpSymtensor(n, 4, t, v)
    Y1 = X.S3TTMc(U, 6, True)
    Y2 = X.S3TTMc(U, 6, True)
    np.testing.assert_array_equal(Y1, Y2)
    assert rel(Y1, orc.s3ttmc(4, n, t, v, U, 6, True)) < FP64_TOL


def test_edge_cases(gpu):
    U = np.random.default_rng(0).standard_normal((10, 3))
    # single nonzero with all ids equal
    X = gpu.SpSymtensor(10, 4, np.array([[2, 2, 2, 2]], np.uint32), np.array([1.5]))
    Yo = orc.s3ttmc(4, 10, np.array([[2, 2, 2, 2]], np.uint32), np.array([1.5]), U, 3, True)
    assert rel(X.S3TTMc(U, 3, True), Yo) < FP64_TOL
    # empty tensor: Y is all zeros
    X0 = gpu.SpSymtensor(10, 4, np.zeros((0, 4), np.uint32), np.zeros(0))
    assert np.all(X0.S3TTMc(U, 3, True) == 0)
    assert X0.norm() == 0.0
    # order 2: the reference leaves Y at zero (empty level loop)
    X2 = gpu.SpSymtensor(10, 2, np.array([[1, 3], [2, 2]], np.uint32), np.array([1.0, 2.0]))
    assert np.all(X2.S3TTMc(U, 3, True) == 0)
    # rank 1
    X1 = gpu.SpSymtensor(10, 3, np.array([[1, 2, 3], [3, 3, 9]], np.uint32), np.array([1.0, -2.0]))
    U1 = U[:, :1].copy()
    Yo1 = orc.s3ttmc(3, 10, np.array([[1, 2, 3], [3, 3, 9]], np.uint32), np.array([1.0, -2.0]), U1, 1, True)
    assert rel(X1.S3TTMc(U1, 1, True), Yo1) < FP64_TOL


def test_invalid_inputs_fail_loudly(gpu):
    with pytest.raises(gpu.SympropError) as e:
        gpu.SpSymtensor(5, 3, np.array([[1, 2, 6]], np.uint32), np.array([1.0]))
    assert e.value.status == gpu.ERR_INVALID
    with pytest.raises(gpu.SympropError) as e:
        gpu.SpSymtensor(5, 3, np.array([[3, 2, 1]], np.uint32), np.array([1.0]))
    assert e.value.status == gpu.ERR_INVALID
    with pytest.raises(gpu.SympropError) as e:
        gpu.SpSymtensor(5, 12, np.ones((1, 12), np.uint32), np.array([1.0]))
    assert e.value.status == gpu.ERR_ORDER


def test_device_pointer_entry_point_with_torch_stream(gpu):
    import torch
    order, n, nnz, R = 4, 300, 5000, 8
    t = synth.zipf_tuples(order, n, nnz, 1.1, 9)
    v = synth.uniform_values(nnz, 9)
    U = np.random.default_rng(1).standard_normal((n, R))
    X = gpu.SpSymtensor(n, order, t, v)
    dU = torch.from_numpy(U).cuda()
    m = gpu.symtens_size(R, order - 1)
    dY = torch.empty((n, m), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        X.s3ttmc_device(dU.data_ptr(), R, dY.data_ptr(), True, gpu.FP64, s.cuda_stream)
    s.synchronize()
    assert rel(dY.cpu().numpy(), orc.s3ttmc(order, n, t, v, U, R, True)) < FP64_TOL
    assert X.s3ttmc_launches(R, True) >= 1


@pytest.mark.parametrize("bands", [1, 2, 5, 64])
def test_host_call_row_bands_match_device_call(gpu, schedule, bands, monkeypatch):
    """The host-pointer call runs the work items in row bands and copies each
    band back while the next is computed; every band count gives the device
    call's result bit for bit, packed and full, FP64 and FP32, with split hub
    rows, empty rows and more bands than rows."""
    import torch
    monkeypatch.setenv("SPB_HOST_BANDS", str(bands))
    rng = np.random.default_rng(bands)
    cases = []
    for order, n, nnz, R in [(4, 300, 6000, 6), (5, 90, 3000, 4), (3, 40, 500, 7), (2, 12, 20, 3), (4, 3, 6, 2)]:
        t = synth.zipf_tuples(order, n, nnz, 1.2, 11 + order)
        if order == 4 and n == 300:  # hub row: every tuple holds id 1
            t = np.unique(np.sort(np.concatenate([np.ones((nnz, 1), np.uint32), t[:, 1:]], axis=1), axis=1),
                          axis=0)
        cases.append((order, n, t, synth.uniform_values(t.shape[0], 3), R))
    for order, n, t, v, R in cases:
        X = gpu.SpSymtensor(n, order, t, v)
        U = rng.standard_normal((n, R))
        for prec, dt in ((gpu.FP64, torch.float64), (gpu.FP32, torch.float32)):
            Uc = U.astype(np.float64 if prec == gpu.FP64 else np.float32)
            for packed in (True, False):
                Yh = run_or_skip(gpu, schedule, lambda: X.S3TTMc(Uc, R, packed, precision=prec))
                dU = torch.from_numpy(Uc).cuda()
                dY = torch.full(Yh.shape, float("nan"), dtype=dt, device="cuda")
                X.s3ttmc_device(dU.data_ptr(), R, dY.data_ptr(), packed, prec)
                torch.cuda.synchronize()
                np.testing.assert_array_equal(Yh, dY.cpu().numpy(), err_msg=f"{order} {n} {prec} {packed}")
                if prec == gpu.FP64 and packed:
                    assert rel(Yh, orc.s3ttmc(order, n, t, v, U, R, True)) < FP64_TOL
