"""Host-injected failures on the GPU path: each one must come back as a
status code (or as NaN where the arithmetic defines it), never as a fault,
a hang or a silently wrong number.  No test here faults or traps the GPU:
the out-of-memory case asks for an allocation the device refuses before
any kernel runs."""
import ctypes

import numpy as np
import pytest

import oracle_lib as orc
from symprop_b200 import synth

pytestmark = pytest.mark.gpu


def test_device_out_of_memory_is_a_status(gpu):
    # C = A^T B with a 2^60-element C: the device allocation is refused
    # before A or B is read (both are one-element host buffers)
    a = np.ones(1)
    c = np.zeros(1)
    big = (1 << 30) - 1
    st = gpu.lib().symprop_gemmtn(c.ctypes.data, a.ctypes.data, a.ctypes.data, 1, big, big)
    assert st == gpu.ERR_OOM, gpu.lib().symprop_last_error()
    # the context is still usable
    C = gpu.matrix.gemmtn(np.arange(6.0), np.arange(12.0), 3, 2, 4)
    assert C.shape == (2, 4)


def test_tensor_core_wait_expiry_is_a_status(gpu):
    """The tcgen05 kernels bound every mbarrier wait.  The failure-injection
    hook lowers the bound of the main-loop waits (TMA copies landing, MMAs
    freeing a stage) to 1 ns, so waits that last longer than one tick of the
    GPU's global timer expire.  The kernel must then drain the copies and
    MMAs it issued, free its tensor memory and report SYMPROP_ERR_TIMEOUT,
    and the next call, with the default bound, must give the right matrix."""
    import torch
    L = gpu.lib()
    n, m = 50000, 330
    g = torch.Generator(device="cpu").manual_seed(5)
    Y = torch.randn(n, m, generator=g).cuda()
    sd = (torch.rand(m, generator=g) + 0.5).cuda()
    G = torch.empty(m, m, dtype=torch.float64, device="cuda")
    P = ctypes.c_void_p
    try:
        assert L.symprop_debug_set_tc_wait_ns(1) == 0
        st = L.symprop_gram_device(P(Y.data_ptr()), n, m, P(sd.data_ptr()), P(G.data_ptr()), gpu.FP32, None)
        assert st == gpu.ERR_TIMEOUT, (st, L.symprop_last_error())
        assert b"bounded wait" in L.symprop_last_error()
    finally:
        L.symprop_debug_set_tc_wait_ns(0)
    st = L.symprop_gram_device(P(Y.data_ptr()), n, m, P(sd.data_ptr()), P(G.data_ptr()), gpu.FP32, None)
    assert st == 0, L.symprop_last_error()
    X = (Y * sd).double()
    ref = X.T @ X
    # FP32 accumulation on the tensor cores: one ulp per accumulator update
    # (3 n / 16 updates) plus the split's 2^-17 per product
    assert float((G - ref).norm() / ref.norm()) < 3 * n / 16 * 2.0 ** -24 + 1e-5


def test_rank_above_dim_is_rejected(gpu):
    t = synth.zipf_tuples(3, 6, 10, 1.2, 1)
    X = gpu.SpSymtensor(6, 3, t, np.ones(t.shape[0]))
    with pytest.raises(gpu.SympropError) as e:
        X.TuckerHOOI(rank=7, max_iter=2)
    assert e.value.status == gpu.ERR_INVALID
    with pytest.raises(gpu.SympropError) as e:
        X.TuckerHOQRI(rank=0, max_iter=2)
    assert e.value.status == gpu.ERR_INVALID


def test_nan_factor_rows_poison_only_their_owners(gpu):
    """A NaN in row k of U reaches exactly the Y rows that have an owner whose
    leaf holds k; every other row matches the oracle."""
    order, n, nnz, R = 4, 200, 3000, 6
    t = synth.zipf_tuples(order, n, nnz, 1.2, 5)
    v = synth.uniform_values(nnz, 5)
    U = np.random.default_rng(5).standard_normal((n, R))
    cnt = np.bincount(t.ravel().astype(np.int64), minlength=n + 1)[1:]
    k = int(np.argmin(np.where(cnt > 0, cnt, cnt.max() + 1)))  # a rarely used id
    U[k, 2] = np.nan
    X = gpu.SpSymtensor(n, order, t, v)
    Y = X.S3TTMc(U, R, True)
    Yo = orc.s3ttmc(order, n, t, v, U, R, True)
    bad = np.isnan(Yo).any(axis=1)
    assert bad.any() and not bad.all()
    np.testing.assert_array_equal(np.isnan(Y).any(axis=1), bad)
    ok = ~bad
    assert np.linalg.norm(Y[ok] - Yo[ok]) <= 1e-12 * np.linalg.norm(Yo[ok])
    Y32 = X.S3TTMc(U.astype(np.float32), R, True, precision=gpu.FP32)
    np.testing.assert_array_equal(np.isnan(Y32).any(axis=1), bad)


def test_nan_tensor_value_ends_the_solve(gpu):
    """A NaN nonzero makes ||X|| NaN; the solve stops within its iteration
    and restart limits with a NaN error or a non-convergence status."""
    t = synth.zipf_tuples(3, 50, 400, 1.2, 9)
    v = np.ones(t.shape[0])
    v[3] = np.nan
    X = gpu.SpSymtensor(50, 3, t, v)
    assert np.isnan(X.norm())
    try:
        d = X.TuckerHOOI(rank=4, max_iter=3, verbose=False)
        assert np.isnan(d.error)
    except gpu.SympropError as e:
        assert e.status in (gpu.ERR_NOCONV, gpu.ERR_INVALID)


def test_bad_tns_is_a_status(gpu, tmp_path):
    p = tmp_path / "bad.tns"
    p.write_text("3 10\n1 2 3 1.0\n4 5 x 2.0\n")
    with pytest.raises(gpu.SympropError) as e:
        gpu.SpSymtensor.load_tns(str(p))
    assert e.value.status == gpu.ERR_INVALID
    p.write_text("3 10\n1 2 11 1.0\n1 2 3 2.0\n")  # id above dim
    with pytest.raises(gpu.SympropError) as e:
        gpu.SpSymtensor.load_tns(str(p))
    assert e.value.status == gpu.ERR_INVALID
    with pytest.raises(gpu.SympropError):
        gpu.SpSymtensor.load_tns(str(tmp_path / "missing.tns"))
