"""GPU: the hoevd initialisation (A = X_(1) X_(1)^T, src/sparse/spsymtensor.cpp:363-439).
The matrix-free operator (csrc/hoevd.cu, used above n = 8192) against the
dense A on small tensors, and both against the reference CLI's own
`-init hoevd` run (oracle/_ref/symtucker) when that build is present: the
HOOI error trajectory is basis-independent and is compared per iteration."""
import os
import re
import subprocess

import numpy as np
import pytest

from symprop_b200 import synth

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "symtucker")
CASES = [(3, 60, 500, 4, 1.3, 11), (4, 120, 2500, 6, 1.2, 12), (5, 90, 1500, 5, 1.2, 13)]


def hoevd_run(gpu, X, rank, iters, matrix_free):
    old = os.environ.get("SPB_HOEVD_MATRIX_FREE")
    os.environ["SPB_HOEVD_MATRIX_FREE"] = "1" if matrix_free else "0"
    try:
        return X.TuckerHOOI(rank=rank, max_iter=iters, delta=0.5, seed=0, init="hoevd", rel_tol=0.0)
    finally:
        if old is None:
            os.environ.pop("SPB_HOEVD_MATRIX_FREE", None)
        else:
            os.environ["SPB_HOEVD_MATRIX_FREE"] = old


@pytest.mark.parametrize("order,n,nnz,rank,s,seed", CASES)
def test_matrix_free_equals_dense(gpu, order, n, nnz, rank, s, seed):
    t = synth.zipf_tuples(order, n, nnz, s, seed)
    X = gpu.SpSymtensor(n, order, t, np.ones(t.shape[0]))
    d0 = hoevd_run(gpu, X, rank, 8, False)
    d1 = hoevd_run(gpu, X, rank, 8, True)
    np.testing.assert_allclose(d1.error_trace, d0.error_trace, rtol=0, atol=1e-10)


@pytest.mark.skipif(not os.path.exists(REF_CLI), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("order,n,nnz,rank,s,seed", CASES)
def test_hoevd_matches_reference_cli(gpu, tmp_path, order, n, nnz, rank, s, seed):
    t = synth.zipf_tuples(order, n, nnz, s, seed)
    tns = tmp_path / "x.tns"
    synth.write_tns(str(tns), order, n, t, np.ones(t.shape[0]))
    out = subprocess.run([REF_CLI, "-f", str(tns), "-r", str(rank), "-i", "8", "-t", "0", "-d", "0.5", "-s", "0",
                          "-a", "0", "-init", "hoevd"], capture_output=True, text=True, timeout=300).stdout
    ref = np.array([float(x) for x in re.findall(r"error (\S+)", out)])
    assert ref.size == 8
    X = gpu.SpSymtensor(n, order, t, np.ones(t.shape[0]))
    for mf in (False, True):
        d = hoevd_run(gpu, X, rank, 8, mf)
        np.testing.assert_allclose(d.error_trace, ref, rtol=0, atol=1e-8)
