"""GPU tests of the reference's matrix:: operations (src/dense/matrixops.cpp)
through the C ABI (symprop_gemmtn, ...): the reference's own known-answer
test for gemmtn (tests/test_matrixops.cpp:8-17) exactly, the rest against
numpy's FP64 LAPACK/BLAS on the same inputs.  Tolerances: products 1e-13
relative (FP64, different summation order); QR 1e-11 absolute on Q;
eigen- and singular vectors by |cos| of the angle to numpy's, >= 1 - 1e-10,
with the order the reference returns (ascending eigenvalues / descending
singular values)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_gemmtn_known_answer(gpu):
    # tests/test_matrixops.cpp:8-17 of the reference: A 3x2, B 3x4
    A = np.array([1, 2, 2, 3, 3, 4], dtype=np.float64)
    B = np.array([1, 2, 3, 4, 2, 3, 4, 5, 3, 4, 5, 6], dtype=np.float64)
    C = gpu.matrix.gemmtn(A, B, 3, 2, 4)
    assert C.reshape(-1).tolist() == [14, 20, 26, 32, 20, 29, 38, 47]


@pytest.mark.parametrize("arow,acol,bcol", [(1000, 16, 816), (100000, 8, 120), (7, 3, 5), (0, 4, 6)])
def test_gemmtn_matches_numpy(gpu, arow, acol, bcol):
    rng = np.random.default_rng(arow + acol)
    A, B = rng.standard_normal((arow, acol)), rng.standard_normal((arow, bcol))
    C = gpu.matrix.gemmtn(A, B, arow, acol, bcol)
    assert rel(C, A.T @ B) < 1e-13
    if arow == 0:
        assert np.all(C == 0)


@pytest.mark.parametrize("I1,I2,m", [(5000, 16, 816), (16, 16, 3876), (33, 7, 1)])
def test_symgemm_matches_numpy(gpu, I1, I2, m):
    rng = np.random.default_rng(I1 + m)
    A, B = rng.standard_normal((I1, m)), rng.standard_normal((I2, m))
    c = rng.integers(1, 24, m).astype(np.float64)
    assert rel(gpu.matrix.symgemm(A, B, c, I1, I2), (A * c) @ B.T) < 1e-13


def test_symsyrk_writes_only_the_upper_triangle(gpu):
    rng = np.random.default_rng(3)
    I1, m = 300, 120
    A = rng.standard_normal((I1, m))
    c = rng.integers(1, 7, m).astype(np.float64)
    C0 = np.full((I1, I1), -7.25)
    C = gpu.matrix.symsyrk(C0, A, c, I1)
    full = (A * c) @ A.T
    iu = np.triu_indices(I1)
    assert rel(C[iu], full[iu]) < 1e-13
    il = np.tril_indices(I1, -1)
    assert np.all(C[il] == -7.25)


@pytest.mark.parametrize("nr,nc", [(200, 16), (50000, 8), (9, 9), (64, 1)])
def test_qr_matches_lapack_q(gpu, nr, nc):
    A = np.random.default_rng(nr).standard_normal((nr, nc))
    Q = gpu.matrix.qr(A, nr, nc)
    Qn, _ = np.linalg.qr(A)  # dgeqrf + dorgqr
    assert np.abs(Q - Qn).max() < 1e-11
    assert np.abs(Q.T @ Q - np.eye(nc)).max() < 1e-13


def _aligned(U, V):
    """|cos| between matching columns."""
    return np.abs(np.sum(U * V, axis=0)) / (np.linalg.norm(U, axis=0) * np.linalg.norm(V, axis=0))


@pytest.mark.parametrize("dim,rank", [(40, 5), (90, 90), (400, 16), (2000, 8)])
def test_syevd_top_eigenvectors_ascending(gpu, dim, rank):
    rng = np.random.default_rng(dim)
    Q, _ = np.linalg.qr(rng.standard_normal((dim, dim)))
    top = min(dim, 24)  # a decaying spectrum with gaps at the top, as Gram matrices have
    lam = np.concatenate([np.linspace(10.0, 4.0, top), rng.uniform(0.0, 1.0, dim - top)])
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    U = gpu.matrix.syevd(A, dim, rank)
    w, V = np.linalg.eigh(A)  # ascending, as LAPACKE_dsyevd
    assert np.all(_aligned(U, V[:, dim - rank:]) > 1 - 1e-10)


@pytest.mark.parametrize("nr,nc,rank", [(3000, 40, 8), (30, 500, 6), (200, 200, 16)])
def test_leftsvd_leading_left_vectors(gpu, nr, nc, rank):
    rng = np.random.default_rng(nr + nc)
    k = min(nr, nc)
    Ul, _ = np.linalg.qr(rng.standard_normal((nr, k)))
    Vr, _ = np.linalg.qr(rng.standard_normal((nc, k)))
    s = np.geomspace(10.0, 0.5, k)
    A = (Ul * s) @ Vr.T
    U = gpu.matrix.leftsvd(A, nr, nc, rank)
    Un = np.linalg.svd(A, full_matrices=False)[0][:, :rank]
    assert np.all(_aligned(U, Un) > 1 - 1e-10)
    assert np.abs(U.T @ U - np.eye(rank)).max() < 1e-12


def test_invalid_shapes_fail_loudly(gpu):
    with pytest.raises(gpu.SympropError) as e:
        gpu.matrix.qr(np.zeros((3, 5)), 3, 5)
    assert e.value.status == gpu.ERR_INVALID
    with pytest.raises(gpu.SympropError) as e:
        gpu.matrix.syevd(np.eye(4), 4, 0)
    assert e.value.status == gpu.ERR_INVALID
    with pytest.raises(gpu.SympropError) as e:
        gpu.matrix.leftsvd(np.ones((4, 3)), 4, 3, 4)
    assert e.value.status == gpu.ERR_INVALID
