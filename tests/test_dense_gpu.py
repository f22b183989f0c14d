"""GPU tests of the dense-step products: the packed Gram matrix in FP64
(CUDA cores) and the tcgen05 tensor-core products of mixed precision (m x m
Gram, n x n row Gram, panel product W = (A diag(s)) (B diag(s))^T), against
torch FP64 references of the same ops.

The tensor-core products split each operand X = A diag(s) (FP32) into
H = bf16(X) and L = bf16(X - H) and keep H H' + H L' + L H'.  Two
references bound them:
  * the exact split emulation (those three products formed in FP64 from the
    same H and L): the kernel differs from it only by its FP32 accumulation;
  * the FP64 product of the unsplit operands: the split adds the dropped
    L L' term and the BF16 rounding of L, about 2^-17 per product.
On top of the split, the tensor cores accumulate in FP32 and this kernel's
error against the emulation grows with the length K of each accumulation
chain, measured at about 0.5 ulp of FP32 per accumulator update (3 K / 16
updates: three products, K = 16 per instruction); the bound below allows
one ulp per update.  The Gram cuts its K axis into splits added in FP64,
which only shortens the chains.  A separate test checks that both cross
terms H L' and L H' are present, on an input whose L is correlated with H.
"""
import pytest

pytestmark = pytest.mark.gpu


def accum_bound(K):
    """One FP32 ulp per tensor-core accumulator update over a K-long chain."""
    return 3 * K / 16 * 2.0 ** -24


# the split itself: the dropped L L' term and the BF16 rounding of L,
# about 2^-17 of each product
SPLIT_TOL = 1e-5


def split_bf16(X):
    """(H, L) of an FP32 torch tensor, as FP64."""
    H = X.bfloat16().float()
    L = (X - H).bfloat16().float()
    return H.double(), L.double()


def rel(a, b):
    return float((a - b).norm() / b.norm())


def check_split_product(G, Ha, La, Hb, Lb, exact, K):
    import torch
    emul = Ha @ Hb.T + Ha @ Lb.T + La @ Hb.T
    e_emul, e_exact = rel(G, emul), rel(G, exact)
    msg = f"K {K}: vs emulation {e_emul:.2e} (bound {accum_bound(K):.2e}), vs FP64 {e_exact:.2e}"
    assert e_emul <= accum_bound(K), msg
    assert e_exact <= accum_bound(K) + SPLIT_TOL, msg
    assert torch.isfinite(G).all()
    return msg


@pytest.mark.parametrize("n,m", [(1000, 56), (3000, 330), (5000, 130), (777, 200), (20000, 816), (4097, 3876)])
def test_gram_fp64_and_tensor_core(gpu, n, m):
    import torch
    g = torch.Generator(device="cpu").manual_seed(n + m)
    Y = torch.randn(n, m, generator=g, dtype=torch.float64)
    sd = torch.rand(m, generator=g, dtype=torch.float64) + 0.5
    ref = (Y * sd).T @ (Y * sd)
    dY, dsd = Y.cuda(), sd.cuda()
    G = torch.empty(m, m, dtype=torch.float64, device="cuda")
    gpu.gram_device(dY.data_ptr(), n, m, dsd.data_ptr(), G.data_ptr(), gpu.FP64)
    torch.cuda.synchronize()
    e64 = rel(G.cpu(), ref)
    assert e64 < 1e-13, e64
    dY32, dsd32 = Y.float().cuda(), sd.float().cuda()
    G2 = torch.empty(m, m, dtype=torch.float64, device="cuda")
    gpu.gram_device(dY32.data_ptr(), n, m, dsd32.data_ptr(), G2.data_ptr(), gpu.FP32)
    torch.cuda.synchronize()
    Ys = Y.float() * sd.float()
    H, L = split_bf16(Ys)
    print(check_split_product(G2.cpu(), H.T, L.T, H.T, L.T, Ys.double().T @ Ys.double(), n))
    assert torch.equal(G2, G2.T)


def correlated_split_input(g, n, m):
    """FP32 X = H0 (1 + 0.75 2^-9) with H0 exactly representable in BF16:
    then bf16(X) = H0 and L = X - H0 = 0.75 2^-9 H0, so each cross term is
    0.75 2^-9 of H H' with the same sign, and dropping one of them moves the
    product by about 1.5e-3 of its size."""
    import torch
    H0 = torch.randn(n, m, generator=g).bfloat16().float()
    return H0 * (1.0 + 0.75 * 2.0 ** -9)


@pytest.mark.parametrize("which", ["cols", "rows", "panel"])
def test_both_cross_terms_present(gpu, which):
    """Emulations that drop H L' or L H' must be at least 10x further from
    the kernel than the full three-term emulation."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(11)
    n, m, r = 2048, 512, 16
    X = correlated_split_input(g, n, m)
    one32 = torch.ones(m).cuda()
    dX = X.cuda()
    if which == "cols":
        G = torch.empty(m, m, dtype=torch.float64, device="cuda")
        gpu.gram_device(dX.data_ptr(), n, m, one32.data_ptr(), G.data_ptr(), gpu.FP32)
        A = B = X.T
        K = n
    elif which == "rows":
        G = torch.empty(n, n, dtype=torch.float64, device="cuda")
        gpu.symsyrk_device(dX.data_ptr(), one32.data_ptr(), G.data_ptr(), m, n)
        A = B = X
        K = m
    else:
        P = correlated_split_input(g, r, m).double()
        dP, one64 = P.cuda(), torch.ones(m, dtype=torch.float64).cuda()
        G = torch.empty(n, r, dtype=torch.float64, device="cuda")
        gpu.symgemm_device(dX.data_ptr(), dP.data_ptr(), one64.data_ptr(), G.data_ptr(), m, n, r)
        A, B = X, P.float()
        K = m
    torch.cuda.synchronize()
    Ha, La = split_bf16(A)
    Hb, Lb = split_bf16(B)
    Gc = G.cpu()
    full = Ha @ Hb.T + Ha @ Lb.T + La @ Hb.T
    e_full = rel(Gc, full)
    d1 = rel(Gc, Ha @ Hb.T + Ha @ Lb.T)
    d2 = rel(Gc, Ha @ Hb.T + La @ Hb.T)
    msg = f"{which}: vs emulation {e_full:.2e}, vs dropped terms {d1:.2e} / {d2:.2e}"
    print(msg)
    # inputs of one sign per column pair accumulate a larger rounding bias
    # than random ones: twice the random-input bound
    assert e_full <= 2 * accum_bound(K), msg
    assert 10 * e_full < min(d1, d2), msg


@pytest.mark.parametrize("n,m", [(250, 330), (300, 4096), (1000, 816), (129, 64)])
def test_row_gram_tensor_core(gpu, n, m):
    """symsyrk_device: the n x n Gram of the rows of A diag(s) (HOOI's
    dense step when n <= m, AltHOOI's symsyrk)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(7 * n + m)
    A = torch.randn(n, m, generator=g)
    s = torch.rand(m, generator=g) + 0.5
    dA, ds = A.cuda(), s.cuda()
    C = torch.empty(n, n, dtype=torch.float64, device="cuda")
    gpu.symsyrk_device(dA.data_ptr(), ds.data_ptr(), C.data_ptr(), m, n)
    torch.cuda.synchronize()
    X = A * s
    H, L = split_bf16(X)
    print(check_split_product(C.cpu(), H, L, H, L, X.double() @ X.double().T, m))
    assert torch.equal(C, C.T)


@pytest.mark.parametrize("n,m,r", [(20000, 3876, 16), (3000, 330, 10), (1000, 816, 5), (777, 200, 20)])
def test_panel_product_tensor_core(gpu, n, m, r):
    """symgemm_device: W = (A diag(s)) (B diag(s))^T with r <= 16 per panel
    (HOOI's Y D^1/2 V and HOQRI's Y D C^T)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(n + 3 * m + r)
    A = torch.randn(n, m, generator=g)
    B = torch.randn(r, m, generator=g, dtype=torch.float64)
    s = torch.rand(m, generator=g, dtype=torch.float64) + 0.5
    dA, dB, ds = A.cuda(), B.cuda(), s.cuda()
    W = torch.empty(n, r, dtype=torch.float64, device="cuda")
    gpu.symgemm_device(dA.data_ptr(), dB.data_ptr(), ds.data_ptr(), W.data_ptr(), m, n, r)
    torch.cuda.synchronize()
    Xa = A * s.float()
    Xb = (B * s).float()
    Ha, La = split_bf16(Xa)
    Hb, Lb = split_bf16(Xb)
    print(check_split_product(W.cpu(), Ha, La, Hb, Lb, Xa.double() @ Xb.double().T, m))
