"""GPU tests of the dense-step kernels: the packed Gram matrix in FP64
(CUDA cores) and on the tcgen05 tensor cores (split-BF16, FP32 accumulate),
against a plain torch FP64 reference of the same op."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,m", [(1000, 56), (3000, 330), (5000, 130), (777, 200), (20000, 816)])
def test_gram_fp64_and_tensor_core(gpu, n, m):
    import torch
    g = torch.Generator(device="cpu").manual_seed(n + m)
    Y = torch.randn(n, m, generator=g, dtype=torch.float64)
    sd = torch.rand(m, generator=g, dtype=torch.float64) + 0.5
    ref = (Y * sd).T @ (Y * sd)
    dY = Y.cuda()
    dsd = sd.cuda()
    G = torch.empty(m, m, dtype=torch.float64, device="cuda")
    gpu.gram_device(dY.data_ptr(), n, m, dsd.data_ptr(), G.data_ptr(), gpu.FP64)
    torch.cuda.synchronize()
    e64 = (G.cpu() - ref).norm() / ref.norm()
    assert e64 < 1e-13, e64
    dY32 = Y.float().cuda()
    dsd32 = sd.float().cuda()
    G2 = torch.empty(m, m, dtype=torch.float64, device="cuda")
    gpu.gram_device(dY32.data_ptr(), n, m, dsd32.data_ptr(), G2.data_ptr(), gpu.FP32)
    torch.cuda.synchronize()
    Ys = Y.float() * sd.float()
    ref32 = Ys.double().T @ Ys.double()
    e32 = (G2.cpu() - ref32).norm() / ref32.norm()
    # against exact FP64: split-BF16 (hi + lo) operands lose ~2^-17 per
    # product and FP32 accumulation adds sqrt(n) eps32
    assert e32 < 5e-4, e32
    # against an exact emulation of the split (H = bf16(Y'), L = bf16(Y' - H),
    # G = H^T H + H^T L + L^T H in FP64): only FP32 accumulation differs
    H = Ys.bfloat16().float()
    Lo = (Ys - H).bfloat16().float()
    H, Lo = H.double(), Lo.double()
    emul = H.T @ H + H.T @ Lo + Lo.T @ H
    ee = (G2.cpu() - emul).norm() / emul.norm()
    # the tensor-core FP32 accumulation over K = 3n terms
    assert ee < 2e-4, ee
    assert torch.equal(G2.cpu(), G2.cpu().T)
