"""Mixed-precision form: the tcgen05 low-precision trailing update against a
plain torch fp32 reference of the same op, and (below) the mixed solve against
the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (128, 256, 512), (200, 300, 512),
                                   (1000, 513, 512), (4096, 2048, 512), (77, 1000, 128),
                                   (1500, 40, 256), (2048, 4096, 192)])
@pytest.mark.parametrize("bf16", [True, False])
def test_gemm_lp_matches_torch_fp32(hlib, m, n, k, bf16):
    import torch

    g = torch.Generator(device="cpu").manual_seed(m + 3 * n + 7 * k + bf16)
    dt = torch.bfloat16 if bf16 else torch.float16
    lda = k + 8
    A = ((torch.rand(m, lda, generator=g) - 0.5) * 2).to(dt).cuda()
    B = ((torch.rand(n, lda, generator=g) - 0.5) * 2).to(dt).cuda()
    tm, tn = (m + 127) // 128, (n + 255) // 256
    sA = (2.0 ** torch.randint(-3, 4, (tm,), generator=g).float()).cuda()
    sB = (2.0 ** torch.randint(-3, 4, (tn,), generator=g).float()).cuda()
    ldc = m + 5
    C = (torch.rand(n, ldc, generator=g) - 0.5).cuda()  # column-major C: C.T[:m]
    C0 = C.clone()
    hlib.gemm_lp_sub(bf16, m, n, k, A.data_ptr(), lda, B.data_ptr(), lda, sA.data_ptr(),
                     sB.data_ptr(), C.data_ptr(), ldc)
    prod = A[:, :k].float() @ B[:, :k].float().T  # m x n, fp32
    scale = sA.repeat_interleave(128)[:m, None] * sB.repeat_interleave(256)[None, :n]
    ref = C0.T[:m].clone() - scale * prod
    got = C.T[:m]
    err = (got - ref).abs().max().item()
    tol = 2e-6 * k * float(scale.max())
    assert err <= tol, (err, tol)
    assert torch.equal(C.T[m:], C0.T[m:])  # padding rows untouched
