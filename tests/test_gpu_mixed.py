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
@pytest.mark.parametrize("ldc_kind", ["odd", "aligned"])
def test_gemm_lp_matches_torch_fp32(hlib, m, n, k, bf16, ldc_kind):
    """ldc_kind "aligned" (a 16-byte leading dimension) takes the TMA
    reduce-add epilogue, "odd" the epilogue that loads and stores C itself."""
    import torch

    g = torch.Generator(device="cpu").manual_seed(m + 3 * n + 7 * k + bf16)
    dt = torch.bfloat16 if bf16 else torch.float16
    lda = k + 8
    A = ((torch.rand(m, lda, generator=g) - 0.5) * 2).to(dt).cuda()
    B = ((torch.rand(n, lda, generator=g) - 0.5) * 2).to(dt).cuda()
    tm, tn = (m + 127) // 128, (n + 255) // 256
    sA = (2.0 ** torch.randint(-3, 4, (tm,), generator=g).float()).cuda()
    sB = (2.0 ** torch.randint(-3, 4, (tn,), generator=g).float()).cuda()
    if ldc_kind == "aligned":
        ldc = (m + 3) // 4 * 4 + 4
    else:
        ldc = m + 5 if (m + 5) % 4 else m + 6
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


# ---- hplb_pdgesv_mixed against the FP64 oracle ----
EPS = 2.0 ** -53


def _mixed(hlib, oracle, n, nb, precision, stored, nbmin=32, seed=100):
    import torch

    from gpu_util import to_dev
    from rochpl_b200.hpl import Algo

    ld = oracle.default_ld(n)
    A0 = oracle.matgen(n, n + 1, seed, ld=ld)
    dA = to_dev(A0) if stored else None
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = hlib.pdgesv_mixed(Algo(nb, nbmin, 2, 2, 2, 1, 0).c(), n, dX.data_ptr(), seed=seed,
                            A=dA.data_ptr() if stored else None, ld=ld if stored else 0,
                            precision=precision, target_resid=1.0)
    return rep, dX.cpu().numpy(), A0, dA


# The x3 forms give FP32-accurate factors; the plain 16-bit forms are checked
# where the preconditioner they give still converges quickly.
MIXED_CASES = [(1000, 128, 2, True), (1000, 128, 3, False), (4096, 256, 2, False),
               (4096, 256, 3, True), (2048, 512, 2, True), (1000, 128, 0, True),
               (1000, 128, 1, False), (777, 96, 2, True)]


@pytest.mark.parametrize("n,nb,precision,stored", MIXED_CASES)
def test_mixed_solve_reaches_fp64_accuracy(hlib, oracle, n, nb, precision, stored):
    rep, x, A0, dA = _mixed(hlib, oracle, n, nb, precision, stored)
    assert rep["info"] == 0 and rep["converged"] == 1, rep
    assert rep["resid"] < 1.0, rep
    res = oracle.residual(A0, n, x)
    assert res["resid"] < 16.0, res
    Ao = A0.copy(order="F")
    xo, _, _ = oracle.pdgesv(Ao, n, nb, 32, 2, 2, 2)
    kappa = np.linalg.cond(A0[:n, :n], np.inf)
    err = np.max(np.abs(x - xo)) / np.max(np.abs(xo))
    assert err <= 64 * n * EPS * kappa, (err, kappa)
    if stored:  # the FP64 [A|b] is not modified
        from gpu_util import from_dev

        assert np.array_equal(from_dev(dA, oracle.default_ld(n), n + 1)[:n], A0[:n])


def test_mixed_lcg_and_stored_agree(hlib, oracle):
    """The regenerated LCG path and the stored-A path take the same steps."""
    r1, x1, _, _ = _mixed(hlib, oracle, 1500, 128, 2, True)
    r2, x2, _, _ = _mixed(hlib, oracle, 1500, 128, 2, False)
    assert r1["gmres_iters"] == r2["gmres_iters"]
    assert np.array_equal(x1, x2)


def test_mixed_pivots_match_fp32_lu_of_oracle_order(hlib, oracle):
    """Pivots of the mixed LU are a permutation consistent with HPL's swap
    convention (ipiv[j] >= j) and the resid_lu of the low-precision LU alone
    is reported."""
    import torch

    from rochpl_b200.hpl import Algo

    n = 1200
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP = torch.zeros(n, dtype=torch.int32, device="cuda")
    rep = hlib.pdgesv_mixed(Algo(128, 32, 2, 2, 2, 1, 0).c(), n, dX.data_ptr(), seed=7,
                            ipiv=dP.data_ptr())
    p = dP.cpu().numpy()
    assert np.all(p >= np.arange(n)) and np.all(p < n)
    assert rep["resid_lu"] >= rep["resid"] and rep["converged"] == 1


def test_mixed_bad_arguments(hlib):
    import torch

    from rochpl_b200.hpl import Algo
    from rochpl_b200.lib import HplError

    dX = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(HplError):
        hlib.pdgesv_mixed(Algo(32, 8, 2, 2, 2, 1, 0).c(), 64, dX.data_ptr(), precision=4)
    with pytest.raises(HplError):
        hlib.pdgesv_mixed(Algo(32, 8, 2, 2, 2, 1, 0).c(), 64, dX.data_ptr(), restart=61)
    with pytest.raises(HplError):  # stored A with ld < n
        hlib.pdgesv_mixed(Algo(32, 8, 2, 2, 2, 1, 0).c(), 64, dX.data_ptr(),
                          A=dX.data_ptr(), ld=10)
    rep = hlib.pdgesv_mixed(Algo(32, 8, 2, 2, 2, 1, 0).c(), 0, dX.data_ptr())
    assert rep["status"] == 0
