"""Multi-RHS solves on the stored HPL factors (hplb_getrs, plain and
transposed), the fused rank-k kernel, and the differentiable solve built on
them: checked against numpy FP64 solves, an FP64 reference gradient and
central finite differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 2.0 ** -53


def _lcg_system(oracle, n, nrhs, seed=100):
    """A (n x n) and B (n x nrhs) from the HPL LCG: B is the next nrhs columns."""
    M = oracle.matgen(n, n + nrhs, seed)
    return np.array(M[:n, :n]), np.array(M[:n, n:n + nrhs])


def _dev_colmajor(M):
    import torch

    return torch.from_numpy(np.ascontiguousarray(np.asarray(M).T)).cuda()


def _factor(hlib, A, nb, nbmin=16):
    import torch

    from rochpl_b200.hpl import Algo

    n = A.shape[0]
    LU = _dev_colmajor(A)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = hlib.getrf(Algo(nb, nbmin, 2, 2, 2, 1, 0).c(), n, LU.data_ptr(), n, ipiv.data_ptr())
    assert info == 0
    return LU, ipiv


@pytest.mark.parametrize("n,nb,nrhs", [(1, 1, 1), (100, 32, 1), (300, 64, 7), (1000, 128, 32),
                                       (1005, 100, 3), (2048, 256, 64), (777, 96, 16),
                                       (64, 16, 4), (64, 8, 4), (200, 16, 3)])
@pytest.mark.parametrize("trans", [0, 1])
def test_getrs_matches_numpy(hlib, oracle, n, nb, nrhs, trans):
    A, B = _lcg_system(oracle, n, nrhs)
    LU, ipiv = _factor(hlib, A, nb)
    X = _dev_colmajor(B)
    hlib.getrs(trans, n, nb, nrhs, LU.data_ptr(), n, ipiv.data_ptr(), X.data_ptr(), n)
    x = X.cpu().numpy().T
    M = A.T if trans else A
    ref = np.linalg.solve(M, B)
    kappa = np.linalg.cond(A, np.inf)
    err = np.max(np.abs(x - ref)) / np.max(np.abs(ref))
    assert err <= 64 * n * EPS * kappa, (err, kappa)


def test_getrf_pivots_equal_pdgesv(hlib, oracle):
    """getrf takes exactly the panels and pivots of pdgesv on the same A."""
    import torch

    from rochpl_b200.hpl import Algo

    n, nb = 700, 64
    ld = oracle.default_ld(n)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + 1, 100, dA.data_ptr(), ld)
    A = dA.view(n + 1, ld)[:n, :n].cpu().numpy().T.copy()
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    p1 = torch.zeros(n, dtype=torch.int32, device="cuda")
    hlib.pdgesv(Algo(nb, 16, 2, 2, 2, 1, 0).c(), n, dA.data_ptr(), ld, dX.data_ptr(),
                p1.data_ptr())
    LU, p2 = _factor(hlib, A, nb)
    assert torch.equal(p1, p2)
    lu1 = dA.view(n + 1, ld)[:n, :n]
    assert torch.allclose(lu1, LU.view(n, n), rtol=1e-13, atol=1e-14)


def test_getrs_rejects_bad_pivots(hlib, oracle):
    import torch

    from rochpl_b200.lib import HplError

    A, B = _lcg_system(oracle, 64, 2)
    LU, ipiv = _factor(hlib, A, 16)
    bad = ipiv.clone()
    bad[10] = 3  # below its own row
    X = _dev_colmajor(B)
    with pytest.raises(HplError):
        hlib.getrs(0, 64, 16, 2, LU.data_ptr(), 64, bad.data_ptr(), X.data_ptr(), 64)
    bad[10] = 64  # past the last row
    with pytest.raises(HplError):
        hlib.getrs(1, 64, 16, 2, LU.data_ptr(), 64, bad.data_ptr(), X.data_ptr(), 64)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (100, 37, 5), (1000, 1000, 32), (513, 700, 64),
                                   (64, 64, 0)])
@pytest.mark.parametrize("accumulate", [False, True])
def test_rank_k_matches_torch(hlib, m, n, k, accumulate):
    import torch

    g = torch.Generator().manual_seed(m * 7 + n + k)
    A = torch.rand(k, m + 3, generator=g, dtype=torch.float64).cuda()  # column-major m x k, ld m+3
    B = torch.rand(k, n + 1, generator=g, dtype=torch.float64).cuda()  # column-major n x k
    Cc = torch.rand(n, m + 2, generator=g, dtype=torch.float64).cuda()  # column-major m x n
    C0 = Cc.clone()
    hlib.rank_k(m, n, k, -0.75, A.data_ptr(), m + 3, B.data_ptr(), n + 1, Cc.data_ptr(), m + 2,
                accumulate)
    ref = -0.75 * (A[:, :m].t() @ B[:, :n])
    if accumulate:
        ref = ref + C0[:, :m].t()
    assert torch.allclose(Cc[:, :m].t(), ref, rtol=1e-14, atol=1e-13)
    assert torch.equal(Cc[:, m:], C0[:, m:])  # padding rows untouched


def _np_grads(A, B, Xbar):
    X = np.linalg.solve(A, B)
    Bbar = np.linalg.solve(A.T, Xbar)
    return X, -Bbar @ X.T, Bbar


@pytest.mark.parametrize("n,nrhs,nb", [(200, 3, 64), (1000, 32, 128), (513, 1, 100)])
def test_hpl_solve_gradient_matches_fp64_reference(hlib, oracle, n, nrhs, nb):
    import torch

    from rochpl_b200.autograd import hpl_solve

    A, B = _lcg_system(oracle, n, nrhs, seed=100 + n)
    rng = np.random.default_rng(n)
    Xbar = rng.standard_normal((n, nrhs))
    tA = torch.tensor(A, device="cuda", requires_grad=True)
    tB = torch.tensor(B, device="cuda", requires_grad=True)
    X = hpl_solve(tA, tB, nb=nb)
    X.backward(torch.tensor(Xbar, device="cuda"))
    Xr, gAr, gBr = _np_grads(A, B, Xbar)
    kappa = np.linalg.cond(A, np.inf)
    tol = 64 * n * EPS * kappa
    for got, ref in ((X.detach(), Xr), (tA.grad, gAr), (tB.grad, gBr)):
        got = got.cpu().numpy()
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err <= tol, (err, tol)


def test_hpl_solve_central_finite_differences(hlib, oracle):
    """Directional derivatives of L(A, B) = <W, X(A, B)> against central
    differences with step 1e-6."""
    import torch

    from rochpl_b200.autograd import hpl_solve

    n, nrhs = 64, 4
    A, B = _lcg_system(oracle, n, nrhs, seed=11)
    A = A + 4.0 * np.eye(n)  # well conditioned, so the differences are accurate
    rng = np.random.default_rng(5)
    W = torch.tensor(rng.standard_normal((n, nrhs)), device="cuda")
    dA = torch.tensor(rng.standard_normal((n, n)), device="cuda")
    dB = torch.tensor(rng.standard_normal((n, nrhs)), device="cuda")
    tA = torch.tensor(A, device="cuda", requires_grad=True)
    tB = torch.tensor(B, device="cuda", requires_grad=True)
    (hpl_solve(tA, tB, nb=16) * W).sum().backward()
    h = 1e-6

    def L(Ap, Bp):
        with torch.no_grad():
            return float((hpl_solve(Ap, Bp, nb=16) * W).sum())

    Ad, Bd = tA.detach(), tB.detach()
    fdA = (L(Ad + h * dA, Bd) - L(Ad - h * dA, Bd)) / (2 * h)
    fdB = (L(Ad, Bd + h * dB) - L(Ad, Bd - h * dB)) / (2 * h)
    assert abs(float((tA.grad * dA).sum()) - fdA) <= 1e-6 * max(1.0, abs(fdA))
    assert abs(float((tB.grad * dB).sum()) - fdB) <= 1e-6 * max(1.0, abs(fdB))


def test_hpl_solve_gradients_at_n16384_with_32_rhs(hlib):
    """The differentiable solve at its own config size (N = 16384, 32 RHS, the
    HPL LCG system of seed 100): X, Abar and Bbar against an FP64 reference
    from torch's dense solve within 64 N eps kappa_oo, and directional
    derivatives along unit-norm directions against central differences with
    step 1e-6 (relative tolerance 1e-4)."""
    import torch

    from rochpl_b200.autograd import hpl_solve

    n, nrhs = 16384, 32
    M = torch.empty((n + nrhs) * n, dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + nrhs, 100, M.data_ptr(), n)
    Mc = M.view(n + nrhs, n)
    A = Mc[:n].t().contiguous().requires_grad_(True)
    B = Mc[n:].t().contiguous().requires_grad_(True)
    del M, Mc
    g = torch.Generator(device="cuda").manual_seed(7)
    Xbar = torch.randn(n, nrhs, generator=g, dtype=torch.float64, device="cuda")
    X = hpl_solve(A, B, nb=512)
    X.backward(Xbar)
    with torch.no_grad():
        Xr = torch.linalg.solve(A, B)
        Bbar = torch.linalg.solve(A.t(), Xbar)
        Abar = -Bbar @ Xr.t()
        kappa = float(A.abs().sum(dim=1).max()) * float(
            torch.linalg.inv(A).abs().sum(dim=1).max())
    tol = 64 * n * EPS * kappa
    for got, ref in ((X.detach(), Xr), (A.grad, Abar), (B.grad, Bbar)):
        err = float((got - ref).abs().max() / ref.abs().max())
        assert err <= tol, (err, tol)
    del Xr, Bbar, Abar
    # Directions: the normalised sum of the computed gradient's direction and a
    # seeded random unit direction, so that the derivative is of the order of
    # the gradient's norm and far above the rounding floor of the difference
    # quotient (a purely random direction of this dimension sees a derivative
    # about sqrt(N^2) times smaller).
    h = 1e-6
    dA = torch.randn(n, n, generator=g, dtype=torch.float64, device="cuda")
    dB = torch.randn(n, nrhs, generator=g, dtype=torch.float64, device="cuda")
    dA = dA / dA.norm() + A.grad / A.grad.norm()
    dB = dB / dB.norm() + B.grad / B.grad.norm()
    dA /= dA.norm()
    dB /= dB.norm()

    def L(Ap, Bp):
        with torch.no_grad():
            return float((hpl_solve(Ap, Bp, nb=512) * Xbar).sum())

    Ad, Bd = A.detach(), B.detach()
    fdA = (L(Ad + h * dA, Bd) - L(Ad - h * dA, Bd)) / (2 * h)
    fdB = (L(Ad, Bd + h * dB) - L(Ad, Bd - h * dB)) / (2 * h)
    assert abs(float((A.grad * dA).sum()) - fdA) <= 1e-4 * abs(fdA)
    assert abs(float((B.grad * dB).sum()) - fdB) <= 1e-4 * abs(fdB)


def test_hpl_solve_vector_rhs_and_errors(hlib, oracle):
    import torch

    from rochpl_b200.autograd import hpl_solve

    A, B = _lcg_system(oracle, 50, 1)
    tA = torch.tensor(A, device="cuda")
    x = hpl_solve(tA, torch.tensor(B[:, 0], device="cuda"))
    assert x.shape == (50,)
    assert np.allclose(x.cpu().numpy(), np.linalg.solve(A, B[:, 0]), rtol=1e-10, atol=1e-12)
    with pytest.raises(ValueError):
        hpl_solve(tA.float(), torch.tensor(B, device="cuda").float())
    with pytest.raises(ValueError):
        hpl_solve(tA.cpu(), torch.tensor(B))


def test_hpl_solve_leaves_column_major_inputs_untouched(hlib, oracle):
    """A and B that are already column-major (strides (1, n), as a tensor made
    from a Fortran-ordered array is) must be copied, not solved in place."""
    import torch

    from rochpl_b200.autograd import hpl_solve

    n = 80
    A, B = _lcg_system(oracle, n, 3)
    tA = torch.tensor(np.asfortranarray(A), device="cuda")
    tB = torch.tensor(np.asfortranarray(B), device="cuda")
    assert tB.stride() == (1, n) and tA.stride() == (1, n)
    A0, B0 = tA.clone(), tB.clone()
    ref = np.linalg.solve(A, B)
    for _ in range(2):
        X = hpl_solve(tA, tB, nb=16)
        assert torch.equal(tA, A0) and torch.equal(tB, B0)
        assert np.allclose(X.cpu().numpy(), ref, rtol=1e-10, atol=1e-12)


def test_hpl_solve_batch_gradients(hlib, oracle):
    """Batched differentiable solve over systems with N in [64, 512]: X, Abar and
    Bbar of every system against the FP64 numpy reference gradient."""
    import torch

    from rochpl_b200.autograd import hpl_solve_batch
    from rochpl_b200.batch import BatchPlan

    rng = np.random.default_rng(1)
    sizes = [64, 100, 257, 512, 333]
    nrhs = 8
    plan = BatchPlan(hlib, np.array(sizes, dtype=np.int32), nrhs)
    As, Bs, Ws = [], [], []
    for i, n in enumerate(sizes):
        A, B = _lcg_system(oracle, n, nrhs, seed=500 + i)
        As.append(torch.tensor(A, device="cuda", requires_grad=True))
        Bs.append(torch.tensor(B, device="cuda", requires_grad=True))
        Ws.append(rng.standard_normal((n, nrhs)))
    Xs = hpl_solve_batch(plan, As, Bs)
    loss = sum((X * torch.tensor(W, device="cuda")).sum() for X, W in zip(Xs, Ws))
    loss.backward()
    for i, n in enumerate(sizes):
        A = As[i].detach().cpu().numpy()
        B = Bs[i].detach().cpu().numpy()
        Xr, gAr, gBr = _np_grads(A, B, Ws[i])
        tol = 64 * n * EPS * np.linalg.cond(A, np.inf)
        for got, ref in ((Xs[i].detach(), Xr), (As[i].grad, gAr), (Bs[i].grad, gBr)):
            got = got.cpu().numpy()
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= tol, (i, n)
