"""The P x Q process-grid solve on the GPU building blocks, with P Q ranks as
threads of this process on one device (each with a context of its own; the
ranks meet on the host through LocalGroup communicators, so no kernel ever
waits on another): every rank's pivots equal those of the single-GPU
hplb_pdgesv of the same system, x is within 64 n eps kappa of the single-GPU
x, the assembled factors agree with the single-GPU factors to the same
tolerance, and the residual is below 16.  Plus the four building blocks
against numpy."""
import threading

import numpy as np
import pytest

from gpu_util import from_dev

pytestmark = pytest.mark.gpu
EPS = 2.0 ** -53


def test_grid2d_building_blocks_against_numpy(hlib):
    import torch

    from rochpl_b200.lib import HplError

    rng = np.random.default_rng(5)
    m, ld, ncol = 300, 310, 40
    A0 = rng.standard_normal((ncol, ld))
    A0[7, 123] = 9.5
    A0[7, 200] = -9.5  # a tie in magnitude: the lower row wins
    dA = torch.tensor(A0.reshape(-1), device="cuda")
    v, r = hlib.col_argmax(dA.data_ptr(), ld, 10, m, 7)
    assert (v, r) == (9.5, 123)
    assert hlib.col_argmax(dA.data_ptr(), ld, 5, 5, 7) == (0.0, -1)
    u = rng.standard_normal(ncol)
    du = torch.tensor(u, device="cuda")
    hlib.col_rank1(dA.data_ptr(), ld, 20, 250, 3, 2, 9, 1.7, du.data_ptr())
    want = A0.copy()
    lcol = want[3 + 2, 20:250] / 1.7
    want[3 + 2, 20:250] = lcol
    for c in range(3, 9):
        want[3 + c, 20:250] -= lcol * u[c]
    got = dA.view(ncol, ld).cpu().numpy()
    assert np.allclose(got, want, rtol=1e-14, atol=1e-14)
    n, nrhs = 70, 5
    L = np.tril(rng.standard_normal((n, n)), -1) / n + np.eye(n)  # solutions of order one
    X = rng.standard_normal((n, nrhs))
    dL = torch.tensor(L.T.reshape(-1), device="cuda")
    dX = torch.tensor(X.T.reshape(-1), device="cuda")
    hlib.trsm_lower_unit(n, nrhs, dL.data_ptr(), n, dX.data_ptr(), n)
    assert np.allclose(dX.view(nrhs, n).cpu().numpy().T, np.linalg.solve(L, X), rtol=1e-12,
                       atol=1e-12)
    U = np.triu(rng.standard_normal((n, n))) + n * np.eye(n)
    dU = torch.tensor(U.T.reshape(-1), device="cuda")
    dY = torch.tensor(X.T.reshape(-1), device="cuda")
    dZ = torch.zeros(n * nrhs, dtype=torch.float64, device="cuda")
    hlib.trsm_upper(n, nrhs, dU.data_ptr(), n, dY.data_ptr(), n, dZ.data_ptr(), n)
    assert np.allclose(dZ.view(nrhs, n).cpu().numpy().T, np.linalg.solve(U, X), rtol=1e-12,
                       atol=1e-12)
    with pytest.raises(HplError):
        hlib.col_argmax(dA.data_ptr(), 10, 0, 20, 0)  # ld below the row range
    with pytest.raises(HplError):
        hlib.col_rank1(dA.data_ptr(), ld, 0, 10, 0, 5, 5, 1.0, du.data_ptr())  # kend <= k


def _single(hlib, n, nb, algo):
    import torch

    from rochpl_b200.hpl import default_ld

    ld = default_ld(n)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP = torch.zeros(n, dtype=torch.int32, device="cuda")
    hlib.matgen(n, n + 1, 100, dA.data_ptr(), ld, nb)
    hlib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr(), dP.data_ptr())
    return dX.cpu().numpy(), dP.cpu().numpy(), from_dev(dA, ld, n + 1)[:n]


@pytest.mark.parametrize("n,nb,P,Q,rfact", [(1000, 128, 2, 1, 2), (1000, 128, 2, 2, 2),
                                            (1531, 96, 3, 2, 2), (800, 256, 1, 2, 2),
                                            (1000, 128, 2, 2, 0), (700, 64, 2, 1, 1)])
def test_grid2d_on_virtual_ranks_matches_single_gpu(hlib, oracle, n, nb, P, Q, rfact):
    import torch

    from rochpl_b200.grid2d import (DeviceBackend2D, Grid2D, LocalGrid2D, matgen_local_2d,
                                    pdgesv_2d)
    from rochpl_b200.hpl import Algo
    from rochpl_b200.lib import Library

    algo = Algo(nb, 32, 2, 2, rfact, 1, 0)
    x1, p1, F1 = _single(hlib, n, nb, algo)
    grp = LocalGrid2D(P, Q)
    out, errs = [None] * (P * Q), []

    def work(p, q):
        try:
            lib = Library(0)  # a context of its own per rank
            be = DeviceBackend2D(lib)
            g = Grid2D(n, nb, p, q, P, Q)
            ld = max(g.mp, 1) + 1
            A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64, device="cuda")
            matgen_local_2d(be, g, 100, A, ld)
            x, ipiv, info = pdgesv_2d(be, grp.comms(p, q), g, algo, A, ld)
            torch.cuda.synchronize()
            out[p * Q + q] = (x.cpu().numpy(), ipiv.numpy(), info, g,
                              A.cpu().numpy()[: ld * max(g.nq, 1)].reshape(max(g.nq, 1), ld).T)
            lib.close()
        except BaseException as e:
            errs.append(e)
            grp.abort()

    ts = [threading.Thread(target=work, args=(p, q)) for p in range(P) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    assert not errs, errs
    A0 = oracle.matgen(n, n + 1, 100)
    kappa = np.linalg.cond(A0[:, :n], np.inf)
    tol = 64 * n * EPS * kappa
    F = np.full((n, n + 1), np.nan)
    for x, ipiv, info, g, Fl in out:
        assert info == 0
        assert np.array_equal(ipiv, p1), np.nonzero(ipiv != p1)[0][:8]
        err = np.max(np.abs(x - x1)) / np.max(np.abs(x1))
        assert err <= tol, (err, tol)
        assert oracle.residual(A0, n, x)["resid"] < 16.0
        for lr, i0, h in g.row_blocks():
            for lc, j0, w in g.col_blocks():
                F[i0:i0 + h, j0:j0 + w] = Fl[lr:lr + h, lc:lc + w]
    assert not np.isnan(F).any()
    assert np.max(np.abs(F[:, :n] - F1[:, :n])) <= tol * np.max(np.abs(F1[:, :n])) * 16
