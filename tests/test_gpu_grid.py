"""The 1 x Q process-grid solve on the GPU building blocks, with Q ranks as
threads of this process on one device (LocalGroup: the ranks meet on the host;
no kernel ever waits on another): every rank's pivots equal those of the
single-GPU hplb_pdgesv of the same system, its columns of the factors are the
single-GPU factors bit for bit (the same kernels per column), and x is within
64 n eps kappa of the single-GPU x; the residual is below 16."""
import threading

import numpy as np
import pytest

from gpu_util import from_dev

pytestmark = pytest.mark.gpu
EPS = 2.0 ** -53


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


@pytest.mark.parametrize("n,nb,Q", [(1000, 128, 1), (2048, 256, 2), (2049, 256, 3),
                                    (1531, 96, 4)])
def test_grid_on_virtual_ranks_matches_single_gpu(hlib, oracle, n, nb, Q):
    import torch

    from rochpl_b200.grid import DeviceBackend, Grid1xQ, LocalGroup, matgen_local, pdgesv_grid
    from rochpl_b200.hpl import Algo, default_ld
    from rochpl_b200.lib import Library

    algo = Algo(nb, 32, 2, 2, 2, 1, 0)
    x1, p1, F1 = _single(hlib, n, nb, algo)
    grp = LocalGroup(Q)
    out, errs = [None] * Q, []

    def work(q):
        try:
            lib = Library(0)  # a context of its own per rank
            be = DeviceBackend(lib)
            g = Grid1xQ(n, nb, q, Q)
            ld = default_ld(n)
            A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64, device="cuda")
            matgen_local(be, g, 100, A, ld)
            x, ipiv, info = pdgesv_grid(be, grp.member(q), g, algo, A, ld)
            torch.cuda.synchronize()
            F = from_dev(A, ld, max(g.nq, 1))
            out[q] = (x.cpu().numpy(), ipiv.cpu().numpy(), info, g, F)
            lib.close()
        except BaseException as e:
            errs.append(e)
            grp.barrier.abort()

    ts = [threading.Thread(target=work, args=(q,)) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    assert not errs, errs
    A0 = oracle.matgen(n, n + 1, 100)
    kappa = np.linalg.cond(A0[:, :n], np.inf)
    covered = 0
    for x, ipiv, info, g, F in out:
        assert info == 0
        assert np.array_equal(ipiv, p1)
        err = np.max(np.abs(x - x1)) / np.max(np.abs(x1))
        assert err <= 64 * n * EPS * kappa, (err, kappa)
        assert oracle.residual(A0, n, x)["resid"] < 16.0
        for lc, g0, w in g.local_blocks():
            assert np.array_equal(F[:n, lc:lc + w].view(np.uint64), F1[:, g0:g0 + w].view(np.uint64))
            covered += w
    assert covered == n + 1


def test_grid_building_blocks_reject_bad_arguments(hlib):
    import torch

    from rochpl_b200.hpl import Algo
    from rochpl_b200.lib import HplError

    A = torch.zeros(64 * 65, dtype=torch.float64, device="cuda")
    piv = torch.zeros(16, dtype=torch.int32, device="cuda")
    with pytest.raises(HplError):  # panel past the last row
        hlib.panel_factor(Algo(16, 8, 2, 2, 2, 1, 0).c(), 64, 60, 16, A.data_ptr(), 64, 0,
                          piv.data_ptr())
    bad = torch.full((16,), 1000, dtype=torch.int32, device="cuda")
    with pytest.raises(HplError):  # pivots outside [j + k, n)
        hlib.panel_update(64, 0, 16, A.data_ptr(), 64, bad.data_ptr(), A.data_ptr(), 64, 16, 8)
    v = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(HplError):
        hlib.trsv_block(64, 60, 16, A.data_ptr(), 64, 0, v.data_ptr(), v.data_ptr(),
                        v.data_ptr(), v.data_ptr())
