"""Batched solver (hplb_batch_*): per-system LCG generation bit-exact with the
oracle's generator, X against LAPACK (scipy) FP64 solves with the x tolerance
of the single-system tests, pivots equal to LAPACK getrf's, the stored-factor
solves (plain and transposed), the batched rank-k product, the on-device HPL
residual against a numpy computation of the same formula, errors, and the
autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 2.0 ** -53


def _plan(hlib, n, nrhs, nb_by_class=None):
    from rochpl_b200.batch import BatchPlan

    return BatchPlan(hlib, n, nrhs, nb_by_class)


def _pools(plan):
    import torch

    dA = torch.zeros(max(plan.a_elems, 1), dtype=torch.float64, device="cuda")
    dB = torch.zeros(max(plan.b_elems, 1), dtype=torch.float64, device="cuda")
    dP = torch.zeros(max(plan.p_elems, 1), dtype=torch.int32, device="cuda")
    dI = torch.full((plan.count,), -1, dtype=torch.int32, device="cuda")
    return dA, dB, dP, dI


def _system(plan, i, hA, hB):
    n, r = int(plan.n[i]), int(plan.nrhs[i])
    A = hA[plan.a_off[i]:plan.a_off[i] + n * n].reshape(n, n).T
    B = hB[plan.b_off[i]:plan.b_off[i] + n * r].reshape(r, n).T
    return A, B


SIZES = [1, 2, 7, 31, 32, 33, 47, 64, 100, 129, 257, 400, 513, 700, 1024]


@pytest.mark.parametrize("nrhs", [1, 16, 64])
@pytest.mark.parametrize("mode", ["default", "recursive"])
def test_batch_gesv_matches_lapack(hlib, oracle, nrhs, mode):
    import scipy.linalg as sl

    from rochpl_b200.lib import HPLB_BATCH_RECURSIVE

    n = np.array(SIZES, dtype=np.int32)
    plan = _plan(hlib, n, nrhs, None if mode == "default" else [HPLB_BATCH_RECURSIVE] * 6)
    seeds = 100 + np.arange(plan.count, dtype=np.uint64)
    dA, dB, dP, dI = _pools(plan)
    plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())
    hA0, hB0 = dA.cpu().numpy(), dB.cpu().numpy()
    plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    hA, hX, hP = dA.cpu().numpy(), dB.cpu().numpy(), dP.cpu().numpy()
    assert np.all(dI.cpu().numpy() == 0)
    for i in range(plan.count):
        A0, B0 = _system(plan, i, hA0, hB0)
        m = int(n[i])
        # The generator is the HPL LCG of the system's seed, m rows.
        M = oracle.matgen(m, m + nrhs, int(seeds[i]))
        assert np.array_equal(A0, M[:m, :m]) and np.array_equal(B0, M[:m, m:])
        lu, piv = sl.lu_factor(A0)
        p = hP[plan.p_off[i]:plan.p_off[i] + m]
        assert np.array_equal(p, piv), f"system {i} (n={m}): pivots differ"
        LUg, X = _system(plan, i, hA, hX)
        assert np.allclose(LUg, lu, rtol=1e-9, atol=1e-12 * m)
        ref = np.linalg.solve(A0, B0)
        kappa = np.linalg.cond(A0, np.inf)
        err = np.max(np.abs(X - ref)) / np.max(np.abs(ref))
        assert err <= 64 * m * EPS * kappa, (i, m, err, kappa)


def _np_resid(A0, B0, X):
    m = A0.shape[0]
    worst = 0.0
    for c in range(B0.shape[1]):
        r = np.max(np.abs(B0[:, c] - A0 @ X[:, c]))
        worst = max(worst, r / (EPS * (np.max(np.sum(np.abs(A0), 1)) * np.max(np.abs(X[:, c]))
                                       + np.max(np.abs(B0[:, c]))) * m))
    return worst


def test_batch_residual_matches_numpy(hlib):
    """Below 16 for the computed solutions; for solutions perturbed well above
    rounding (so that b - A x does not depend on the summation order) the
    device value equals numpy's to 1e-6."""
    import torch

    n = np.array([5, 64, 300, 1000], dtype=np.int32)
    nrhs = np.array([3, 1, 16, 9], dtype=np.int32)
    plan = _plan(hlib, n, nrhs)
    seeds = np.array([7, 8, 9, 10], dtype=np.uint64)
    dA, dB, dP, dI = _pools(plan)
    plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())
    hA0, hB0 = dA.cpu().numpy(), dB.cpu().numpy()
    plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    res = torch.zeros(plan.count, dtype=torch.float64, device="cuda")
    plan.residual(seeds, dB.data_ptr(), res.data_ptr())
    assert float(res.max()) < 16.0 and float(res.min()) >= 0.0
    hX = dB.cpu().numpy() * (1.0 + 1e-7 * np.sin(np.arange(plan.b_elems)))
    dB.copy_(torch.from_numpy(hX).cuda())
    plan.residual(seeds, dB.data_ptr(), res.data_ptr())
    got = res.cpu().numpy()
    for i in range(plan.count):
        A0, B0 = _system(plan, i, hA0, hB0)
        _, X = _system(plan, i, hA0, hX)
        ref = _np_resid(A0, B0, X)
        assert ref > 1e3 and abs(got[i] - ref) <= 1e-6 * ref, (i, got[i], ref)


@pytest.mark.parametrize("trans", [0, 1])
def test_batch_getrs_matches_numpy(hlib, trans):
    n = np.array([3, 40, 96, 250, 512], dtype=np.int32)
    plan = _plan(hlib, n, 5)
    seeds = 55 + np.arange(plan.count, dtype=np.uint64)
    dA, dB, dP, dI = _pools(plan)
    plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())
    hA0, hB0 = dA.cpu().numpy(), dB.cpu().numpy()
    plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    # Solve again with the stored factors, for the original right-hand sides.
    dB.copy_(__import__("torch").from_numpy(hB0).cuda())
    plan.getrs(trans, dA.data_ptr(), dP.data_ptr(), dB.data_ptr())
    hX = dB.cpu().numpy()
    for i in range(plan.count):
        A0, B0 = _system(plan, i, hA0, hB0)
        _, X = _system(plan, i, hA0, hX)
        M = A0.T if trans else A0
        ref = np.linalg.solve(M, B0)
        m = int(n[i])
        kappa = np.linalg.cond(A0, np.inf)
        assert np.max(np.abs(X - ref)) / np.max(np.abs(ref)) <= 64 * m * EPS * kappa


def test_batch_rank_k_matches_numpy(hlib):
    import torch

    n = np.array([1, 17, 64, 130, 500], dtype=np.int32)
    nrhs = np.array([1, 5, 32, 64, 40], dtype=np.int32)
    plan = _plan(hlib, n, nrhs)
    g = torch.Generator().manual_seed(3)
    X = torch.rand(plan.b_elems, generator=g, dtype=torch.float64).cuda()
    Y = torch.rand(plan.b_elems, generator=g, dtype=torch.float64).cuda()
    Cp = torch.zeros(plan.a_elems, dtype=torch.float64, device="cuda")
    plan.rank_k(-1.5, X.data_ptr(), Y.data_ptr(), Cp.data_ptr())
    hX, hY, hC = X.cpu().numpy(), Y.cpu().numpy(), Cp.cpu().numpy()
    for i in range(plan.count):
        m, r = int(n[i]), int(nrhs[i])
        Xi = hX[plan.b_off[i]:plan.b_off[i] + m * r].reshape(r, m).T
        Yi = hY[plan.b_off[i]:plan.b_off[i] + m * r].reshape(r, m).T
        Ci = hC[plan.a_off[i]:plan.a_off[i] + m * m].reshape(m, m).T
        assert np.allclose(Ci, -1.5 * Xi @ Yi.T, rtol=1e-13, atol=1e-13)


def test_batch_zero_pivot_is_reported(hlib):
    import torch

    n = np.array([4, 6], dtype=np.int32)
    plan = _plan(hlib, n, 1)
    dA, dB, dP, dI = _pools(plan)
    plan.matgen(np.array([1, 2], dtype=np.uint64), dA.data_ptr(), dB.data_ptr())
    hA = dA.cpu().numpy()
    o = plan.a_off[1]
    hA[o + 2 * 6:o + 3 * 6] = 0.0  # column 2 of system 1 is zero
    dA.copy_(torch.from_numpy(hA).cuda())
    plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    info = dI.cpu().numpy()
    assert info[0] == 0 and info[1] == 3


def test_batch_arguments(hlib):
    from rochpl_b200.lib import HplError

    with pytest.raises(HplError):
        _plan(hlib, np.array([4, 3000], dtype=np.int32), 1)  # above HPLB_BATCH_MAX_N
    with pytest.raises(HplError):
        _plan(hlib, np.array([4, 0], dtype=np.int32), 1)
    with pytest.raises(HplError):
        _plan(hlib, np.array([4], dtype=np.int32), 1, nb_by_class=[8, 16, 12, 16, 16, 16])
    plan = _plan(hlib, np.array([1024, 40], dtype=np.int32), 2, nb_by_class=[32] * 6)
    assert int(plan.nb[0]) < 32 and int(plan.nb[1]) == 32  # lowered only where it must be
    empty = _plan(hlib, np.zeros(0, dtype=np.int32), 1)
    empty.gesv(0, 0, 0, 0)


def test_batch_autotuner_and_workload(hlib):
    import torch

    from rochpl_b200.batch import autotune, workload_sizes

    table = autotune(hlib, nrhs=1, use_cache=False)
    assert len(table) == 6 and all(v in (8, 16, 32, 64) for v in table)
    n = workload_sizes(512)
    assert n.min() >= 32 and n.max() <= 1024
    plan = _plan(hlib, n, 1, table)
    seeds = 100 + np.arange(plan.count, dtype=np.uint64)
    dA, dB, dP, dI = _pools(plan)
    plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())
    plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    res = torch.zeros(plan.count, dtype=torch.float64, device="cuda")
    plan.residual(seeds, dB.data_ptr(), res.data_ptr())
    assert float(res.max()) < 16.0
    assert plan.last_ms > 0


def test_batch_shards_reproduce_the_whole_batch(hlib):
    """The batched workload split over 3 ranks (each shard solved here in
    turn, no collective involved) gives, system by system, bit for bit the X
    and pivots of the one-plan solve: the per-system seeds and panel widths
    do not depend on the split."""
    import torch

    from rochpl_b200.batch import BatchShard
    from rochpl_b200.ranks import Ranks

    n = np.array([40, 300, 33, 1000, 64, 129, 512, 7, 700, 96], dtype=np.int32)
    table = [16] * 6
    whole = _plan(hlib, n, 4, table)
    dA, dB, dP, dI = _pools(whole)
    seeds = 100 + np.arange(whole.count, dtype=np.uint64)
    whole.matgen(seeds, dA.data_ptr(), dB.data_ptr())
    whole.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    hX, hP = dB.cpu().numpy(), dP.cpu().numpy()
    resid = np.zeros(whole.count)
    local = Ranks("gloo")  # world size 1: assemble is a local scatter
    seen = []
    for rank in range(3):
        sh = BatchShard(hlib, n, 4, rank, 3, table)
        p = sh.plan
        if p.count == 0:
            continue
        sA, sB, sP, sI = _pools(p)
        p.matgen(sh.seeds, sA.data_ptr(), sB.data_ptr())
        p.gesv(sA.data_ptr(), sB.data_ptr(), sP.data_ptr(), sI.data_ptr())
        r = torch.zeros(p.count, dtype=torch.float64, device="cuda")
        p.residual(sh.seeds, sB.data_ptr(), r.data_ptr())
        resid += local.assemble(r.cpu().numpy(), sh.index, sh.total)
        sX, sPv = sB.cpu().numpy(), sP.cpu().numpy()
        for li, gi in enumerate(sh.index):
            m = int(n[gi])
            assert np.array_equal(sX[p.b_off[li]:p.b_off[li] + m * 4],
                                  hX[whole.b_off[gi]:whole.b_off[gi] + m * 4]), gi
            assert np.array_equal(sPv[p.p_off[li]:p.p_off[li] + m],
                                  hP[whole.p_off[gi]:whole.p_off[gi] + m]), gi
            seen.append(int(gi))
        sh.close()
    assert sorted(seen) == list(range(whole.count))
    assert resid.max() < 16.0 and resid.min() > 0.0
