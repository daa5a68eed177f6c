"""End-to-end parity of hplb_pdgesv against the oracle: identical pivot
vectors, x within tolerance, HPL scaled residual below 16, plus the error and
bounded-wait paths."""
import numpy as np
import pytest

from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

# x tolerance: ||x - x_oracle||oo / ||x_oracle||oo <= 64 * n * eps * kappa_est, with
# kappa_est = ||A||oo * ||A^-1||oo estimated from the oracle solve; HPL LCG matrices
# at these sizes have kappa ~ 1e3..1e5.
EPS = 2.0 ** -53


def solve_both(hlib, oracle, n, nb, nbmin=32, ndiv=2, pfact=2, rfact=2, seed=100):
    import torch

    from rochpl_b200.hpl import Algo

    ld = oracle.default_ld(n)
    A0 = oracle.matgen(n, n + 1, seed, ld=ld)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + 1, seed, dA.data_ptr(), ld, nb)
    dX = torch.zeros(max(n, 1), dtype=torch.float64, device="cuda")
    dP = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    info = hlib.pdgesv(Algo(nb, nbmin, ndiv, pfact, rfact, 1, 0).c(), n, dA.data_ptr(), ld,
                       dX.data_ptr(), dP.data_ptr())
    Ao = A0.copy(order="F")
    xo, po, info_o = oracle.pdgesv(Ao, n, nb, nbmin, ndiv, pfact, rfact)
    return dict(x=dX.cpu().numpy()[:n], ipiv=dP.cpu().numpy()[:n], info=info, A0=A0, dA=dA,
                dX=dX, ld=ld, xo=xo, po=po, info_o=info_o, Ao=Ao)


CASES = [(1, 1, 1), (2, 1, 1), (31, 8, 4), (100, 32, 8), (257, 64, 16), (257, 256, 32),
         (1000, 256, 32), (1000, 128, 16), (1031, 96, 32), (2048, 512, 32), (4096, 256, 32)]


@pytest.mark.parametrize("n,nb,nbmin", CASES)
def test_solve_parity(hlib, oracle, n, nb, nbmin):
    r = solve_both(hlib, oracle, n, nb, nbmin)
    assert r["info"] == 0 and r["info_o"] == 0
    div = np.nonzero(r["ipiv"] != r["po"])[0]
    assert div.size == 0, f"pivot divergence at columns {div[:10]}"
    xo = r["xo"]
    kappa = np.linalg.cond(r["A0"][:n, :n], np.inf) if n <= 2048 else 1e5
    tol = 64 * n * EPS * kappa
    err = np.max(np.abs(r["x"] - xo)) / np.max(np.abs(xo))
    assert err <= tol, (err, tol)
    res = oracle.residual(r["A0"], n, r["x"])
    assert res["resid"] < 16.0


def test_leaf_kinds_give_identical_results(hlib, oracle):
    """The places the leaf can keep its slice (hplb_set_option HPLB_OPT_LEAF:
    one cluster's registers, registers across the GPU, shared memory, global
    memory) perform the same operations in the same order: the same pivots as
    the oracle and bit-identical x."""
    import torch

    from rochpl_b200.lib import LEAF_AUTO, LEAF_GLOBAL, LEAF_REGISTERS, LEAF_SHARED, HplError

    xs = []
    try:
        for kind in (LEAF_AUTO, LEAF_REGISTERS, LEAF_SHARED, LEAF_GLOBAL):
            hlib.set_leaf(kind)
            r = solve_both(hlib, oracle, 2048, 256, 32)
            assert np.array_equal(r["ipiv"], r["po"]), kind
            xs.append(r["x"])
    finally:
        hlib.set_leaf(LEAF_AUTO)
    assert all(np.array_equal(x.view(np.uint64), xs[0].view(np.uint64)) for x in xs)
    with pytest.raises(HplError):
        hlib.set_leaf(4)


@pytest.mark.parametrize("n,nb,nrhs,ld", [(1, 1, 3, None), (100, 32, 2, None), (100, 8, 70, None),
                                          (500, 64, 5, 501),
                                          (1031, 96, 33, None), (2048, 256, 1, None),
                                          (2048, 256, 32, None), (4096, 512, 70, None)])
def test_gesv_multi_rhs(hlib, oracle, n, nb, nrhs, ld):
    """hplb_gesv: B in columns n .. n + nrhs - 1 of [A | B] rides through the
    factorisation.  The factors and pivots are bit-identical to hplb_pdgesv's
    on the same A (the extra columns never feed back into A), every column of
    X is within 64 n eps kappa_oo of LAPACK's solve, and with one right-hand
    side x is hplb_pdgesv's x bit for bit (the same back-solve kernel).  An
    odd ld takes the back-solve's 8-byte staging path."""
    import torch

    from rochpl_b200.hpl import Algo

    ld = ld or oracle.default_ld(n)
    algo = Algo(nb, min(32, nb), 2, 2, 2, 1, 0).c()
    dAB = torch.empty(ld * (n + nrhs), dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + nrhs, 7, dAB.data_ptr(), ld, nb)
    AB = dAB.view(n + nrhs, ld).cpu().numpy()
    A0, B0 = AB[:n, :n].T.copy(), AB[n:, :n].T.copy()
    dX = torch.full((nrhs, n), float("nan"), dtype=torch.float64, device="cuda")
    dP = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert hlib.gesv(algo, n, nrhs, dAB.data_ptr(), ld, dX.data_ptr(), n, dP.data_ptr()) == 0

    dA1 = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + 1, 7, dA1.data_ptr(), ld, nb)
    dx1 = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP1 = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert hlib.pdgesv(algo, n, dA1.data_ptr(), ld, dx1.data_ptr(), dP1.data_ptr()) == 0
    assert np.array_equal(dP.cpu().numpy(), dP1.cpu().numpy())
    f_multi = dAB[: ld * n].view(n, ld)[:, :n].cpu().numpy().view(np.uint64)
    f_one = dA1[: ld * n].view(n, ld)[:, :n].cpu().numpy().view(np.uint64)
    assert np.array_equal(f_multi, f_one)

    X = dX.cpu().numpy().T
    Xr = np.linalg.solve(A0, B0)
    kappa = np.linalg.cond(A0, np.inf)
    tol = 64 * n * EPS * kappa
    err = np.max(np.abs(X - Xr), axis=0) / np.max(np.abs(Xr), axis=0)
    assert np.all(err <= tol), (err.max(), tol)
    if nrhs == 1:
        assert np.array_equal(X[:, 0].view(np.uint64), dx1.cpu().numpy().view(np.uint64))


def test_panel_sms_cap_gives_identical_results(hlib, oracle):
    """hplb_set_option(HPLB_OPT_PANEL_SMS) only changes how the trailing
    update's tiles are spread over CTAs, never a tile's arithmetic: capped and
    uncapped solves give the oracle's pivots and bit-identical x; values
    outside [-1, SMs) are rejected."""
    from rochpl_b200.lib import PANEL_SMS_AUTO, HplError

    xs = []
    try:
        for keep in (PANEL_SMS_AUTO, 0, 16, 100):
            hlib.set_panel_sms(keep)
            r = solve_both(hlib, oracle, 4096, 256, 32)
            assert np.array_equal(r["ipiv"], r["po"]), keep
            xs.append(r["x"])
    finally:
        hlib.set_panel_sms(PANEL_SMS_AUTO)
    assert all(np.array_equal(x.view(np.uint64), xs[0].view(np.uint64)) for x in xs)
    for bad in (-2, 100000):
        with pytest.raises(HplError):
            hlib.set_panel_sms(bad)


def test_solve_parity_n16384_against_the_oracle(hlib, oracle):
    """The parity solve at N = 16384, NB = 512 (the size the bench's CPU leg
    factors): identical pivot vectors, x within 64 N eps kappa_oo of the
    oracle's x, residual < 16.  The oracle's level 3 runs in the host OpenBLAS
    here (the scalar restatement would take half an hour at this size)."""
    import torch

    n, nb = 16384, 512
    if not oracle.use_blas(0):
        pytest.skip("no host OpenBLAS for the oracle")
    try:
        x_o, p_o, info_o, resid_o = oracle.hpl_test(n, nb, 32, 2)
    finally:
        oracle.no_blas()
    from rochpl_b200.hpl import Algo

    ld = oracle.default_ld(n)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + 1, 100, dA.data_ptr(), ld, nb)
    A = dA.view(n + 1, ld)[:n, :n].t()
    kappa = float(A.abs().sum(dim=1).max()) * float(torch.linalg.inv(A).abs().sum(dim=1).max())
    del A
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = hlib.pdgesv(Algo(nb, 32, 2, 2, 2, 1, 0).c(), n, dA.data_ptr(), ld, dX.data_ptr(),
                       dP.data_ptr())
    assert info == 0 and info_o == 0
    div = np.nonzero(dP.cpu().numpy() != p_o)[0]
    assert div.size == 0, f"pivot divergence at columns {div[:10]}"
    x = dX.cpu().numpy()
    err = np.max(np.abs(x - x_o)) / np.max(np.abs(x_o))
    tol = 64 * n * EPS * kappa
    assert err <= tol, (err, tol)
    assert hlib.residual_lcg(n, 100, dX.data_ptr())["resid"] < 16.0 and resid_o < 16.0


@pytest.mark.parametrize("pfact,rfact", [(0, 0), (1, 1), (2, 0), (0, 2), (1, 2), (2, 1)])
def test_solve_variants(hlib, oracle, pfact, rfact):
    r = solve_both(hlib, oracle, 600, 128, 16, 2, pfact, rfact)
    assert np.array_equal(r["ipiv"], r["po"])
    assert oracle.residual(r["A0"], 600, r["x"])["resid"] < 16.0


@pytest.mark.parametrize("ndiv", [2, 3, 4])
def test_solve_ndiv(hlib, oracle, ndiv):
    r = solve_both(hlib, oracle, 700, 192, 16, ndiv)
    assert np.array_equal(r["ipiv"], r["po"])
    assert oracle.residual(r["A0"], 700, r["x"])["resid"] < 16.0


@pytest.mark.parametrize("n", [1000, 4096])
def test_device_residual_matches_oracle(hlib, oracle, n):
    """hplb_residual (stored matrix) and hplb_residual_lcg (regenerated in the
    kernel) against the oracle's long-double residual of the same x."""
    import torch

    r = solve_both(hlib, oracle, n, 256, 32)
    ld = r["ld"]
    hlib.matgen(n, n + 1, 100, r["dA"].data_ptr(), ld)
    d1 = hlib.residual(n, r["dA"].data_ptr(), ld, r["dX"].data_ptr())
    d2 = hlib.residual_lcg(n, 100, r["dX"].data_ptr())
    o = oracle.residual(r["A0"], n, r["x"])
    for d in (d1, d2):
        for k in ("anorm_1", "anorm_inf", "xnorm_1", "xnorm_inf", "bnorm_inf"):
            assert d[k] == pytest.approx(o[k], rel=1e-12), k
        # ||r|| is itself a rounding-level quantity: agree to within the
        # rounding of the sum (n * eps * ||A||oo ||x||oo).
        assert abs(d["rnorm_inf"] - o["rnorm_inf"]) <= n * EPS * o["anorm_inf"] * o["xnorm_inf"]
        assert d["resid"] < 16.0
    for k in d1:
        assert d1[k] == d2[k], k  # the two sources are bit-identical


def test_factors_match_oracle(hlib, oracle):
    """The factored matrix (U, panel multipliers, y) against the oracle's."""
    n = 512
    r = solve_both(hlib, oracle, n, 128, 32)
    got = from_dev(r["dA"], r["ld"], n + 1)[:n]
    ref = r["Ao"][:n]
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) / scale < 1e-9


def test_zero_pivot_reports_singular(hlib, oracle):
    import torch

    from rochpl_b200.hpl import Algo

    n = 300
    ld = oracle.default_ld(n)
    A = oracle.matgen(n, n + 1, 100, ld=ld)
    A[:, 77] = 0.0
    dA = to_dev(A)
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    info = hlib.pdgesv(Algo(64, 16, 2, 2, 2, 1, 0).c(), n, dA.data_ptr(), ld, dX.data_ptr())
    assert info == 78


def test_bad_arguments(hlib):
    from rochpl_b200.hpl import Algo
    from rochpl_b200.lib import HPLB_ERR_ARG, HPLB_ERR_UNSUPPORTED, HplError

    with pytest.raises(HplError) as e:
        hlib.pdgesv(Algo(0, 32, 2, 2, 2, 1, 0).c(), 10, 1, 10, 1)
    assert e.value.status == HPLB_ERR_ARG
    with pytest.raises(HplError) as e:
        hlib.pdgesv(Algo(64, 32, 2, 2, 2, 0, 0).c(), 10, 1, 10, 1)
    assert e.value.status == HPLB_ERR_UNSUPPORTED
    with pytest.raises(HplError) as e:
        hlib.pdgesv(Algo(64, 32, 1, 2, 2, 1, 0).c(), 10, 1, 10, 1)
    assert e.value.status == HPLB_ERR_ARG
    with pytest.raises(HplError) as e:
        hlib.pdgesv(Algo(64, 32, 2, 2, 2, 1, 0).c(), 100, 1, 50, 1)  # ld < n
    assert e.value.status == HPLB_ERR_ARG


def test_bounded_wait_times_out_and_context_survives(hlib, oracle):
    from rochpl_b200.lib import HPLB_ERR_TIMEOUT

    assert hlib.selftest_wait_timeout(200_000_000) == HPLB_ERR_TIMEOUT  # 0.2 s
    r = solve_both(hlib, oracle, 200, 64, 16)  # the context still works
    assert np.array_equal(r["ipiv"], r["po"])


def test_repeat_solves_are_bitwise_reproducible(hlib, oracle):
    a = solve_both(hlib, oracle, 1500, 256, 32)
    b = solve_both(hlib, oracle, 1500, 256, 32)
    assert np.array_equal(a["x"].view(np.uint64), b["x"].view(np.uint64))


@pytest.mark.parametrize("n,nb", [(1000, 128), (777, 100), (64, 128)])
def test_step_times(hlib, n, nb):
    """hplb_last_steps: one entry per NB-wide step, at columns 0, NB, 2 NB...,
    positive times that add up to the factorisation's (the last step ends
    where the LU ends)."""
    import torch

    from rochpl_b200.hpl import Algo, default_ld

    ld = default_ld(n)
    A = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    X = torch.zeros(n, dtype=torch.float64, device="cuda")
    hlib.matgen(n, n + 1, 100, A.data_ptr(), ld, nb)
    hlib.pdgesv(Algo(nb, 16, 2, 2, 2, 1, 0).c(), n, A.data_ptr(), ld, X.data_ptr())
    steps = hlib.last_steps()
    assert [c for c, _ in steps] == list(range(0, n, nb))
    assert all(ms > 0 for _, ms in steps)
    lu = hlib.last_timing()["lu_ms"]
    assert abs(sum(ms for _, ms in steps) - lu) <= 0.02 * lu + 0.05
    hlib.pdgesv(Algo(nb, 16, 2, 2, 2, 1, 0).c(), 0, A.data_ptr(), ld, X.data_ptr())
    assert hlib.last_steps() == []  # a call with N = 0 keeps no earlier steps


def test_driver_on_the_gpu(hlib):
    """The run driver end to end on the device: two sizes, two repetitions
    each, with the progress report; every residual passes."""
    import io

    from rochpl_b200.driver import GpuSolver, run
    from rochpl_b200.hpl import HplConfig

    out = io.StringIO()
    cfg = HplConfig(ns=[300, 1000], nbs=[64], ps=[1], qs=[1], iters=2, nbmins=[16])
    tally = run(cfg, out, GpuSolver(0), progress=True)
    assert tally == {"passed": 4, "failed": 0, "skipped": 0}
    text = out.getvalue()
    assert text.count(" ...... PASSED") == 4 and text.count("Overall GFLOPS") == 4
    assert ("WC10R2R16" + "1000".rjust(12) + " " + "64".rjust(5) + " " + "1".rjust(5) + " "
            + "1".rjust(5)) in text


def test_native_driver_on_the_gpu(hlib, tmp_path):
    """rochpl_b200/hplb (the C++ driver over the C ABI): a command-line run
    with two repetitions and the progress report, and an HPL.dat run with a
    skipped 2 x 1 grid, written to the file HPL.dat names."""
    import os
    import subprocess

    from rochpl_b200.build import build

    build()
    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rochpl_b200",
                       "hplb")
    r = subprocess.run([cli, "-N", "1000", "-NB", "128", "-it", "2", "--progress"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.count(" ...... PASSED") == 2 and r.stdout.count("Overall GFLOPS") == 2
    assert "Finished      2 tests with the following results:" in r.stdout
    dat = "\n".join([
        "HPLinpack benchmark input file", "test", "out.txt      output file name (if any)",
        "8            device out (6=stdout,7=stderr,file)", "1            # of problems sizes (N)",
        "777          Ns", "1            # of NBs", "64           NBs",
        "0            PMAP process mapping (0=Row-,1=Column-major)",
        "2            # of process grids (P x Q)", "1 2          Ps", "1 1          Qs",
        "16.0         threshold", "2            # of panel fact", "0 1          PFACTs",
        "1            # of recursive stopping criterium", "8            NBMINs",
        "1            # of panels in recursion", "2            NDIVs",
        "1            # of recursive panel fact.", "2            RFACTs",
        "1            # of broadcast", "1            BCASTs",
        "1            # of lookahead depth", "1            DEPTHs",
        "1            SWAP (0=bin-exch,1=long,2=mix)", "64           swapping threshold",
        "0            L1 in (0=transposed,1=no-transposed) form",
        "0            U  in (0=transposed,1=no-transposed) form",
        "0            Equilibration (0=no,1=yes)", "8            memory alignment in double (> 0)"])
    (tmp_path / "HPL.dat").write_text(dat + "\n")
    r = subprocess.run([cli, "-i", "HPL.dat"], capture_output=True, text=True, timeout=300,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    text = (tmp_path / "out.txt").read_text()
    assert text.count(" ...... PASSED") == 2
    assert "WR11R2L8" in text and "WR11R2C8" in text
    assert "              2 tests skipped because of illegal input values." in text
