"""The run driver on the CPU (rochpl_b200/driver.py): the sweep order and
counts of src/HPL_pddriver.cpp, the `-it` repetitions and warm-ups of
src/HPL_pdtest.cpp, and the reference's output lines, with a stand-in solver
in place of the GPU.  Expected lines are rebuilt here with explicit padding
(not with the driver's printf-style strings)."""
import io

import pytest

from rochpl_b200.driver import (progress_lines, residual_lines, result_lines, run, summary_lines,
                                sweep, tv_code)
from rochpl_b200.hpl import Algo, HplConfig, parse_hpl_dat

EPS = 2.0 ** -53


class FakeSolver:
    """Returns fixed times and a residual chosen per N; records the calls."""

    def __init__(self, resid_by_n=None, steps=None):
        self.calls, self.warmups = [], []
        self.resid_by_n = resid_by_n or {}
        self.steps = steps

    def warmup(self, algo, n):
        self.warmups.append((algo.nb, n))

    def __call__(self, algo, n, progress=False):
        self.calls.append((n, algo.nb, algo.pfact, algo.rfact, algo.nbmin, algo.ndiv))
        out = {"wtime": 2.0, "t_start": 0.0, "t_end": 2.0, "resid": self.resid_by_n.get(n, 0.5),
               "rnorm_inf": 1e-9, "anorm_inf": 10.0, "anorm_1": 11.0, "xnorm_inf": 3.0,
               "xnorm_1": 30.0, "bnorm_inf": 0.5}
        if progress and self.steps is not None:
            out["steps"] = self.steps
        return out


def test_tv_code_and_result_line():
    a = Algo(nb=256, nbmin=32, ndiv=2, pfact=1, rfact=0, depth=1)
    assert tv_code(a, 0, 1) == "WC10L2C32"
    assert tv_code(Algo(nb=64, nbmin=4, ndiv=3, pfact=2, rfact=2), 5, 0) == "WR15R3R4"
    line = result_lines(a, 0, 1, 4096, 1, 1, 1.5, 0.0, 1.5).splitlines()[0]
    gflops = (2.0 / 3.0 * 4096 ** 3 + 1.5 * 4096 ** 2) / 1.5 / 1e9
    expect = ("WC10L2C32" + "4096".rjust(12) + " " + "256".rjust(5) + " " + "1".rjust(5) + " "
              + "1".rjust(5) + " " + "1.50".rjust(18) + "     " + ("%.3e" % gflops).rjust(18))
    assert line == expect
    assert result_lines(a, 0, 1, 4096, 1, 1, 0.0, 0.0, 0.0) == ""  # no line for a zero time


def test_residual_and_summary_lines():
    r = {"resid": 0.0123456, "rnorm_inf": 1.0, "anorm_inf": 2.0, "anorm_1": 3.0, "xnorm_inf": 4.0,
         "xnorm_1": 5.0, "bnorm_inf": 6.0}
    ok = residual_lines(r, 16.0).splitlines()
    assert ok[0] == "-" * 80
    assert ok[1] == ("||Ax-b||_oo/(eps*(||A||_oo*||x||_oo+||b||_oo)*N)= " + "0.0123456".rjust(16)
                     + " ...... PASSED")
    assert len(ok) == 2
    bad = residual_lines(dict(r, resid=20.0), 16.0).splitlines()
    assert bad[1].endswith(" ...... FAILED") and len(bad) == 8
    assert bad[3] == "||A||_oo . . . . . . . . . . . . . . . . . . . = " + "2.000000".rjust(18)
    s = summary_lines(3, 1, 2, 16.0).splitlines()
    assert s[0] == "=" * 80 and s[1] == ""
    assert s[2] == "Finished " + "6".rjust(6) + " tests with the following results:"
    assert s[3] == " " * 9 + "3".rjust(6) + " tests completed and passed residual checks,"
    assert s[4] == " " * 9 + "1".rjust(6) + " tests completed and failed residual checks,"
    assert s[5] == " " * 9 + "2".rjust(6) + " tests skipped because of illegal input values."
    assert s[-3:] == ["", "End of Tests.", "=" * 80]
    s0 = summary_lines(4, 0, 0, 0.0).splitlines()
    assert s0[3].endswith("tests completed without checking,") and len(s0) == len(s) - 1


def test_sweep_order_matches_the_reference_loops():
    cfg = HplConfig(ns=[100, 200], nbs=[32, 64], ps=[1], qs=[1], pfacts=[0, 2], nbmins=[4, 8],
                    ndivs=[2], rfacts=[1, 2], bcasts=[0, 1])
    got = [(n, bc, a.nb, a.rfact, a.pfact, a.nbmin) for n, _, _, bc, a in sweep(cfg)]
    # N, NB, DEPTH, BCAST, RFACT, PFACT, NBMIN, NDIV -- innermost last.
    expect = [(n, bc, nb, rf, pf, nbm) for n in (100, 200) for nb in (32, 64) for bc in (0, 1)
              for rf in (1, 2) for pf in (0, 2) for nbm in (4, 8)]
    assert got == expect


def test_run_counts_repeats_and_skips():
    cfg = HplConfig(ns=[100, 300], nbs=[32], ps=[1, 2], qs=[1, 1], iters=3, thrsh=16.0)
    solver = FakeSolver(resid_by_n={300: 99.0})
    out = io.StringIO()
    tally = run(cfg, out, solver)
    # Grid 1x1: 2 tests x 3 repetitions, N = 300 fails; grid 2x1: both skipped.
    assert tally == {"passed": 3, "failed": 3, "skipped": 2}
    assert [c[0] for c in solver.calls] == [100] * 3 + [300] * 3
    assert solver.warmups == [(32, 100), (32, 300)]  # one warm-up per test
    text = out.getvalue()
    assert text.count("T/V                N    NB") == 6  # a header before each checked result
    assert text.count("PASSED") == 3 and text.count("FAILED") == 3
    assert "Finished      8 tests with the following results:" in text
    assert text.rstrip().endswith("=" * 80)


def test_run_without_checking_prints_one_header():
    cfg = HplConfig(ns=[64], nbs=[16, 32], ps=[1], qs=[1], iters=2, thrsh=0.0)
    out = io.StringIO()
    tally = run(cfg, out, FakeSolver())
    assert tally == {"passed": 4, "failed": 0, "skipped": 0}
    text = out.getvalue()
    assert text.count("T/V") == 1 and "PASSED" not in text
    assert "tests completed without checking," in text


def test_progress_report():
    n, nb = 1000, 256
    steps = [(0, 40.0), (256, 30.0), (512, 20.0), (768, 10.0)]
    text = progress_lines(steps, n).splitlines()
    assert text[1] == "   %   | Column    | Step Time (s) | Overall GFLOPS"
    rows = text[4:]
    assert len(rows) == 4
    assert rows[1].startswith(" 25.6% | 000000256 | ")
    # Overall rate after the last step: all of the factorisation's flops.
    full = 2.0 / 3.0 * n ** 3 - 0.5 * n ** 2 - n / 6.0
    assert rows[-1].split("|")[-1].strip() == "%.3e" % (full / 0.1 / 1e9)
    # The driver prints it before each result line when asked.
    out = io.StringIO()
    run(HplConfig(ns=[n], nbs=[nb], ps=[1], qs=[1]), out, FakeSolver(steps=steps), progress=True)
    body = out.getvalue()
    assert body.index("Overall GFLOPS") < body.index("WC10R2R32")


def test_hpl_dat_drives_the_sweep():
    dat = "\n".join([
        "HPLinpack benchmark input file", "Innovative Computing Laboratory",
        "HPL.out      output file name (if any)", "6            device out (6=stdout,7=stderr,file)",
        "2            # of problems sizes (N)", "1000 2000     Ns",
        "1            # of NBs", "128          NBs",
        "0            PMAP process mapping (0=Row-,1=Column-major)",
        "2            # of process grids (P x Q)", "1 2          Ps", "1 1          Qs",
        "16.0         threshold", "1            # of panel fact", "2            PFACTs",
        "1            # of recursive stopping criterium", "16           NBMINs",
        "1            # of panels in recursion", "2            NDIVs",
        "1            # of recursive panel fact.", "1            RFACTs",
        "2            # of broadcast", "0 3          BCASTs",
        "1            # of lookahead depth", "1            DEPTHs",
        "1            SWAP (0=bin-exch,1=long,2=mix)", "64           swapping threshold",
        "0            L1 in (0=transposed,1=no-transposed) form",
        "0            U  in (0=transposed,1=no-transposed) form",
        "0            Equilibration (0=no,1=yes)", "8            memory alignment in double (> 0)"])
    cfg = parse_hpl_dat(dat)
    assert cfg.pmap == 0 and cfg.bcasts == [0, 3] and cfg.outfile is None
    out = io.StringIO()
    tally = run(cfg, out, FakeSolver())
    assert tally == {"passed": 4, "failed": 0, "skipped": 4}
    codes = [ln.split()[0] for ln in out.getvalue().splitlines() if ln.startswith("WR")]
    assert codes == ["WR10C2R16", "WR13C2R16"] * 2


def test_grids_run_when_they_match_the_process_count():
    """Under W processes the driver runs the 1 x W grids and skips the rest
    (1 x 1 with W = 1, as before)."""
    cfg = HplConfig(ns=[100], nbs=[32], ps=[1, 1, 2, 1], qs=[1, 2, 1, 4])
    for world, runs in ((1, 1), (2, 1), (4, 1), (3, 0)):
        s = FakeSolver()
        tally = run(cfg, io.StringIO(), solver=s, world=world)
        assert tally == {"passed": runs, "failed": 0, "skipped": 4 - runs}, world
        assert len(s.calls) == runs


def test_two_d_grids_run_with_a_grid_solver():
    """A solver that takes the grid shape (GridSolver) gets P x Q grids with
    P > 1 when P Q is the process count, every panel variant included."""
    class GridFake(FakeSolver):
        takes_grid = True

        def warmup(self, algo, n, grid=None):
            self.warmups.append((algo.nb, n, grid))

        def __call__(self, algo, n, progress=False, grid=None):
            self.calls.append((n, grid, algo.pfact, algo.rfact))
            return super().__call__(algo, n, progress)

    cfg = HplConfig(ns=[100], nbs=[32], ps=[1, 2, 2], qs=[2, 1, 2], pfacts=[2, 0], rfacts=[2])
    s = GridFake()
    tally = run(cfg, io.StringIO(), solver=s, world=2)
    grids = [c[1] for c in s.calls if c[0] == 100 and len(c) == 4]
    assert (1, 2) in grids and (2, 1) in grids and (2, 2) not in grids
    assert sorted(pf for _, g, pf, _ in [c for c in s.calls if len(c) == 4] if g == (2, 1)) == [0, 2]
    assert tally["passed"] == 4 and tally["skipped"] == 2


_GRID_DAT = """HPLinpack benchmark input file
process-grid driver test
HPL.out      output file name (if any)
6            device out (6=stdout,7=stderr,file)
2            # of problems sizes (N)
64 100       Ns
1            # of NBs
16           NBs
{pmap}            PMAP process mapping (0=Row-,1=Column-major)
4            # of process grids (P x Q)
2 4 1 1      Ps
2 1 2 4      Qs
16.0         threshold
1            # of panel fact
2            PFACTs (0=left, 1=Crout, 2=Right)
1            # of recursive stopping criterium
4            NBMINs (>= 1)
1            # of panels in recursion
2            NDIVs
1            # of recursive panel fact.
2            RFACTs (0=left, 1=Crout, 2=Right)
1            # of broadcast
0            BCASTs (0=1rg,1=1rM,2=2rg,3=2rM,4=Lng,5=LnM)
1            # of lookahead depth
1            DEPTHs (>=0)
1            SWAP (0=bin-exch,1=long,2=mix)
64           swapping threshold
0            L1 in (0=transposed,1=no-transposed) form
0            U  in (0=transposed,1=no-transposed) form
0            Equilibration (0=no,1=yes)
8            memory alignment in double (> 0)
"""

_GRID_CHILD = r"""
import ctypes, io, json, os, sys
import numpy as np
import torch
import torch.distributed as dist
sys.path.insert(0, os.path.join(os.getcwd(), "tests"))
from oracle import oracle as O
from grid_host import HostBackend
from grid2d_host import HostBackend2D
from rochpl_b200.driver import GridSolver, run
from rochpl_b200.hpl import parse_hpl_dat


class HostResidual:  # the library's hplb_residual_lcg, on host memory
    def residual_lcg(self, n, seed, xptr):
        x = np.ctypeslib.as_array((ctypes.c_double * n).from_address(xptr)).copy()
        return O.residual(O.matgen(n, n + 1, seed), n, x)


dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
cfg = parse_hpl_dat(open(os.environ["DAT"]).read())
solver = GridSolver(0, pmap=cfg.pmap, lib=HostResidual(), backend=HostBackend(O),
                    backend2d=HostBackend2D(O), dev=torch.device("cpu"))
out = io.StringIO()
tally = run(cfg, out, solver=solver, world=dist.get_world_size())
print("RESULT " + json.dumps({"rank": rank, "tally": tally, "out": out.getvalue()}))
dist.destroy_process_group()
"""


@pytest.mark.parametrize("pmap", [0, 1])
def test_grid_solver_runs_an_hpl_dat_on_four_gloo_processes(tmp_path, pmap):
    """GridSolver's orchestration on CPU: four gloo processes run an HPL.dat
    with grids 2 x 2, 4 x 1, 1 x 2 and 1 x 4 through the driver, host backends
    standing in for the GPU.  The 1 x 4 grid takes the 1 x Q solve, 2 x 2 and
    4 x 1 the P x Q solve in PMAP order, 1 x 2 is skipped (not four
    processes); every solve passes the residual check on process 0."""
    import json
    import os
    import socket
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = tmp_path / "HPL.dat"
    path.write_text(_GRID_DAT.format(pmap=pmap))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = []
    for rank in range(4):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="4", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), DAT=str(path),
                   PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
        procs.append(subprocess.Popen([sys.executable, "-c", _GRID_CHILD], env=env, cwd=root,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=300)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, se[-3000:]
        res.append(json.loads([ln for ln in so.splitlines() if ln.startswith("RESULT ")][-1][7:]))
    res.sort(key=lambda r: r["rank"])
    assert all(r["tally"] == {"passed": 6, "failed": 0, "skipped": 2} for r in res)
    lines = res[0]["out"].splitlines()
    tv = "WC" if pmap == 1 else "WR"
    results = [ln.split() for ln in lines if ln.startswith(tv)]
    assert sorted((int(f[1]), int(f[3]), int(f[4])) for f in results) == sorted(
        (n, p, q) for n in (64, 100) for p, q in ((2, 2), (4, 1), (1, 4)))
    assert sum("PASSED" in ln for ln in lines) == 6
