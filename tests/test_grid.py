"""The 1 x Q process-grid solve (rochpl_b200.grid) on CPU: the block-cyclic
bookkeeping against a brute-force layout, and the whole distributed loop --
panel ownership, broadcast, look-ahead order, distributed back-solve -- with
the oracle's building blocks as each process's local work, against the
single-process oracle solve: the same pivots, the same factored columns bit
for bit, x within 64 n eps kappa.  Run as threads (Q = 1, 2, 3) and as a
world-size-2 gloo group of two processes on 127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from rochpl_b200.grid import Grid1xQ, numroc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EPS = 2.0 ** -53


@pytest.mark.parametrize("n,nb,Q", [(1, 1, 1), (10, 3, 2), (100, 16, 3), (128, 32, 4),
                                    (1000, 128, 3), (1001, 128, 8), (257, 64, 5)])
def test_grid_bookkeeping_matches_brute_force(n, nb, Q):
    ncols = n + 1
    owner = [(c // nb) % Q for c in range(ncols)]
    for q in range(Q):
        g = Grid1xQ(n, nb, q, Q)
        mine = [c for c in range(ncols) if owner[c] == q]
        assert g.nq == len(mine) == numroc(ncols, nb, q, Q)
        for lc, c in enumerate(mine):
            assert g.owner(c) == q and g.local(c) == lc
        # blocks: contiguous runs of mine, in order
        flat = [g0 + i for lc, g0, w in g.local_blocks() for i in range(w)]
        assert flat == mine
        for gcol in range(ncols + 1):
            first = next((lc for lc, c in enumerate(mine) if c >= gcol), len(mine))
            lf = g.local_from(gcol)
            assert min(lf, len(mine)) == first, (q, gcol)
    for p in range((n + nb - 1) // nb):
        j, jb, o, lc = Grid1xQ(n, nb, 0, Q).panel(p)
        assert j == p * nb and jb == min(nb, n - j) and o == owner[j]
        assert lc == Grid1xQ(n, nb, o, Q).local(j)


def _run_rank(oracle, comm, n, nb, Q, q, seed, algo):
    import torch

    from grid_host import HostBackend, local_to_global
    from rochpl_b200.grid import matgen_local, pdgesv_grid

    be = HostBackend(oracle)
    g = Grid1xQ(n, nb, q, Q)
    ld = oracle.default_ld(n)
    A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64)
    matgen_local(be, g, seed, A, ld)
    x, ipiv, info = pdgesv_grid(be, comm, g, algo, A, ld)
    return x.numpy().copy(), ipiv.numpy().copy(), info, local_to_global(g, A, ld)


def _reference(oracle, n, nb, seed, algo):
    ld = oracle.default_ld(n)
    A = oracle.matgen(n, n + 1, seed, ld=ld)
    A0 = A.copy(order="F")
    x, ipiv, info = oracle.pdgesv(A, n, nb, algo.nbmin, algo.ndiv, algo.pfact, algo.rfact)
    return x, ipiv, info, A[:n], A0


def _check(oracle, n, nb, seed, algo, results):
    xo, po, info_o, Ao, A0 = _reference(oracle, n, nb, seed, algo)
    assert info_o == 0
    cover = np.zeros((n, n + 1), dtype=bool)
    for x, ipiv, info, F in results:
        assert info == 0
        assert np.array_equal(ipiv, po)  # the same pivots on every rank
        kappa = np.linalg.cond(A0[:n, :n], np.inf)
        err = np.max(np.abs(x - xo)) / np.max(np.abs(xo))
        assert err <= 64 * n * EPS * kappa, (err, kappa)
        held = ~np.isnan(F)
        # This rank's factored columns equal the single-process factors bit for bit.
        assert np.array_equal(F[held].view(np.uint64), Ao[held].view(np.uint64))
        cover |= held
    assert cover.all()  # the ranks hold every column between them


@pytest.mark.parametrize("n,nb,Q", [(200, 32, 1), (200, 32, 2), (301, 48, 3), (256, 64, 2),
                                    (97, 16, 4), (64, 64, 2)])
@pytest.mark.parametrize("pfact,rfact", [(2, 2), (0, 1)])
def test_grid_solve_threads_match_the_oracle(oracle, n, nb, Q, pfact, rfact):
    import threading

    from rochpl_b200.grid import LocalGroup
    from rochpl_b200.hpl import Algo

    algo = Algo(nb, 8, 2, pfact, rfact, 1, 0)
    grp = LocalGroup(Q)
    out, errs = [None] * Q, []

    def work(q):
        try:
            out[q] = _run_rank(oracle, grp.member(q), n, nb, Q, q, 100, algo)
        except BaseException as e:  # surfaced below
            errs.append(e)
            grp.barrier.abort()

    ts = [threading.Thread(target=work, args=(q,)) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=120)
    assert not errs, errs
    _check(oracle, n, nb, 100, algo, out)


_CHILD = r"""
import json, os, sys
import numpy as np
import torch.distributed as dist
sys.path.insert(0, os.path.join(os.getcwd(), "tests"))
from oracle import oracle as O
from rochpl_b200.grid import DistGroup
from rochpl_b200.hpl import Algo
from test_grid import _run_rank
n, nb = int(os.environ["GN"]), int(os.environ["GNB"])
dist.init_process_group("gloo", init_method="env://")
q, Q = dist.get_rank(), dist.get_world_size()
x, ipiv, info, F = _run_rank(O, DistGroup(), n, nb, Q, q, 100, Algo(nb, 16, 2, 2, 2, 1, 0))
np.save(os.environ["GOUT"] + f"/rank{q}.npy", F)
print("RESULT " + json.dumps({"rank": q, "x": x.tolist(), "ipiv": ipiv.tolist(), "info": info}))
dist.destroy_process_group()
"""


def test_grid_solve_two_gloo_processes(oracle, tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    n, nb = 300, 32
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), GN=str(n), GNB=str(nb),
                   GOUT=str(tmp_path),
                   PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
        procs.append(subprocess.Popen([sys.executable, "-c", _CHILD], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, se[-3000:]
        line = [ln for ln in so.splitlines() if ln.startswith("RESULT ")][-1]
        res.append(json.loads(line[7:]))
    res.sort(key=lambda r: r["rank"])
    from rochpl_b200.hpl import Algo

    results = [(np.array(r["x"]), np.array(r["ipiv"], dtype=np.int32), r["info"],
                np.load(tmp_path / f"rank{r['rank']}.npy")) for r in res]
    _check(oracle, n, nb, 100, Algo(nb, 16, 2, 2, 2, 1, 0), results)


def test_grid_rejects_a_local_array_that_is_too_small(oracle):
    import torch

    from grid_host import HostBackend
    from rochpl_b200.grid import LocalGroup, pdgesv_grid
    from rochpl_b200.hpl import Algo

    g = Grid1xQ(64, 16, 0, 1)
    comm = LocalGroup(1).member(0)
    be, algo = HostBackend(oracle), Algo(16, 4, 2, 2, 2, 1, 0)
    with pytest.raises(ValueError, match="ld >= 64"):
        pdgesv_grid(be, comm, g, algo, torch.zeros(63 * 65, dtype=torch.float64), 63)
    with pytest.raises(ValueError, match="entries"):
        pdgesv_grid(be, comm, g, algo, torch.zeros(64 * 65 - 1, dtype=torch.float64), 64)
    with pytest.raises(ValueError, match="float64"):
        pdgesv_grid(be, comm, g, algo, torch.zeros(64 * 65, dtype=torch.float32), 64)


@pytest.mark.parametrize("kw,msg", [({"nb": 0}, "at least 1"), ({"nbmin": 0}, "at least 1"),
                                    ({"ndiv": 1}, "NDIV at least 2"), ({"pfact": 3}, "PFACT 3"),
                                    ({"rfact": -1}, "RFACT -1"), ({"depth": 0}, "depth 1"),
                                    ({"nbmin": 129}, "above the limits"),
                                    ({"nb": 2049}, "above the limits")])
def test_grid_algo_checks(kw, msg):
    from dataclasses import replace

    from rochpl_b200.grid import check_algo
    from rochpl_b200.hpl import Algo

    check_algo(Algo(512))
    with pytest.raises(ValueError, match=msg):
        check_algo(replace(Algo(512), **kw))


@pytest.mark.parametrize("fault", ["small_array", "other_nb", "bad_algo_on_one"])
def test_grid_bad_call_on_one_process_stops_every_process(oracle, fault):
    """A bad call on one process (its local array too small, a different NB,
    an invalid solve parameter) makes every process raise at the start of
    the solve; none is left waiting in an exchange."""
    import threading
    from dataclasses import replace

    import torch

    from grid_host import HostBackend
    from rochpl_b200.grid import LocalGroup, pdgesv_grid
    from rochpl_b200.hpl import Algo

    n, Q = 64, 2
    grp = LocalGroup(Q)
    errs = [None] * Q

    def work(q):
        nb = 8 if (fault == "other_nb" and q == 1) else 16
        algo = Algo(16, 4, 2, 2, 2, 1, 0)
        if fault == "bad_algo_on_one" and q == 1:
            algo = replace(algo, ndiv=1)
        g = Grid1xQ(n, nb, q, Q)
        ld = oracle.default_ld(n)
        size = ld * max(g.nq, 1) - (1 if (fault == "small_array" and q == 1) else 0)
        try:
            pdgesv_grid(HostBackend(oracle), grp.member(q), g, algo,
                        torch.zeros(size, dtype=torch.float64), ld)
        except ValueError as e:
            errs[q] = str(e)
        except BaseException as e:  # anything else is a failure of the test
            errs[q] = e
            grp.barrier.abort()

    ts = [threading.Thread(target=work, args=(q,)) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert not any(t.is_alive() for t in ts), "a process was left waiting"
    assert all(isinstance(e, str) for e in errs), errs


_BAD_CHILD = r"""
import os, sys
import torch
import torch.distributed as dist
sys.path.insert(0, os.path.join(os.getcwd(), "tests"))
from oracle import oracle as O
from grid_host import HostBackend
from rochpl_b200.grid import DistGroup, Grid1xQ, pdgesv_grid
from rochpl_b200.hpl import Algo
dist.init_process_group("gloo", init_method="env://")
rank, Q = dist.get_rank(), dist.get_world_size()
nb = 8 if rank == 1 else 16  # rank 1 was given another NB
g = Grid1xQ(64, nb, rank, Q)
ld = O.default_ld(64)
A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64)
try:
    pdgesv_grid(HostBackend(O), DistGroup(), g, Algo(16, 4, 2, 2, 2, 1, 0), A, ld)
    print("SOLVED")
except ValueError as e:
    print("REJECTED " + str(e))
dist.destroy_process_group()
"""


def test_grid_bad_call_stops_two_gloo_processes(tmp_path):
    """Two gloo processes, one given another NB: both reject the call at the
    start of the solve and exit, long before any process-group timeout."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
        procs.append(subprocess.Popen([sys.executable, "-c", _BAD_CHILD], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, se[-3000:]
        outs.append(so)
    assert all("REJECTED" in so and "SOLVED" not in so for so in outs), outs
