"""The P x Q process-grid solve (rochpl_b200.grid2d) on CPU: the 2-D
block-cyclic bookkeeping against a brute-force layout, and the whole
distributed loop -- the panel's pivot search across the process column with
the replicated top block, the panel broadcast along process rows, the
interchanges gathered over the process column, the trailing update and the
distributed back-solve -- with a host backend as each process's local work,
against the single-process oracle solve of the same system: the same pivots,
the factored matrix and x within 64 n eps kappa.  Run as threads for several
grid shapes and as a 2 x 2 group of four gloo processes on 127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from rochpl_b200.grid import numroc
from rochpl_b200.grid2d import Grid2D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EPS = 2.0 ** -53


@pytest.mark.parametrize("n,nb,P,Q", [(1, 1, 1, 1), (10, 3, 2, 2), (100, 16, 3, 2),
                                      (257, 64, 2, 3), (1000, 128, 4, 2), (33, 8, 5, 1)])
def test_grid2d_bookkeeping_matches_brute_force(n, nb, P, Q):
    rown = [(r // nb) % P for r in range(n)]
    coln = [(c // nb) % Q for c in range(n + 1)]
    for p in range(P):
        for q in range(Q):
            g = Grid2D(n, nb, p, q, P, Q)
            rows = [r for r in range(n) if rown[r] == p]
            cols = [c for c in range(n + 1) if coln[c] == q]
            assert g.mp == len(rows) == numroc(n, nb, p, P)
            assert g.nq == len(cols)
            for lr, r in enumerate(rows):
                assert g.row_owner(r) == p and g.lrow(r) == lr and g.grow(lr) == r
            for lc, c in enumerate(cols):
                assert g.col_owner(c) == q and g.lcol(c) == lc
            assert [g0 + i for _, g0, h in g.row_blocks() for i in range(h)] == rows
            assert [g0 + i for _, g0, w in g.col_blocks() for i in range(w)] == cols
            for gr in range(n + 2):
                assert g.lrow_from(gr) == next((i for i, r in enumerate(rows) if r >= gr),
                                               len(rows))
            for gc in range(n + 2):
                assert g.lcol_from(gc) == next((i for i, c in enumerate(cols) if c >= gc),
                                               len(cols))


@pytest.mark.parametrize("P,Q", [(1, 1), (2, 3), (3, 2), (4, 1), (1, 4)])
@pytest.mark.parametrize("pmap", [0, 1])
def test_grid2d_process_order(P, Q, pmap):
    """PMAP's two orders (HPL_grid_init): every rank has one (p, q) and back."""
    seen = set()
    for rank in range(P * Q):
        p, q = Grid2D.coords(rank, P, Q, pmap)
        assert 0 <= p < P and 0 <= q < Q
        assert Grid2D(10, 2, p, q, P, Q, pmap).rank_of(p, q) == rank
        assert rank == (p * Q + q if pmap == 0 else q * P + p)
        seen.add((p, q))
    assert len(seen) == P * Q


def _run_rank(oracle, comms, n, nb, P, Q, p, q, seed, algo, pmap=0):
    import torch

    from grid2d_host import HostBackend2D, local_to_global_2d
    from rochpl_b200.grid2d import matgen_local_2d, pdgesv_2d

    be = HostBackend2D(oracle)
    g = Grid2D(n, nb, p, q, P, Q, pmap)
    ld = max(g.mp, 1) + 3  # any ld >= mp
    A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64)
    matgen_local_2d(be, g, seed, A, ld)
    x, ipiv, info = pdgesv_2d(be, comms, g, algo, A, ld)
    return x.numpy().copy(), ipiv.numpy().copy(), info, local_to_global_2d(g, A, ld)


def _check(oracle, n, nb, seed, algo, results):
    A0 = oracle.matgen(n, n + 1, seed, ld=n)
    Ao = A0.copy(order="F")
    xo, po, info_o = oracle.pdgesv(Ao, n, nb, algo.nbmin, algo.ndiv, algo.pfact, algo.rfact)
    kappa = np.linalg.cond(A0[:n, :n], np.inf)
    tol = 64 * n * EPS * kappa
    F = np.full((n, n + 1), np.nan)
    for x, ipiv, info, part in results:
        assert info == info_o == 0
        assert np.array_equal(ipiv, po[:n]), np.nonzero(ipiv != po[:n])[0][:8]
        err = np.max(np.abs(x - xo)) / np.max(np.abs(xo))
        assert err <= tol, (err, tol)
        have = ~np.isnan(part)
        F[have] = part[have]
    assert not np.isnan(F).any()  # every block held by exactly one process
    Fo = np.asarray(Ao)[:n, :n + 1]
    scale = np.max(np.abs(Fo))
    assert np.max(np.abs(F[:, :n] - Fo[:, :n])) <= tol * scale * 16
    res = oracle.residual(A0, n, results[0][0])
    assert res["resid"] < 16.0


@pytest.mark.parametrize("n,nb,P,Q", [(64, 16, 1, 1), (64, 16, 2, 1), (100, 16, 1, 2),
                                      (100, 16, 2, 2), (97, 8, 3, 2), (150, 32, 2, 3),
                                      (40, 16, 4, 1)])
@pytest.mark.parametrize("nbmin,ndiv", [(4, 2), (16, 2), (4, 3)])
def test_grid2d_solve_threads_match_the_oracle(oracle, n, nb, P, Q, nbmin, ndiv):
    import threading

    from rochpl_b200.grid2d import LocalGrid2D
    from rochpl_b200.hpl import Algo

    algo = Algo(nb, min(nbmin, nb), ndiv, 2, 2, 1, 0)
    grp = LocalGrid2D(P, Q)
    out, errs = [None] * (P * Q), []

    def work(p, q):
        try:
            out[p * Q + q] = _run_rank(oracle, grp.comms(p, q), n, nb, P, Q, p, q, 100, algo)
        except BaseException as e:  # surfaced below
            errs.append(e)
            grp.abort()

    ts = [threading.Thread(target=work, args=(p, q)) for p in range(P) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=180)
    assert not errs, errs
    _check(oracle, n, nb, 100, algo, out)


@pytest.mark.parametrize("n,nb,P,Q,rfact", [(100, 16, 2, 2, 2), (97, 8, 3, 2, 2),
                                            (100, 16, 2, 2, 0), (97, 8, 3, 2, 1)])
def test_grid2d_device_backend_mapping_on_host_memory(oracle, n, nb, P, Q, rfact):
    """DeviceBackend2D's calls (element offsets, leading dimensions, sizes)
    through a stand-in for the library that does each C ABI call's work on
    host memory: the same solve as with the host backend."""
    import threading

    import torch

    from grid2d_host import FakeDeviceLib, local_to_global_2d
    from rochpl_b200.grid2d import (DeviceBackend2D, LocalGrid2D, matgen_local_2d,
                                    pdgesv_2d)
    from rochpl_b200.hpl import Algo

    algo = Algo(nb, 4, 2, 2, rfact, 1, 0)
    grp = LocalGrid2D(P, Q)
    out, errs = [None] * (P * Q), []

    def work(p, q):
        try:
            be = DeviceBackend2D(FakeDeviceLib(oracle))
            g = Grid2D(n, nb, p, q, P, Q)
            ld = max(g.mp, 1) + 1
            A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64)
            matgen_local_2d(be, g, 100, A, ld)
            x, ipiv, info = pdgesv_2d(be, grp.comms(p, q), g, algo, A, ld)
            out[p * Q + q] = (x.numpy().copy(), ipiv.numpy().copy(), info,
                              local_to_global_2d(g, A, ld))
        except BaseException as e:  # surfaced below
            errs.append(e)
            grp.abort()

    ts = [threading.Thread(target=work, args=(p, q)) for p in range(P) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=180)
    assert not errs, errs
    _check(oracle, n, nb, 100, algo, out)


@pytest.mark.parametrize("n,nb,P,Q", [(100, 16, 2, 2), (150, 32, 3, 2)])
@pytest.mark.parametrize("pfact,rfact", [(0, 1), (1, 0), (2, 1)])
def test_grid2d_left_and_crout_orderings_match_the_oracle(oracle, n, nb, P, Q, pfact, rfact):
    """RFACT's left-looking and Crout recursion orderings on the 2-D grid
    (the leaves right-looking for every PFACT, as hplb_pdgesv's)."""
    import threading

    from rochpl_b200.grid2d import LocalGrid2D
    from rochpl_b200.hpl import Algo

    algo = Algo(nb, 4, 2, pfact, rfact, 1, 0)
    grp = LocalGrid2D(P, Q)
    out, errs = [None] * (P * Q), []

    def work(p, q):
        try:
            out[p * Q + q] = _run_rank(oracle, grp.comms(p, q), n, nb, P, Q, p, q, 100, algo)
        except BaseException as e:  # surfaced below
            errs.append(e)
            grp.abort()

    ts = [threading.Thread(target=work, args=(p, q)) for p in range(P) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=180)
    assert not errs, errs
    _check(oracle, n, nb, 100, algo, out)


@pytest.mark.parametrize("n,nb,P,Q", [(100, 16, 2, 3), (97, 8, 3, 2)])  # P != Q: the orders differ
def test_grid2d_column_major_process_order_matches_the_oracle(oracle, n, nb, P, Q):
    """PMAP = 1: the world ranks in column-major order on the grid (the
    back-solve's broadcasts of x use them); the same solve as row-major."""
    import threading

    from rochpl_b200.grid2d import LocalGrid2D
    from rochpl_b200.hpl import Algo

    algo = Algo(nb, 4, 2, 2, 2, 1, 0)
    grp = LocalGrid2D(P, Q, pmap=1)
    out, errs = [None] * (P * Q), []

    def work(p, q):
        try:
            out[q * P + p] = _run_rank(oracle, grp.comms(p, q), n, nb, P, Q, p, q, 100, algo,
                                       pmap=1)
        except BaseException as e:  # surfaced below
            errs.append(e)
            grp.abort()

    ts = [threading.Thread(target=work, args=(p, q)) for p in range(P) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=180)
    assert not errs, errs
    _check(oracle, n, nb, 100, algo, out)


_CHILD = r"""
import json, os, sys
import numpy as np
import torch.distributed as dist
sys.path.insert(0, os.path.join(os.getcwd(), "tests"))
from oracle import oracle as O
from rochpl_b200.grid2d import dist_comms
from rochpl_b200.hpl import Algo
from test_grid2d import _run_rank
from rochpl_b200.grid2d import Grid2D
n, nb, P, Q, pmap = (int(os.environ[k]) for k in ("GN", "GNB", "GP", "GQ", "GPMAP"))
dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
p, q = Grid2D.coords(rank, P, Q, pmap)
comms = dist_comms(P, Q, pmap)
x, ipiv, info, F = _run_rank(O, comms, n, nb, P, Q, p, q, 100, Algo(nb, 8, 2, 2, 2, 1, 0),
                             pmap=pmap)
np.save(os.environ["GOUT"] + f"/rank{rank}.npy", F)
print("RESULT " + json.dumps({"rank": rank, "x": x.tolist(), "ipiv": ipiv.tolist(), "info": info}))
dist.destroy_process_group()
"""


@pytest.mark.parametrize("pmap", [0, 1])
def test_grid2d_solve_four_gloo_processes(oracle, tmp_path, pmap):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    n, nb, P, Q = 120, 16, 2, 2
    procs = []
    for rank in range(P * Q):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(P * Q), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), GN=str(n), GNB=str(nb),
                   GP=str(P), GQ=str(Q), GPMAP=str(pmap), GOUT=str(tmp_path),
                   PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
        procs.append(subprocess.Popen([sys.executable, "-c", _CHILD], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    res = []
    for pr in procs:
        try:
            so, se = pr.communicate(timeout=300)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert pr.returncode == 0, se[-3000:]
        line = [ln for ln in so.splitlines() if ln.startswith("RESULT ")][-1]
        res.append(json.loads(line[7:]))
    res.sort(key=lambda r: r["rank"])
    from rochpl_b200.hpl import Algo

    results = [(np.array(r["x"]), np.array(r["ipiv"], dtype=np.int32), r["info"],
                np.load(tmp_path / f"rank{r['rank']}.npy")) for r in res]
    _check(oracle, n, nb, 100, Algo(nb, 8, 2, 2, 2, 1, 0), results)


def test_grid2d_rejects_a_local_array_that_is_too_small(oracle):
    import torch

    from grid2d_host import HostBackend2D
    from rochpl_b200.grid2d import LocalGrid2D, pdgesv_2d
    from rochpl_b200.hpl import Algo

    g = Grid2D(64, 16, 0, 0, 1, 1)
    comms = LocalGrid2D(1, 1).comms(0, 0)
    algo = Algo(16, 4, 2, 2, 2, 1, 0)
    be = HostBackend2D(oracle)
    with pytest.raises(ValueError, match="ld >= 64"):
        pdgesv_2d(be, comms, g, algo, torch.zeros(63 * 65, dtype=torch.float64), 63)
    with pytest.raises(ValueError, match="entries"):
        pdgesv_2d(be, comms, g, algo, torch.zeros(64 * 65 - 1, dtype=torch.float64), 64)
    with pytest.raises(ValueError, match="float64"):
        pdgesv_2d(be, comms, g, algo, torch.zeros(64 * 65, dtype=torch.float32), 64)


def test_grid2d_rejects_nb_above_the_limit_before_any_exchange(oracle):
    import torch

    from grid2d_host import FakeDeviceLib
    from rochpl_b200.grid2d import DeviceBackend2D, LocalGrid2D, pdgesv_2d
    from rochpl_b200.hpl import Algo

    g = Grid2D(3000, 4096, 0, 0, 1, 1)
    with pytest.raises(ValueError, match="NB 4096 above the limits"):
        pdgesv_2d(DeviceBackend2D(FakeDeviceLib(oracle)), LocalGrid2D(1, 1).comms(0, 0), g,
                  Algo(4096), torch.zeros(3000 * 3001, dtype=torch.float64), 3000)


@pytest.mark.parametrize("fault", ["small_array", "other_n", "bad_algo_on_one"])
def test_grid2d_bad_call_on_one_process_stops_every_process(oracle, fault):
    """As for the 1 x Q grid: a bad call on one process of a 2 x 2 grid makes
    all four raise at the start of the solve."""
    import threading
    from dataclasses import replace

    import torch

    from grid2d_host import HostBackend2D
    from rochpl_b200.grid2d import LocalGrid2D, pdgesv_2d
    from rochpl_b200.hpl import Algo

    P, Q = 2, 2
    grp = LocalGrid2D(P, Q)
    errs = [None] * (P * Q)

    def work(p, q):
        r = p * Q + q
        n = 63 if (fault == "other_n" and r == 3) else 64
        algo = Algo(16, 4, 2, 2, 2, 1, 0)
        if fault == "bad_algo_on_one" and r == 2:
            algo = replace(algo, pfact=5)
        g = Grid2D(n, 16, p, q, P, Q)
        ld = max(g.mp, 1)
        size = ld * max(g.nq, 1) - (1 if (fault == "small_array" and r == 1) else 0)
        try:
            pdgesv_2d(HostBackend2D(oracle), grp.comms(p, q), g, algo,
                      torch.zeros(size, dtype=torch.float64), ld)
        except ValueError as e:
            errs[r] = str(e)
        except BaseException as e:  # anything else is a failure of the test
            errs[r] = e
            grp.abort()

    ts = [threading.Thread(target=work, args=(p, q)) for p in range(P) for q in range(Q)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=60)
    assert not any(t.is_alive() for t in ts), "a process was left waiting"
    assert all(isinstance(e, str) for e in errs), errs
