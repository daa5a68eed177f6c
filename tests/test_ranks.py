"""Multi-rank host logic on CPU: the cost-balanced split of the batched
workload (batch.partition_systems) and the rank plumbing (ranks.Ranks: max
over ranks, barrier, the residual assembly) over a world-size-2 gloo group,
two processes on 127.0.0.1.  No GPU: these check what every rank computes and
exchanges, not the kernels."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from rochpl_b200.batch import partition_systems, system_cost, workload_sizes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("nrhs", [1, 16, 64])
def test_partition_covers_and_balances(world, nrhs):
    n = workload_sizes(4096)
    parts = partition_systems(n, nrhs, world)
    assert len(parts) == world
    allidx = np.concatenate(parts)
    assert np.array_equal(np.sort(allidx), np.arange(n.size))  # each system exactly once
    for p in parts:
        assert np.all(np.diff(p) > 0)  # increasing global order
    cost = system_cost(n, nrhs)
    loads = np.array([cost[p].sum() for p in parts])
    assert loads.max() - loads.min() <= cost.max() * (1 + 1e-12)
    # The greedy's makespan bound against the trivial lower bound.
    assert loads.max() <= 4.0 / 3.0 * max(cost.sum() / world, cost.max()) * (1 + 1e-12)
    # The split depends on the sizes only.
    again = partition_systems(n.copy(), nrhs, world)
    assert all(np.array_equal(a, b) for a, b in zip(parts, again))


def test_partition_edges():
    assert [p.tolist() for p in partition_systems(np.array([5, 7], np.int32), 1, 4)] == \
        [[1], [0], [], []]
    assert [p.tolist() for p in partition_systems(np.zeros(0, np.int32), 1, 2)] == [[], []]
    # Equal costs: round robin from rank 0, in index order.
    assert [p.tolist() for p in partition_systems(np.full(5, 9, np.int32), 1, 2)] == \
        [[0, 2, 4], [1, 3]]
    with pytest.raises(ValueError):
        partition_systems(np.array([4], np.int32), 1, 0)


def test_ranks_world_one_is_local():
    from rochpl_b200.ranks import Ranks

    env = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        r = Ranks("gloo")
        assert (r.rank, r.world) == (0, 1) and r.dist is None
        assert r.max(2.5) == 2.5 and r.sum(1.5) == 1.5
        r.barrier()
        full = r.assemble([3.0, 4.0], [2, 0], 3)
        assert full.tolist() == [4.0, 0.0, 3.0]
        with pytest.raises(ValueError):
            r.assemble([1.0], [5], 3)
        r.close()
    finally:
        os.environ.update(env)


_CHILD = r"""
import json, sys
import numpy as np
from rochpl_b200.batch import partition_systems, system_cost, workload_sizes
from rochpl_b200.ranks import Ranks

r = Ranks("gloo", timeout_s=60)
out = {"rank": r.rank, "world": r.world}
out["max"] = r.max(10.0 + r.rank)
out["sum"] = r.sum(1.0 + r.rank)
r.barrier()
n = workload_sizes(4096)
mine = partition_systems(n, 16, r.world)[r.rank]
# A per-system result each rank computes for its own systems only.
vals = np.sin(mine.astype(np.float64)) * system_cost(n[mine], 16)
full = r.assemble(vals, mine, n.size)
ref = np.sin(np.arange(n.size, dtype=np.float64)) * system_cost(n, 16)
out["assembled_exact"] = bool(np.array_equal(full, ref))
out["owned"] = int(mine.size)
# A wrong split (both ranks claim system 0) is caught on every rank.
bad = np.union1d(mine, [0])
try:
    r.assemble(np.ones(bad.size), bad, n.size)
    out["overlap_caught"] = False
except ValueError:
    out["overlap_caught"] = True
r.close()
print("RESULT " + json.dumps(out))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_group():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
        procs.append(subprocess.Popen([sys.executable, "-c", _CHILD], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    results = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, se[-2000:]
        line = [ln for ln in so.splitlines() if ln.startswith("RESULT ")][-1]
        results.append(json.loads(line[7:]))
    assert sorted(r["rank"] for r in results) == [0, 1]
    for r in results:
        assert r["world"] == 2 and r["max"] == 11.0 and r["sum"] == 3.0
        assert r["assembled_exact"] and r["overlap_caught"]
    assert sum(r["owned"] for r in results) == 4096
