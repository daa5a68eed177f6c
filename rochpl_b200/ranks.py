"""Host-side plumbing for runs over several ranks, one process per GPU.

The FP64 solve at P = Q = 1 does not shard: each rank solves its own system
(replicas, seed 100 + rank) and the one exchange is the timing, the max over
ranks.  (One system across ranks is the process-grid solve of
rochpl_b200.grid, 1 x Q, and rochpl_b200.grid2d, P x Q, with communicators of
their own.)  The batched form shards: its systems are split across ranks
by a cost-balanced partition (batch.partition_systems), every rank generates
and solves only its own systems, and the one data exchange is the per-system
residual vector, assembled once at the end (Ranks.assemble).

Ranks reads RANK / WORLD_SIZE / LOCAL_RANK (and MASTER_ADDR / MASTER_PORT for
the rendezvous) from the environment, as torch.distributed.run sets them.
"""
from __future__ import annotations

import datetime
import os

import numpy as np

__all__ = ["Ranks", "rank_env"]


def rank_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Ranks:
    """One process group (NCCL on GPUs, gloo for host-only runs) or, at world
    size 1, none: every method is then a local no-op, so single-GPU code runs
    unchanged.  Every rank must call the same methods in the same order."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 1800.0):
        self.rank, self.world, self.local = rank_env()
        if not 0 <= self.rank < self.world:
            raise ValueError(f"RANK={self.rank} is outside WORLD_SIZE={self.world}")
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _tensor(self, values):
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.as_tensor(np.asarray(values, dtype=np.float64), device=dev).clone()

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, v: float) -> float:
        """The max of v over all ranks (device times are reported this way)."""
        if self.dist is None:
            return float(v)
        t = self._tensor([v])
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.cpu()[0])

    def sum(self, v: float) -> float:
        if self.dist is None:
            return float(v)
        t = self._tensor([v])
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.cpu()[0])

    def assemble(self, local_values, index, total: int) -> np.ndarray:
        """The full per-system vector (length `total`) from each rank's values
        for its own systems (`local_values[i]` belongs to global system
        `index[i]`).  Each rank places its values into a zero vector and one
        sum-all-reduce assembles it: every entry has exactly one owner, so the
        sum adds only zeros to it and is exact (NaN and inf included)."""
        index = np.asarray(index, dtype=np.int64)
        vals = np.asarray(local_values, dtype=np.float64).reshape(-1)
        if vals.size != index.size:
            raise ValueError("one value per owned system")
        if index.size and (index.min() < 0 or index.max() >= total):
            raise ValueError("system index outside the workload")
        full = np.zeros(total, dtype=np.float64)
        full[index] = vals
        if self.dist is None:
            return full
        owned = np.zeros(total, dtype=np.float64)
        owned[index] = 1.0
        t, c = self._tensor(full), self._tensor(owned)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        self.dist.all_reduce(c, op=self.dist.ReduceOp.SUM)
        if not np.array_equal(c.cpu().numpy(), np.ones(total)):
            raise ValueError("the ranks' systems do not cover the workload exactly once")
        return t.cpu().numpy()

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
