"""Batched solver: many independent LCG systems of uneven size in one
persistent, graph-captured launch (include/hplb.h, hplb_batch_*).

BatchPlan wraps one plan (layout, panel widths, work order, CUDA graphs);
autotune() runs the library's tuner and caches its table per GPU model and
right-hand-side count; workload_sizes() draws the system sizes of the batched
workload (N log-uniform in [32, 1024]).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os

import numpy as np

from .lib import HPLB_BATCH_CLASSES, Library

__all__ = ["BatchPlan", "BatchShard", "autotune", "workload_sizes", "batch_flops",
           "system_cost", "partition_systems"]

_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "batch_nb.json")


def workload_sizes(count: int = 4096, lo: int = 32, hi: int = 1024,
                   seed: int = 20261203) -> np.ndarray:
    """N_i = round(exp(U(ln lo, ln hi))) from numpy's PCG64 seeded with `seed`."""
    u = np.random.default_rng(seed).random(count)
    return np.rint(np.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))).astype(np.int32)


def system_cost(n, nrhs) -> np.ndarray:
    """Per-system flops 2/3 n^3 + 2 n^2 nrhs (LU + both triangular solves)."""
    n = np.asarray(n, dtype=np.float64)
    r = np.broadcast_to(np.asarray(nrhs, dtype=np.float64), n.shape)
    return 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2 * r


def batch_flops(n, nrhs) -> float:
    """Sum of system_cost over the systems."""
    return float(np.sum(system_cost(n, nrhs)))


def partition_systems(n, nrhs, world: int) -> list[np.ndarray]:
    """Split a batched workload across `world` ranks with balanced flops.

    Longest-processing-time greedy: systems in decreasing cost (ties by
    index) go one by one to the rank with the least cost so far (ties to the
    lowest rank).  The result depends only on the sizes, so every rank
    computes the same split and nothing is exchanged to agree on it.  The
    heaviest rank carries at most 4/3 of the optimal makespan, and exceeds the
    lightest by at most one system's cost.  Returns, per rank, the global
    indices of its systems in increasing order."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    cost = system_cost(n, nrhs)
    order = np.lexsort((np.arange(cost.size), -cost))
    load = [0.0] * world
    owner = np.empty(cost.size, dtype=np.int64)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += float(cost[i])
    return [np.flatnonzero(owner == r) for r in range(world)]


class BatchPlan:
    """One hplb_batch plan on a Library context."""

    def __init__(self, lib: Library, n, nrhs, nb_by_class=None):
        self.lib = lib
        self.n = np.ascontiguousarray(n, dtype=np.int32)
        nrhs = np.broadcast_to(np.asarray(nrhs, dtype=np.int32), self.n.shape)
        self.nrhs = np.ascontiguousarray(nrhs)
        self.count = int(self.n.size)
        L = lib.L
        table = None
        if nb_by_class is not None:
            table = (C.c_int * HPLB_BATCH_CLASSES)(*[int(v) for v in nb_by_class])
        h = C.c_void_p()
        ip = C.POINTER(C.c_int)
        st = L.hplb_batch_create(lib.ctx, self.count, self.n.ctypes.data_as(ip),
                                 self.nrhs.ctypes.data_as(ip), table, C.byref(h))
        lib._check(st)
        self.h = h
        a, b, p = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        self.a_off = np.zeros(self.count, dtype=np.int64)
        self.b_off = np.zeros(self.count, dtype=np.int64)
        self.p_off = np.zeros(self.count, dtype=np.int64)
        self.nb = np.zeros(self.count, dtype=np.int32)
        i64p = C.POINTER(C.c_int64)
        lib._check(L.hplb_batch_layout(h, C.byref(a), C.byref(b), C.byref(p),
                                       self.a_off.ctypes.data_as(i64p),
                                       self.b_off.ctypes.data_as(i64p),
                                       self.p_off.ctypes.data_as(i64p),
                                       self.nb.ctypes.data_as(ip)))
        self.a_elems, self.b_elems, self.p_elems = a.value, b.value, p.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.L.hplb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _seeds(self, seeds):
        s = np.ascontiguousarray(np.broadcast_to(np.asarray(seeds, dtype=np.uint64),
                                                 self.n.shape))
        return s, s.ctypes.data_as(C.POINTER(C.c_uint64))

    def matgen(self, seeds, dA: int, dB: int):
        s, sp = self._seeds(seeds)
        self.lib._check(self.lib.L.hplb_batch_matgen(self.h, sp, dA, dB or None))

    def gesv(self, dA: int, dB: int, dipiv: int, dinfo: int):
        self.lib._check(self.lib.L.hplb_batch_gesv(self.h, dA, dB or None, dipiv, dinfo))

    def getrs(self, trans: int, dLU: int, dipiv: int, dB: int):
        self.lib._check(self.lib.L.hplb_batch_getrs(self.h, int(trans), dLU, dipiv, dB))

    def rank_k(self, alpha: float, dX: int, dY: int, dC: int):
        self.lib._check(self.lib.L.hplb_batch_rank_k(self.h, float(alpha), dX or None,
                                                     dY or None, dC))

    def residual(self, seeds, dX: int, dres: int):
        s, sp = self._seeds(seeds)
        self.lib._check(self.lib.L.hplb_batch_residual(self.h, sp, dX or None, dres))

    @property
    def last_ms(self) -> float:
        v = C.c_double(0)
        self.lib._check(self.lib.L.hplb_batch_last_ms(self.h, C.byref(v)))
        return v.value

    def flops(self) -> float:
        return batch_flops(self.n, self.nrhs)


class BatchShard:
    """One rank's part of a batched workload split by partition_systems: the
    global indices of its systems, their seeds (seed_base + global index, so
    every system is generated and solved exactly as in a one-rank run) and a
    BatchPlan over them.  Ranks.assemble puts per-system results back in
    global order."""

    def __init__(self, lib: Library, n, nrhs, rank: int, world: int, nb_by_class=None,
                 seed_base: int = 100):
        n = np.asarray(n, dtype=np.int32)
        nrhs = np.broadcast_to(np.asarray(nrhs, dtype=np.int32), n.shape)
        if not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside world size {world}")
        self.total = int(n.size)
        self.total_flops = batch_flops(n, nrhs)
        self.index = partition_systems(n, nrhs, world)[rank]
        self.seeds = (np.uint64(seed_base) + self.index.astype(np.uint64)).astype(np.uint64)
        self.plan = BatchPlan(lib, n[self.index], nrhs[self.index], nb_by_class)

    def close(self):
        self.plan.close()


def autotune(lib: Library, nrhs: int = 16, use_cache: bool = True) -> list[int]:
    """Panel width per size class from hplb_batch_tune, cached in
    tuning/batch_nb.json under the GPU model and nrhs."""
    import torch

    key = f"{torch.cuda.get_device_name(lib.device)}|nrhs={nrhs}"
    cache = {}
    if use_cache and os.path.exists(_CACHE):
        try:
            with open(_CACHE) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return [int(v) for v in cache[key]["nb_by_class"]]
    nb = (C.c_int * HPLB_BATCH_CLASSES)()
    ms = (C.c_double * (HPLB_BATCH_CLASSES * 4))()
    st = lib.L.hplb_batch_tune(lib.ctx, nrhs, nb, ms)
    lib._check(st)
    table = [int(v) for v in nb]
    cache[key] = {"nb_by_class": table, "ms_nb8_16_32_recursive": [float(v) for v in ms]}
    try:
        os.makedirs(os.path.dirname(_CACHE), exist_ok=True)
        with open(_CACHE, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
    return table
