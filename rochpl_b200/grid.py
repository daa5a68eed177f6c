"""HPL_pdgesv on a 1 x Q process grid: one system across Q GPUs.

rocHPL distributes [A|b] over a P x Q process grid in NB x NB blocks
(src/matgen/HPL_pdmatgen.cpp:85-383) and factors it with HPL_pdgesv
(src/pgesv/HPL_pdgesv.cpp:168-344): the process column owning panel j factors
it (HPL_pdfact), broadcasts it along the process row
(src/panel/HPL_pdpanel_bcast.cpp:49), and every process applies the row
interchanges and the trailing update to its own columns (HPL_pdlaswp,
HPL_pdupdateTT), with look-ahead: the owner of panel j+1 updates that panel
first, factors it and starts its broadcast before the rest of the update.
The back-solve (HPL_pdtrsv) walks the column blocks from the last.

This module is that loop for P = 1, Q >= 1 (each process holds every row of
its column blocks, so the pivot search needs no communication and no U
broadcast is needed), written once, SPMD style, over two interfaces:

* a backend for the local work -- DeviceBackend runs the C ABI building
  blocks (hplb_matgen_block, hplb_panel_factor, hplb_panel_update,
  hplb_trsv_block) on the GPU; the tests supply a host backend;
* a communicator with broadcast / all_reduce on torch tensors --
  torch.distributed (NCCL over NVLink between GPUs, gloo on the host), or
  LocalGroup, which runs Q ranks as threads of one process (for tests on one
  device: no kernel ever waits on another, the ranks meet on the host).

The panel broadcast is asynchronous: ranks that do not own panel j+1 start
receiving it before they update with panel j, so the transfer overlaps the
update as HPL's look-ahead intends.  Layout: NB-wide column block c of [A|b]
lives on process c mod Q at local columns (c div Q) * NB .. + NB, all n rows,
leading dimension ld (>= n); the right-hand side b is global column n.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass

import torch

__all__ = ["check_algo", "numroc", "Grid1xQ", "DeviceBackend", "LocalGroup", "DistGroup",
           "pdgesv_grid", "matgen_local"]


def check_algo(algo) -> None:
    """The checks hplb_pdgesv makes on the solve's HPL.dat parameters (the
    HPL_pdinfo rules, src/pauxil/HPL_pdinfo.cpp, plus this library's limits),
    made by every process before its first exchange, so that a bad value stops
    the whole grid at once instead of the one process that factors a panel."""
    if algo.nb < 1 or algo.nbmin < 1 or algo.ndiv < 2:
        raise ValueError(f"NB {algo.nb}, NBMIN {algo.nbmin}, NDIV {algo.ndiv}: "
                         "NB and NBMIN must be at least 1, NDIV at least 2")
    if not (0 <= algo.pfact <= 2 and 0 <= algo.rfact <= 2):
        raise ValueError(f"PFACT {algo.pfact} / RFACT {algo.rfact} outside 0 (left), "
                         "1 (Crout), 2 (right)")
    if algo.depth != 1:
        raise ValueError("only look-ahead depth 1 is supported")
    if algo.nbmin > 128 or algo.nb > 2048:
        raise ValueError(f"NBMIN {algo.nbmin} / NB {algo.nb} above the limits 128 / 2048")


def start_checks(comm, values, local_error, algo, device) -> None:
    """The first step of a grid solve, the same on every process: one small
    all-gather of this process's problem and solve parameters (`values`) and
    of whether its local array is usable (`local_error`: a message, or None).
    Then every process raises if its own array is unusable, if another
    process's is, if the parameters differ between processes, or if
    check_algo rejects them -- so a bad call stops the whole grid at once
    instead of leaving processes waiting in an exchange that one of them
    never reaches."""
    flags = [float(v) for v in values] + [0.0 if local_error is None else 1.0]
    allv = comm.all_gather(torch.tensor(flags, dtype=torch.float64, device=device)).cpu()
    if local_error is not None:
        raise ValueError(local_error)
    bad = [r for r in range(allv.shape[0]) if allv[r, -1] != 0]
    if bad:
        raise ValueError(f"process {bad[0]} of the grid cannot run the solve (its local array)")
    diff = [r for r in range(allv.shape[0]) if not torch.equal(allv[r, :-1], allv[0, :-1])]
    if diff:
        raise ValueError(f"the problem or solve parameters of process {diff[0]} differ from "
                         "those of process 0")
    check_algo(algo)


def _algo_values(algo):
    return [algo.nb, algo.nbmin, algo.ndiv, algo.pfact, algo.rfact, algo.depth]


def numroc(n: int, nb: int, iproc: int, nprocs: int) -> int:
    """Columns of an n-column matrix in NB blocks that process iproc of nprocs
    holds, the distribution starting on process 0 (HPL_numroc)."""
    nblocks, rem = divmod(n, nb)
    num = (nblocks // nprocs) * nb
    extra = nblocks % nprocs
    if iproc < extra:
        num += nb
    elif iproc == extra:
        num += rem
    return num


@dataclass
class Grid1xQ:
    """Column-block bookkeeping of the N x (N+1) [A|b] on process q of Q."""
    n: int
    nb: int
    q: int
    Q: int

    @property
    def nq(self) -> int:
        return numroc(self.n + 1, self.nb, self.q, self.Q)

    @property
    def npanels(self) -> int:
        return (self.n + self.nb - 1) // self.nb

    def owner(self, gcol: int) -> int:
        return (gcol // self.nb) % self.Q

    def local(self, gcol: int) -> int:
        """Local column of global column gcol (on its owner)."""
        return (gcol // self.nb // self.Q) * self.nb + gcol % self.nb

    def _blocks_before(self, b: int) -> int:
        """How many of this process's blocks come before global block b."""
        return max(0, -(-(b - self.q) // self.Q))

    def local_from(self, gcol: int) -> int:
        """First local column holding a global column >= gcol: inside block
        gcol / NB if that block is here, else the start of this process's next
        block."""
        b = gcol // self.nb
        if b % self.Q == self.q:
            return self._blocks_before(b) * self.nb + gcol % self.nb
        return self._blocks_before(b + 1) * self.nb

    def local_blocks(self):
        """(local column, first global column, width) of each block held here."""
        lc = 0
        for b in range(self.q, (self.n + 1 + self.nb - 1) // self.nb, self.Q):
            g0 = b * self.nb
            w = min(self.nb, self.n + 1 - g0)
            yield lc, g0, w
            lc += w

    def panel(self, p: int):
        """(first row/column j, width jb, owner, owner's local column)."""
        j = p * self.nb
        jb = min(self.nb, self.n - j)
        return j, jb, p % self.Q, (p // self.Q) * self.nb


class DeviceBackend:
    """The local work through the C ABI on this process's GPU."""

    def __init__(self, lib):
        self.lib = lib

    def matgen_block(self, n: int, g0: int, w: int, seed: int, A, ld: int, lc: int):
        self.lib.matgen_block(n, n + 1, 0, g0, n, w, seed, A.data_ptr() + 8 * lc * ld, ld)

    def panel_factor(self, algo, n, j, jb, A, ld, lc, ipiv) -> int:
        return self.lib.panel_factor(algo.c(), n, j, jb, A.data_ptr(), ld, lc, ipiv.data_ptr())

    def update(self, n, j, jb, L, ldl, ipiv, A, ld, c0, ncols):
        if ncols > 0:
            self.lib.panel_update(n, j, jb, L.data_ptr(), ldl, ipiv.data_ptr(), A.data_ptr(), ld,
                                  c0, ncols)

    def trsv_block(self, n, j, jb, A, ld, lc, y, s, x, z):
        self.lib.trsv_block(n, j, jb, A.data_ptr(), ld, lc, y.data_ptr(), s.data_ptr(),
                            x.data_ptr(), z.data_ptr())


class _Done:
    def wait(self):
        return None


class DistGroup:
    """torch.distributed collectives (NCCL between GPUs, gloo on the host)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def broadcast(self, t, src: int, async_op: bool = False):
        w = self.dist.broadcast(t, src=self.dist.get_global_rank(self.group, src)
                                if self.group is not None else src,
                                group=self.group, async_op=async_op)
        return w if async_op else _Done()

    def all_reduce_sum(self, t):
        self.dist.all_reduce(t, group=self.group)

    def all_gather(self, t):
        """(size, *t.shape): every member's t, in rank order."""
        out = [torch.empty_like(t) for _ in range(self.size)]
        self.dist.all_gather(out, t, group=self.group)
        return torch.stack(out)


class LocalGroup:
    """Q ranks as threads of one process: rank r calls LocalGroup.member(r)
    from its own thread.  Collectives meet on a barrier and copy between the
    ranks' tensors (device-to-device on a GPU), so no kernel waits on another."""

    def __init__(self, size: int):
        self.size = size
        self.barrier = threading.Barrier(size)
        self.slots = [None] * size

    def member(self, rank: int):
        return _LocalMember(self, rank)


class _LocalMember:
    def __init__(self, group: LocalGroup, rank: int):
        self.g, self.rank, self.size = group, rank, group.size

    def _sync(self, t):
        if t.is_cuda:
            torch.cuda.synchronize(t.device)

    def broadcast(self, t, src: int, async_op: bool = False):
        self._sync(t)
        self.g.slots[self.rank] = t
        self.g.barrier.wait()
        if self.rank != src:
            t.copy_(self.g.slots[src])
            self._sync(t)
        self.g.barrier.wait()
        return _Done()

    def all_reduce_sum(self, t):
        self._sync(t)
        self.g.slots[self.rank] = t.clone()
        self.g.barrier.wait()
        acc = self.g.slots[0].clone()
        for r in range(1, self.size):
            acc += self.g.slots[r]
        self.g.barrier.wait()
        t.copy_(acc)
        self._sync(t)

    def all_gather(self, t):
        self._sync(t)
        self.g.slots[self.rank] = t.clone()
        self.g.barrier.wait()
        out = torch.stack([s.to(t.device) for s in self.g.slots])
        self.g.barrier.wait()
        self._sync(out)
        return out


def matgen_local(backend, grid: Grid1xQ, seed: int, A, ld: int):
    """This process's columns of the HPL LCG [A|b] (HPL_pdmatgen at P = 1)."""
    for lc, g0, w in grid.local_blocks():
        backend.matgen_block(grid.n, g0, w, seed, A, ld, lc)


def pdgesv_grid(backend, comm, grid: Grid1xQ, algo, A, ld: int):
    """Factor and solve the distributed [A|b] (this process's local array A,
    a flat float64 tensor of ld * nq entries, column-major).  Every process
    returns (x, ipiv, info): x (n), the global pivot vector (ipiv[j] = row
    swapped into row j) and the first zero-pivot column (1-based, 0 if none),
    all replicated.  On exit A holds this process's columns of the factors."""
    n, nb, q = grid.n, grid.nb, grid.q
    dev, f64, i32 = A.device, torch.float64, torch.int32
    err = None
    if A.dtype != f64:
        err = "A must be a float64 tensor"
    elif ld < max(n, 1) or A.numel() < ld * grid.nq:
        err = (f"process {q} holds {n} x {grid.nq}: needs ld >= {max(n, 1)} and "
               f"ld * {grid.nq} entries (ld {ld}, {A.numel()} entries)")
    start_checks(comm, [n, nb, grid.Q] + _algo_values(algo), err, algo, dev)
    ldl = (n + 1) & ~1  # even leading dimension of the broadcast panels
    Lb = [torch.zeros(ldl * nb, dtype=f64, device=dev) for _ in range(2)]
    # nb pivots + the panel's zero-pivot column, per buffer.
    Pb = [torch.zeros(nb + 1, dtype=i32, device=dev) for _ in range(2)]
    ipiv = torch.zeros(max(n, 1), dtype=i32, device=dev)
    nq = grid.nq
    Acols = A.view(-1)[: ld * nq].view(nq, ld) if nq > 0 else None
    info = 0

    def factor(p: int, buf: int):
        """Owner of panel p: factor it and pack L and the pivots for broadcast."""
        j, jb, owner, lc = grid.panel(p)
        if q != owner:
            return
        inf = backend.panel_factor(algo, n, j, jb, A, ld, lc, Pb[buf])
        Pb[buf][nb] = inf
        m = n - j
        Lb[buf][: ldl * jb].view(jb, ldl)[:, :m].copy_(Acols[lc:lc + jb, j:n])

    def send(p: int, buf: int):
        j, jb, owner, _ = grid.panel(p)
        m = n - j
        h1 = comm.broadcast(Lb[buf][: ldl * jb], owner, async_op=True)
        h2 = comm.broadcast(Pb[buf], owner, async_op=True)
        return (h1, h2)

    npan = grid.npanels
    if npan == 0:
        return torch.zeros(0, dtype=f64, device=dev), ipiv[:0], 0
    factor(0, 0)
    pending = send(0, 0)
    for p in range(npan):
        buf = p & 1
        for h in pending:
            h.wait()
        j, jb, owner, _ = grid.panel(p)
        ipiv[j:j + jb] = Pb[buf][:jb]
        pinfo = int(Pb[buf][nb])
        if pinfo and not info:
            info = pinfo
        c0 = grid.local_from(j + jb)
        ncols = nq - c0
        L = Lb[buf]
        if p + 1 < npan:
            nj, njb, nowner, nlc = grid.panel(p + 1)
            if q == nowner:  # look-ahead: the next panel's columns, then factor it
                backend.update(n, j, jb, L, ldl, Pb[buf], A, ld, nlc, njb)
                factor(p + 1, buf ^ 1)
            pending = send(p + 1, buf ^ 1)
            if q == nowner:
                backend.update(n, j, jb, L, ldl, Pb[buf], A, ld, nlc + njb, ncols - njb)
            else:
                backend.update(n, j, jb, L, ldl, Pb[buf], A, ld, c0, ncols)
        else:
            backend.update(n, j, jb, L, ldl, Pb[buf], A, ld, c0, ncols)

    # Back-solve U x = y, y = column n after the updates, on its owner.
    y = torch.zeros(n, dtype=f64, device=dev)
    if q == grid.owner(n):
        y.copy_(Acols[grid.local(n), :n])
    comm.broadcast(y, grid.owner(n))
    z = torch.zeros(n, dtype=f64, device=dev)  # this process's sum of U[:, c] x_c so far
    x = torch.zeros(n, dtype=f64, device=dev)
    s = torch.zeros(nb, dtype=f64, device=dev)
    for p in range(npan - 1, -1, -1):
        j, jb, owner, lc = grid.panel(p)
        s[:jb].copy_(z[j:j + jb])
        comm.all_reduce_sum(s[:jb])
        if q == owner:
            backend.trsv_block(n, j, jb, A, ld, lc, y, s, x, z)
    comm.all_reduce_sum(x)  # each block of x is nonzero on its owner only
    return x, ipiv[:n], info
