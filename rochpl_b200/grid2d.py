"""HPL_pdgesv on a P x Q process grid: one system across P * Q GPUs.

rocHPL distributes [A|b] over the grid in NB x NB blocks, block (I, J) on
process (I mod P, J mod Q) (src/matgen/HPL_pdmatgen.cpp:85-383), and
HPL_pdgesv (src/pgesv/HPL_pdgesv.cpp:168-344) runs, per panel j:

* the panel factorisation on the process column owning columns j .. j+jb
  (HPL_pdfact, src/pfact/HPL_pdfact.cpp:20-110): the recursion of
  HPL_pdrpanrlT (src/pfact/HPL_pdrpanrlT.cpp:74-160) over NBMIN-wide leaves;
  every column's pivot is the arg-max over all P processes of the column,
  combined with the pivot row and the current diagonal row as
  HPL_pdmxswp / HPL_all_reduce_dmxswp do (src/pfact/HPL_pdmxswp.cpp:19-126);
  the jb x jb top block ("L1") is kept replicated on every process of the
  column, the rows below ("L2") stay where they live;
* the panel broadcast along each process row (src/panel/HPL_pdpanel_bcast.cpp);
* the row interchanges of the trailing columns (HPL_pdlaswp,
  src/pgesv/HPL_pdlaswp.cpp:261-289): the top rows and the rows they trade
  with are gathered over the process column, U = L1^-1 (new top rows) is
  formed from them, and each process writes back the rows it owns;
* the trailing update A22 -= L2 U on every process's own blocks.

The back-solve (HPL_pdtrsv) walks the row blocks from the last: the partial
sums of each block's rows are reduced along its process row, the owner of the
diagonal block solves, and x_b is broadcast to every process.

This module is that algorithm written once, SPMD style, over a backend for the
local work (DeviceBackend2D runs it through the C ABI on each process's GPU;
the tests supply a host one) and three communicators -- the process row, the
process column and the whole grid -- with broadcast / all_gather /
all_reduce on tensors (torch.distributed groups, or LocalGroup threads).  The
panel recursion takes RFACT's right-looking or left-looking / Crout order (the
orderings of hplb_pdgesv's panel); its leaves are right-looking for every
PFACT, as hplb_pdgesv's are.  Look-ahead is not used (the order of the work
changes, its results do not).  Every process returns x, the global pivot vector and info, replicated.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .grid import _algo_values, numroc, start_checks

__all__ = ["Grid2D", "DeviceBackend2D", "pdgesv_2d", "matgen_local_2d", "LocalGrid2D", "dist_comms"]


@dataclass
class Grid2D:
    """Block-cyclic bookkeeping of the N x (N+1) [A|b] on process (p, q) of a
    P x Q grid.  pmap is HPL.dat's PMAP, the order of the processes on the
    grid (HPL_grid_init, src/grid/HPL_grid_init.cpp:86-109, on one node,
    where rocHPL's node-local tile is the whole grid): 0 row-major
    (rank = p Q + q), 1 column-major (rank = q P + p)."""
    n: int
    nb: int
    p: int
    q: int
    P: int
    Q: int
    pmap: int = 0

    @property
    def mp(self) -> int:
        return numroc(self.n, self.nb, self.p, self.P)

    @property
    def nq(self) -> int:
        return numroc(self.n + 1, self.nb, self.q, self.Q)

    @property
    def npanels(self) -> int:
        return (self.n + self.nb - 1) // self.nb

    def rank_of(self, p: int, q: int) -> int:
        return p * self.Q + q if self.pmap == 0 else q * self.P + p

    @staticmethod
    def coords(rank: int, P: int, Q: int, pmap: int = 0):
        """(p, q) of `rank` on a P x Q grid in PMAP order."""
        return divmod(rank, Q) if pmap == 0 else (rank % P, rank // P)

    def row_owner(self, g: int) -> int:
        return (g // self.nb) % self.P

    def col_owner(self, g: int) -> int:
        return (g // self.nb) % self.Q

    def lrow(self, g: int) -> int:
        """Local row of global row g (on its owner)."""
        return (g // self.nb // self.P) * self.nb + g % self.nb

    def lcol(self, g: int) -> int:
        return (g // self.nb // self.Q) * self.nb + g % self.nb

    @staticmethod
    def _from(g: int, nb: int, me: int, nprocs: int) -> int:
        b = g // nb
        before = lambda bb: max(0, -(-(bb - me) // nprocs))  # noqa: E731
        if b % nprocs == me:
            return before(b) * nb + g % nb
        return before(b + 1) * nb

    def lrow_from(self, g: int) -> int:
        """First local row holding a global row >= g."""
        return min(self._from(g, self.nb, self.p, self.P), self.mp)

    def lcol_from(self, g: int) -> int:
        return min(self._from(g, self.nb, self.q, self.Q), self.nq)

    def grow(self, lr: int) -> int:
        """Global row of local row lr."""
        return ((lr // self.nb) * self.P + self.p) * self.nb + lr % self.nb

    def row_blocks(self):
        """(local row, first global row, height) of each row block held here."""
        lr = 0
        for b in range(self.p, self.npanels, self.P):
            h = min(self.nb, self.n - b * self.nb)
            yield lr, b * self.nb, h
            lr += h

    def col_blocks(self):
        lc = 0
        for b in range(self.q, (self.n + 1 + self.nb - 1) // self.nb, self.Q):
            w = min(self.nb, self.n + 1 - b * self.nb)
            yield lc, b * self.nb, w
            lc += w

    def panel(self, k: int):
        """(first row/column j, width jb, diagonal process row, owner column)."""
        j = k * self.nb
        return j, min(self.nb, self.n - j), k % self.P, k % self.Q


class DeviceBackend2D:
    """The local work of the 2-D grid through the C ABI on this process's GPU.
    Local arrays are flat float64 CUDA tensors, column-major, addressed by
    element offsets."""

    def __init__(self, lib):
        self.lib = lib

    @staticmethod
    def _p(t, off=0):
        return t.data_ptr() + 8 * off

    def matgen_block(self, n, i0, j0, m, w, seed, A, ld, lr, lc):
        self.lib.matgen_block(n, n + 1, i0, j0, m, w, seed, self._p(A, lr + lc * ld), ld)

    def col_argmax(self, A, ld, r0, r1, c):
        return self.lib.col_argmax(self._p(A), ld, r0, r1, c)

    def col_rank1(self, A, ld, r0, r1, c0, k, kend, piv, u):
        self.lib.col_rank1(self._p(A), ld, r0, r1, c0, k, kend, piv, self._p(u))

    def gemm_sub(self, m, n, k, A, lda, ao, B, ldb, bo, C, ldc, co):
        if m > 0 and n > 0 and k > 0:
            self.lib.dgemm_sub(m, n, k, self._p(A, ao), lda, self._p(B, bo), ldb,
                               self._p(C, co), ldc)

    def trsm_lower_unit(self, n, nrhs, L, ldl, lo, X, ldx, xo):
        if n > 0 and nrhs > 0:
            self.lib.trsm_lower_unit(n, nrhs, self._p(L, lo), ldl, self._p(X, xo), ldx)

    def upper_solve(self, U, ldu, uo, n, y, x):
        self.lib.trsm_upper(n, 1, self._p(U, uo), ldu, self._p(y), n, self._p(x), n)


def _block(A, ld, r0, c0, m, w):
    """View of the m x w block at (r0, c0) of a flat column-major array, as a
    (w, m) tensor (one row per column)."""
    if m <= 0 or w <= 0:
        return A[:0].view(0, 0)
    end = r0 + c0 * ld + (w - 1) * ld + m
    if r0 < 0 or c0 < 0 or end > A.numel():
        raise IndexError(f"block ({r0}, {c0}) {m} x {w} outside an array of {A.numel()}")
    return A.as_strided((w, m), (ld, 1), A.storage_offset() + r0 + c0 * ld)


def matgen_local_2d(backend, grid: Grid2D, seed: int, A, ld: int):
    """This process's blocks of the HPL LCG [A|b] (HPL_pdmatgen)."""
    for lr, i0, h in grid.row_blocks():
        for lc, j0, w in grid.col_blocks():
            backend.matgen_block(grid.n, i0, j0, h, w, seed, A, ld, lr, lc)


def _better(av, ar, bv, br) -> bool:
    """HPL's order: the larger |value|, then the lower global row."""
    if br < 0:
        return ar >= 0
    if ar < 0:
        return False
    if abs(av) != abs(bv):
        return abs(av) > abs(bv)
    return ar < br


def pdgesv_2d(backend, comms, grid: Grid2D, algo, A, ld: int):
    """Factor and solve the distributed [A|b] (this process's local array A,
    a flat float64 tensor of ld * nq entries, column-major, ld >= mp).
    comms = (row, col, world): the process row (rank q of Q), the process
    column (rank p of P) and the whole grid (rank p Q + q).  Returns
    (x, ipiv, info) on every process: x (n), the global pivot vector
    (ipiv[j] = row swapped into row j) and the first zero-pivot column
    (1-based, 0 if none).  On exit A holds this process's blocks of the
    factors (U; the multipliers unpivoted across panels, as in rocHPL)."""
    row, col, world = comms
    n, nb, p, q = grid.n, grid.nb, grid.p, grid.q
    dev, f64 = A.device, torch.float64
    mp, nq = grid.mp, grid.nq
    err = None
    if A.dtype != f64 or A.dim() != 1:
        err = "A must be a flat float64 tensor"
    elif ld < max(mp, 1) or A.numel() < ld * max(nq, 1):
        err = (f"process ({p}, {q}) holds {mp} x {nq}: needs ld >= {max(mp, 1)} and "
               f"ld * {max(nq, 1)} entries (ld {ld}, {A.numel()} entries)")
    # Over the whole grid, before any other exchange (NB <= 2048 among the checks).
    start_checks(world, [n, nb, grid.P, grid.Q] + _algo_values(algo), err, algo, dev)
    nbmin = max(1, min(algo.nbmin, nb))
    ndiv = max(2, algo.ndiv)
    ipiv = torch.zeros(max(n, 1), dtype=torch.int64)
    info = 0
    for k in range(grid.npanels):
        j, jb, pj, qj = grid.panel(k)
        lr2 = grid.lrow_from(j + jb)  # first local row below the panel's top block
        m2 = mp - lr2
        T = torch.zeros(jb * jb, dtype=f64, device=dev)  # the replicated top block (L1)
        Lb = torch.zeros(max(m2, 0) * jb, dtype=f64, device=dev)  # this row's L2
        piv = torch.zeros(jb + 1, dtype=f64, device=dev)  # pivots (global rows) and info
        if q == qj:
            lc = grid.lcol(j)
            if p == pj:
                _block(T, jb, 0, 0, jb, jb).copy_(_block(A, ld, grid.lrow(j), lc, jb, jb))
            col.broadcast(T, pj)
            pinfo = _factor_panel(backend, col, grid, j, jb, lc, lr2, T, A, ld, nbmin, ndiv,
                                  algo.rfact, piv)
            piv[jb] = float(pinfo)
            if p == pj:
                _block(A, ld, grid.lrow(j), lc, jb, jb).copy_(_block(T, jb, 0, 0, jb, jb))
            if m2 > 0:
                _block(Lb, m2, 0, 0, m2, jb).copy_(_block(A, ld, lr2, lc, m2, jb))
        row.broadcast(T, qj)
        row.broadcast(piv, qj)
        if m2 > 0:
            row.broadcast(Lb, qj)
        pv = piv.cpu()
        ipiv[j:j + jb] = pv[:jb].to(torch.int64)
        if int(pv[jb]) and not info:
            info = int(pv[jb])
        _update(backend, col, grid, j, jb, pj, T, Lb, lr2, m2, ipiv, A, ld)
    x = _backsolve(backend, row, world, grid, A, ld)
    return x, ipiv[:n].to(torch.int32), info


def _factor_panel(be, col, grid, j, jb, lc, lr2, T, A, ld, nbmin, ndiv, rfact, piv) -> int:
    """The panel's recursion and leaves on one process column; T (jb x jb,
    leading dimension jb) is the replicated top block, the local rows
    [lr2, mp) of columns [lc, lc + jb) the rest.  Fills piv[:jb] with the
    global pivot rows; returns the first zero-pivot column (1-based) or 0."""
    mp, dev = grid.mp, A.device
    state = {"info": 0}

    def leaf(jj, w):
        for k in range(jj, jj + w):
            vT, rT = be.col_argmax(T, jb, k, jb, k)
            vL, rL = be.col_argmax(A, ld, lr2, mp, lc + k)
            gT = j + rT if rT >= 0 else -1
            gL = grid.grow(rL) if rL >= 0 else -1
            rec = torch.zeros(2 + jb, dtype=torch.float64, device=dev)
            if _better(vL, gL, vT, gT):
                rec[0], rec[1] = vL, float(gL)
                rec[2:] = _block(A, ld, rL, lc, 1, jb)[:, 0]
            elif gT >= 0:
                rec[0], rec[1] = vT, float(gT)
                rec[2:] = _block(T, jb, rT, 0, 1, jb)[:, 0]
            else:
                rec[1] = -1.0
            allr = col.all_gather(rec).cpu()
            bv, bg, bi = 0.0, -1, -1
            for i in range(allr.shape[0]):
                v, g = float(allr[i, 0]), int(allr[i, 1])
                if _better(v, g, bv, bg):
                    bv, bg, bi = v, g, i
            if bg < 0:  # no row at or below the diagonal: cannot happen for j + k < n
                bv, bg, bi = 0.0, j + k, -1
            u = allr[bi, 2:].to(dev) if bi >= 0 else _block(T, jb, k, 0, 1, jb)[:, 0].clone()
            piv[k] = float(bg)
            if bv == 0.0 and not state["info"]:
                state["info"] = j + k + 1
            # The interchange of rows j + k and bg over the panel's jb columns.
            old = _block(T, jb, k, 0, 1, jb)[:, 0].clone()
            _block(T, jb, k, 0, 1, jb)[:, 0].copy_(u)
            if bg < j + jb:
                if bg != j + k:
                    _block(T, jb, bg - j, 0, 1, jb)[:, 0].copy_(old)
            elif grid.row_owner(bg) == grid.p:
                _block(A, ld, grid.lrow(bg), lc, 1, jb)[:, 0].copy_(old)
            # Scale by the pivot and the rank-1 update of the leaf's columns.
            be.col_rank1(T, jb, k + 1, jb, 0, k, jj + w, bv, u)
            be.col_rank1(A, ld, lr2, mp, lc, k, jj + w, bv, u)

    def node_update(a, k, b, w):
        """Columns [b, b + w) of the rows at and below panel row a: the top
        rows a .. a+k get U = L11^-1 (L11 the unit-lower k x k block at
        (a, a) of the replicated top block), every row below them
        -= (its columns [a, a + k)) U -- the rest of the top block and the
        local rows."""
        be.trsm_lower_unit(k, w, T, jb, a + a * jb, T, jb, a + b * jb)
        be.gemm_sub(jb - (a + k), w, k, T, jb, (a + k) + a * jb, T, jb, a + b * jb, T, jb,
                    (a + k) + b * jb)
        be.gemm_sub(mp - lr2, w, k, A, ld, lr2 + (lc + a) * ld, T, jb, a + b * jb, A, ld,
                    lr2 + (lc + b) * ld)

    def rpanel(jj, w):
        if w <= nbmin:
            leaf(jj, w)
            return
        nbs = (((w + nbmin - 1) // nbmin + ndiv - 1) // ndiv) * nbmin
        off, rem, jbs = 0, w, nbs
        while rem > 0:
            rem -= jbs
            a = jj + off
            if rfact == 2:  # right-looking: factor the piece, then update everything to its right
                rpanel(a, jbs)
                if rem > 0:
                    node_update(a, jbs, a + jbs, rem)
            else:  # left-looking / Crout: bring the piece up to date, then factor it
                if off > 0:
                    node_update(jj, off, a, jbs)
                rpanel(a, jbs)
            off += jbs
            jbs = min(rem, nbs)

    rpanel(0, jb)
    return state["info"]


def _update(be, col, grid, j, jb, pj, T, Lb, lr2, m2, ipiv, A, ld):
    """Row interchanges, U = L1^-1 (new top rows) and A22 -= L2 U on this
    process's trailing columns (global columns >= j + jb, b included)."""
    c0 = grid.lcol_from(j + jb)
    ncols = max(grid.nq - c0, 0)  # the same on every process of this column
    # The panel's interchanges as a map: perm[r] = the original row now at r.
    perm = {}
    for x in range(jb):
        r, s = j + x, int(ipiv[j + x])
        perm[r], perm[s] = perm.get(s, s), perm.get(r, r)
    src = [perm.get(j + x, j + x) for x in range(jb)]
    lows = sorted(r for r in perm if r >= j + jb and perm[r] != r)  # displaced-to rows
    rows = list(range(j, j + jb)) + lows  # every row whose trailing values change
    idx = {r: i for i, r in enumerate(rows)}
    dev = A.device
    buf = torch.zeros(len(rows) * max(ncols, 1), dtype=torch.float64, device=dev)
    if ncols > 0:
        Bv = buf.view(len(rows), ncols)
        for i, r in enumerate(rows):
            if grid.row_owner(r) == grid.p:
                Bv[i].copy_(_block(A, ld, grid.lrow(r), c0, 1, ncols)[:, 0])
    allb = col.all_gather(buf)  # every member joins, with or without trailing columns
    if ncols == 0:
        return
    old = torch.stack([allb[grid.row_owner(r)].view(len(rows), ncols)[i]
                       for i, r in enumerate(rows)])
    U = torch.stack([old[idx[src[x]]] for x in range(jb)]).T.contiguous().view(-1)  # jb x ncols
    be.trsm_lower_unit(jb, ncols, T, jb, 0, U, jb, 0)
    Uv = U.view(ncols, jb)
    if grid.p == pj:
        _block(A, ld, grid.lrow(j), c0, jb, ncols).copy_(Uv)
    for r in lows:  # an old top row lands where its pivot row came from
        if grid.row_owner(r) == grid.p:
            _block(A, ld, grid.lrow(r), c0, 1, ncols)[:, 0].copy_(old[idx[perm[r]]])
    if m2 > 0:
        be.gemm_sub(m2, ncols, jb, Lb, m2, 0, U, jb, 0, A, ld, lr2 + c0 * ld)


def _backsolve(be, row, world, grid, A, ld):
    """U x = y, y = column n after the updates; x replicated on every process."""
    n, nb, p, q = grid.n, grid.nb, grid.p, grid.q
    dev = A.device
    mp = grid.mp
    qn = grid.col_owner(n)
    yl = torch.zeros(max(mp, 1), dtype=torch.float64, device=dev)
    if q == qn and mp > 0:
        yl[:mp].copy_(_block(A, ld, 0, grid.lcol(n), mp, 1)[0])
    zn = torch.zeros(max(mp, 1), dtype=torch.float64, device=dev)  # -(sum of U x) per local row
    x = torch.zeros(max(n, 1), dtype=torch.float64, device=dev)
    xb = torch.zeros(nb, dtype=torch.float64, device=dev)
    for b in range(grid.npanels - 1, -1, -1):
        j, bw = b * nb, min(nb, n - b * nb)
        pb, qb = b % grid.P, b % grid.Q
        if p == pb:
            lr = grid.lrow(j)
            t = -zn[lr:lr + bw].clone()
            if q == qn:
                t -= yl[lr:lr + bw]
            row.all_reduce_sum(t)  # s - y over the process row
            if q == qb:
                rhs = (-t).contiguous()
                be.upper_solve(A, ld, lr + grid.lcol(j) * ld, bw, rhs, xb)
        world.broadcast(xb, grid.rank_of(pb, qb))
        x[j:j + bw] = xb[:bw]
        if q == qb and j > 0:
            m = grid.lrow_from(j)  # local rows above block b
            if m > 0:
                be.gemm_sub(m, 1, bw, A, ld, grid.lcol(j) * ld, xb, bw, 0, zn, mp, 0)
    return x[:n]


class LocalGrid2D:
    """The three communicators of each process of a P x Q grid run as threads
    of one process (rochpl_b200.grid.LocalGroup for each process row, each
    process column and the whole grid): comms(p, q) -> (row, col, world),
    the world ranks in PMAP order."""

    def __init__(self, P: int, Q: int, pmap: int = 0):
        from .grid import LocalGroup

        self.P, self.Q, self.pmap = P, Q, pmap
        self.rows = [LocalGroup(Q) for _ in range(P)]
        self.cols = [LocalGroup(P) for _ in range(Q)]
        self.world = LocalGroup(P * Q)

    def comms(self, p: int, q: int):
        rank = p * self.Q + q if self.pmap == 0 else q * self.P + p
        return self.rows[p].member(q), self.cols[q].member(p), self.world.member(rank)

    def abort(self):
        for g in self.rows + self.cols + [self.world]:
            g.barrier.abort()


def dist_comms(P: int, Q: int, pmap: int = 0):
    """(row, col, world) communicators of this process of a P x Q grid over
    torch.distributed (world size P Q; ranks on the grid in PMAP order, as
    Grid2D.coords).  Every process creates every group, in the same order."""
    import torch.distributed as dist

    from .grid import DistGroup

    rank = dist.get_rank()
    if dist.get_world_size() != P * Q:
        raise ValueError(f"a {P} x {Q} grid needs {P * Q} processes, not {dist.get_world_size()}")
    p, q = Grid2D.coords(rank, P, Q, pmap)
    at = Grid2D(0, 1, 0, 0, P, Q, pmap).rank_of
    rows = [dist.new_group([at(pp, qq) for qq in range(Q)]) for pp in range(P)]
    cols = [dist.new_group([at(pp, qq) for pp in range(P)]) for qq in range(Q)]
    return DistGroup(rows[p]), DistGroup(cols[q]), DistGroup()
