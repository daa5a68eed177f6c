"""Differentiable HPL solve: X = A^-1 B as a torch.autograd.Function.

Forward: hplb_gesv factors a column-major copy of [A | B] with the HPL panel
algorithm (partial pivoting, recursive panel, look-ahead; the same kernels as
hplb_pdgesv), B riding through the interchanges and updates as HPL's b does,
then back-solves with U for the columns of X.  The factors and pivots are
saved for the backward pass, which never refactors:

    Bbar = A^-T Xbar      hplb_getrs(trans = 1) on the stored LU and pivots
    Abar = -Bbar X^T      hplb_rank_k, one fused kernel per 64 right-hand sides

HplSolveBatch / hpl_solve_batch do the same for a whole batch of systems of
uneven size (hplb_batch_gesv forward; hplb_batch_getrs with trans = 1 and
hplb_batch_rank_k backward).

Everything runs in FP64 on the device through the C ABI (include/hplb.h); the
tensors are only the carriers of device memory.  There is no CPU path: a CPU
tensor is an error.
"""
from __future__ import annotations

import torch

from .hpl import Algo, default_ld
from .lib import HplError, library

__all__ = ["HplSolve", "hpl_solve", "HplSolveBatch", "hpl_solve_batch"]


def _colmajor(M: torch.Tensor, ld: int | None = None) -> torch.Tensor:
    """Column-major copy of a 2-D tensor: returns T (M.shape[1] x ld) with
    T[j, i] = M[i, j] for i < M.shape[0], i.e. M stored column by column with
    leading dimension ld (default M.shape[0]; rows beyond are padding).
    Always a new buffer (the solve overwrites it): for an M that is already
    column-major, M.t().contiguous() would return M's own storage."""
    ld = M.shape[0] if ld is None else ld
    out = torch.empty((M.shape[1], ld), dtype=M.dtype, device=M.device)
    out[:, : M.shape[0]].copy_(M.t())
    return out


RANK_K_MAX = 64  # right-hand sides per hplb_rank_k call


def _rank_k_chunks(lib, n: int, nrhs: int, Bc: torch.Tensor, Xc: torch.Tensor,
                   Ac: torch.Tensor) -> None:
    """Ac (n x n, column-major) = -Bbar X^T from the column-major n x nrhs
    Bbar and X held as (nrhs, n) tensors Bc and Xc: one hplb_rank_k call per
    RANK_K_MAX right-hand sides, the first storing and the rest accumulating
    (nrhs = 0: one call with k = 0, which stores zeros)."""
    for c0 in range(0, max(nrhs, 1), RANK_K_MAX):
        kc = min(RANK_K_MAX, nrhs - c0)
        lib.rank_k(n, n, kc, -1.0, Bc.data_ptr() + 8 * c0 * n, max(n, 1),
                   Xc.data_ptr() + 8 * c0 * n, max(n, 1), Ac.data_ptr(), max(n, 1),
                   accumulate=c0 > 0)


class HplSolve(torch.autograd.Function):
    """X = A^-1 B for a square FP64 CUDA A (n x n) and B (n x nrhs)."""

    @staticmethod
    def forward(ctx, A: torch.Tensor, B: torch.Tensor, nb: int = 256, nbmin: int = 32):
        if not (A.is_cuda and B.is_cuda):
            raise ValueError("hpl_solve runs on the GPU only: A and B must be CUDA tensors")
        if A.dtype != torch.float64 or B.dtype != torch.float64:
            raise ValueError("hpl_solve computes in FP64: A and B must be float64")
        if A.dim() != 2 or A.shape[0] != A.shape[1] or B.dim() != 2 or B.shape[0] != A.shape[0]:
            raise ValueError(f"shapes {tuple(A.shape)} and {tuple(B.shape)} do not form A X = B")
        n, nrhs = A.shape[0], B.shape[1]
        lib = library(A.device.index or 0)
        lib.set_stream(torch.cuda.current_stream(A.device).cuda_stream)
        nbe = max(1, min(nb, max(n, 1)))
        # The factors get HPL's padded leading dimension: a power-of-two
        # column stride (n = 16384) maps every column to the same L2 sets and
        # DRAM channels and slows the factorisation.
        ld = int(default_ld(n)) if n > 0 else 1
        # [A | B] column-major in one buffer: B takes every interchange and
        # trailing update with the factorisation (hplb_gesv), so the forward
        # needs only the back-solve with U afterwards.
        LU = torch.empty((n + nrhs, ld), dtype=torch.float64, device=A.device)
        LU[:n, :n].copy_(A.detach().t())
        LU[n:, :n].copy_(B.detach().t())
        ipiv = torch.zeros(max(n, 1), dtype=torch.int32, device=A.device)
        Xc = torch.empty((nrhs, n), dtype=torch.float64, device=A.device)
        algo = Algo(nbe, min(nbmin, nbe), 2, 2, 2, 1, 0).c()
        if nrhs > 0:
            info = lib.gesv(algo, n, nrhs, LU.data_ptr(), ld, Xc.data_ptr(), max(n, 1),
                            ipiv.data_ptr())
        else:
            info = lib.getrf(algo, n, LU.data_ptr(), ld, ipiv.data_ptr())
        if info:
            raise HplError(3, f"hpl_solve: A is singular (zero pivot in column {info})")
        ctx.save_for_backward(LU, ipiv, Xc)
        ctx.nb = nbe
        ctx.ld = ld
        return Xc.t()

    @staticmethod
    def backward(ctx, Xbar: torch.Tensor):
        LU, ipiv, Xc = ctx.saved_tensors
        n, nrhs = Xc.shape[1], Xc.shape[0]
        lib = library(LU.device.index or 0)
        lib.set_stream(torch.cuda.current_stream(LU.device).cuda_stream)
        Bc = _colmajor(Xbar.to(torch.float64))
        lib.getrs(1, n, ctx.nb, nrhs, LU.data_ptr(), ctx.ld, ipiv.data_ptr(), Bc.data_ptr(),
                  max(n, 1))
        gA = None
        if ctx.needs_input_grad[0]:
            Ac = torch.empty(n, n, dtype=torch.float64, device=LU.device)
            _rank_k_chunks(lib, n, nrhs, Bc, Xc, Ac)
            gA = Ac.t()
        gB = Bc.t() if ctx.needs_input_grad[1] else None
        return gA, gB, None, None


def hpl_solve(A: torch.Tensor, B: torch.Tensor, nb: int = 256, nbmin: int = 32) -> torch.Tensor:
    """X = A^-1 B, differentiable in A and B.  A 1-D B is one right-hand side."""
    if B.dim() == 1:
        return HplSolve.apply(A, B.unsqueeze(1), nb, nbmin).squeeze(1)
    return HplSolve.apply(A, B, nb, nbmin)


class HplSolveBatch(torch.autograd.Function):
    """X_i = A_i^-1 B_i for every system of a BatchPlan, on packed pools (the
    plan's A and B layouts, 1-D FP64 CUDA tensors).  Forward: one batched
    factor-and-solve launch; the factors and pivots are saved.  Backward:
    Bbar_i = A_i^-T Xbar_i by the batched transposed solve on the stored
    factors, Abar_i = -Bbar_i X_i^T by the batched rank-k kernel."""

    @staticmethod
    def forward(ctx, plan, A_pool: torch.Tensor, B_pool: torch.Tensor):
        if not (A_pool.is_cuda and B_pool.is_cuda):
            raise ValueError("hpl_solve_batch runs on the GPU only")
        if A_pool.dtype != torch.float64 or B_pool.dtype != torch.float64:
            raise ValueError("hpl_solve_batch computes in FP64")
        if A_pool.numel() != plan.a_elems or B_pool.numel() != plan.b_elems:
            raise ValueError("pool sizes do not match the plan's layout")
        lib = plan.lib
        lib.set_stream(torch.cuda.current_stream(A_pool.device).cuda_stream)
        LU = A_pool.detach().clone()
        X = B_pool.detach().clone()
        ipiv = torch.zeros(max(plan.p_elems, 1), dtype=torch.int32, device=A_pool.device)
        info = torch.zeros(max(plan.count, 1), dtype=torch.int32, device=A_pool.device)
        plan.gesv(LU.data_ptr(), X.data_ptr(), ipiv.data_ptr(), info.data_ptr())
        bad = int(info.max()) if plan.count else 0
        if bad:
            raise HplError(3, f"hpl_solve_batch: a system is singular (zero pivot, column {bad})")
        ctx.plan = plan
        ctx.save_for_backward(LU, ipiv, X)
        return X

    @staticmethod
    def backward(ctx, Xbar: torch.Tensor):
        LU, ipiv, X = ctx.saved_tensors
        plan = ctx.plan
        plan.lib.set_stream(torch.cuda.current_stream(LU.device).cuda_stream)
        Bbar = Xbar.to(torch.float64).contiguous().clone()
        plan.getrs(1, LU.data_ptr(), ipiv.data_ptr(), Bbar.data_ptr())
        gA = None
        if ctx.needs_input_grad[1]:
            gA = torch.empty(plan.a_elems, dtype=torch.float64, device=LU.device)
            plan.rank_k(-1.0, Bbar.data_ptr(), X.data_ptr(), gA.data_ptr())
        return None, gA, (Bbar if ctx.needs_input_grad[2] else None)


def pack_batch(plan, mats, pool_elems: int, offsets) -> torch.Tensor:
    """Pack square or tall matrices (list of 2-D tensors) into a plan pool,
    column-major, at the plan's offsets.  Differentiable."""
    parts = []
    for M in mats:
        parts.append(M.t().reshape(-1))
    out = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.float64)
    if out.numel() != pool_elems:
        raise ValueError("matrices do not match the plan's layout")
    return out


def unpack_batch(plan, pool: torch.Tensor, rows, cols, offsets):
    """Views of the systems' matrices (rows[i] x cols[i]) in a pool."""
    return [pool[int(o):int(o) + int(r) * int(c)].view(int(c), int(r)).t()
            for o, r, c in zip(offsets, rows, cols)]


def hpl_solve_batch(plan, As, Bs):
    """X_i = A_i^-1 B_i for lists of FP64 CUDA matrices matching the plan's
    sizes; differentiable in every A_i and B_i.  Returns the list of X_i."""
    A_pool = pack_batch(plan, As, plan.a_elems, plan.a_off)
    B_pool = pack_batch(plan, Bs, plan.b_elems, plan.b_off)
    X = HplSolveBatch.apply(plan, A_pool, B_pool)
    return unpack_batch(plan, X, plan.n, plan.nrhs, plan.b_off)
