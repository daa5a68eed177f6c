"""Differentiable HPL solve: X = A^-1 B as a torch.autograd.Function.

Forward: hplb_getrf factors a column-major copy of A with the HPL panel
algorithm (partial pivoting, recursive panel, look-ahead; the same kernels as
hplb_pdgesv), then hplb_getrs solves for the columns of B.  The factors and
pivots are saved for the backward pass, which never refactors:

    Bbar = A^-T Xbar      hplb_getrs(trans = 1) on the stored LU and pivots
    Abar = -Bbar X^T      hplb_rank_k, one fused rank-nrhs kernel

Everything runs in FP64 on the device through the C ABI (include/hplb.h); the
tensors are only the carriers of device memory.  There is no CPU path: a CPU
tensor is an error.
"""
from __future__ import annotations

import torch

from .hpl import Algo
from .lib import HplError, library

__all__ = ["HplSolve", "hpl_solve"]


def _colmajor(M: torch.Tensor) -> torch.Tensor:
    """Column-major copy of a 2-D tensor: returns T with T[j, i] = M[i, j],
    i.e. M stored column by column with leading dimension M.shape[0].  Always
    a new buffer (the solve overwrites it): for an M that is already
    column-major, M.t().contiguous() would return M's own storage."""
    out = torch.empty((M.shape[1], M.shape[0]), dtype=M.dtype, device=M.device)
    out.copy_(M.t())
    return out


class HplSolve(torch.autograd.Function):
    """X = A^-1 B for a square FP64 CUDA A (n x n) and B (n x nrhs, nrhs <= 64
    for the adjoint's fused rank-k kernel)."""

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
        LU = _colmajor(A.detach())
        ipiv = torch.zeros(max(n, 1), dtype=torch.int32, device=A.device)
        info = lib.getrf(Algo(nbe, min(nbmin, nbe), 2, 2, 2, 1, 0).c(), n, LU.data_ptr(),
                         max(n, 1), ipiv.data_ptr())
        if info:
            raise HplError(3, f"hpl_solve: A is singular (zero pivot in column {info})")
        Xc = _colmajor(B.detach())
        lib.getrs(0, n, nbe, nrhs, LU.data_ptr(), max(n, 1), ipiv.data_ptr(), Xc.data_ptr(),
                  max(n, 1))
        ctx.save_for_backward(LU, ipiv, Xc)
        ctx.nb = nbe
        return Xc.t()

    @staticmethod
    def backward(ctx, Xbar: torch.Tensor):
        LU, ipiv, Xc = ctx.saved_tensors
        n, nrhs = Xc.shape[1], Xc.shape[0]
        lib = library(LU.device.index or 0)
        lib.set_stream(torch.cuda.current_stream(LU.device).cuda_stream)
        Bc = _colmajor(Xbar.to(torch.float64))
        lib.getrs(1, n, ctx.nb, nrhs, LU.data_ptr(), max(n, 1), ipiv.data_ptr(), Bc.data_ptr(),
                  max(n, 1))
        gA = None
        if ctx.needs_input_grad[0]:
            if nrhs > 64:
                raise HplError(6, "hpl_solve backward: the fused rank-k kernel takes <= 64 RHS")
            Ac = torch.empty(n, n, dtype=torch.float64, device=LU.device)
            lib.rank_k(n, n, nrhs, -1.0, Bc.data_ptr(), max(n, 1), Xc.data_ptr(), max(n, 1),
                       Ac.data_ptr(), max(n, 1))
            gA = Ac.t()
        gB = Bc.t() if ctx.needs_input_grad[1] else None
        return gA, gB, None, None


def hpl_solve(A: torch.Tensor, B: torch.Tensor, nb: int = 256, nbmin: int = 32) -> torch.Tensor:
    """X = A^-1 B, differentiable in A and B.  A 1-D B is one right-hand side."""
    if B.dim() == 1:
        return HplSolve.apply(A, B.unsqueeze(1), nb, nbmin).squeeze(1)
    return HplSolve.apply(A, B, nb, nbmin)
