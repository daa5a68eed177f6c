"""Small, self-contained GPU cases for profiling one kernel at a time.

    python -m rochpl_b200.profile_cases dgemm 8192        # 3 x hplb_dgemm_sub, 8192^2 x 512
    python -m rochpl_b200.profile_cases solve 16384 512   # one hplb_pdgesv (N, NB)

Each case prints its event-timed rate, so the same command can be run plainly
before it is run under a profiler.
"""
from __future__ import annotations

import sys
import time


def dgemm(m: int, k: int = 512, reps: int = 3) -> None:
    import torch

    from . import library

    lib = library(0)
    n = m
    A = torch.randn(m * k, dtype=torch.float64, device="cuda")
    B = torch.randn(k * n, dtype=torch.float64, device="cuda")
    C = torch.randn(m * n, dtype=torch.float64, device="cuda")
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        lib.dgemm_sub(m, n, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        print(f"dgemm_sub {m}x{n}x{k}: {2.0 * m * n * k / dt / 1e12:.2f} TFLOP/s")


def solve(n: int, nb: int = 512) -> None:
    from .hpl import Algo, HPL_pdtest

    r = HPL_pdtest(Algo(nb=nb), n, lib_fused_residual=True)
    print(f"solve N={n} NB={nb}: {r['gflops'] / 1e3:.2f} TFLOP/s resid={r['resid']:.3e}")


if __name__ == "__main__":
    case = sys.argv[1]
    args = [int(a) for a in sys.argv[2:]]
    {"dgemm": dgemm, "solve": solve}[case](*args)
