"""Small, self-contained GPU cases for profiling one kernel at a time.

    python -m rochpl_b200.profile_cases dgemm 8192        # 3 x hplb_dgemm_sub, 8192^2 x 512
    python -m rochpl_b200.profile_cases solve 16384 512   # one hplb_pdgesv (N, NB)
    python -m rochpl_b200.profile_cases gemm_lp 8192 1536 # 13 x hplb_gemm_lp_sub (FP16), 8192^2 x k
    python -m rochpl_b200.profile_cases getrf 16384 512   # one hplb_getrf (the leaves, the panel)
    python -m rochpl_b200.profile_cases mixed 131072 3    # hplb_pdgesv_mixed (N, precision), with
                                                          # a per-kernel breakdown from CUPTI tracing
    python -m rochpl_b200.profile_cases batch 1024 16     # 592 systems of one size (N, NB), nrhs 16
                                                          # (NB 64: the recursive factorisation)

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


def gemm_lp(mn: int = 8192, k: int = 1536, reps: int = 13) -> None:
    import torch

    from . import library

    lib = library(0)
    m = n = mn
    A = (torch.rand(m, k, device="cuda") - 0.5).to(torch.float16)
    B = (torch.rand(n, k, device="cuda") - 0.5).to(torch.float16)
    sA = torch.ones((m + 127) // 128, device="cuda")
    sB = torch.ones((n + 255) // 256, device="cuda")
    C = torch.zeros(n, m, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(reps):
        if i == 3:
            torch.cuda.synchronize()
            e0.record()
        lib.gemm_lp_sub(False, m, n, k, A.data_ptr(), k, B.data_ptr(), k, sA.data_ptr(),
                        sB.data_ptr(), C.data_ptr(), m)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (reps - 3)
    print(f"gemm_lp {m}x{n}x{k}: {ms:.3f} ms, {2.0 * m * n * k / ms / 1e9:.1f} TFLOP/s")


def getrf(n: int, nb: int = 512) -> None:
    import torch

    from . import library
    from .hpl import Algo

    lib = library(0)
    A = torch.empty(n * n, dtype=torch.float64, device="cuda")
    lib.matgen(n, n, 100, A.data_ptr(), n)
    ip = torch.zeros(n, dtype=torch.int32, device="cuda")
    lib.getrf(Algo(nb=nb).c(), n, A.data_ptr(), n, ip.data_ptr())
    t = lib.last_timing()
    print(f"getrf N={n} NB={nb}: {t['total_ms']:.1f} ms (panels {t['panel_ms']:.1f} ms)")


def mixed(n: int, precision: int = 3) -> None:
    import collections

    import torch
    from torch.profiler import ProfilerActivity, profile

    from . import library
    from .hpl import Algo

    lib = library(0)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    lib.pdgesv_mixed(Algo(nb=512).c(), n, x.data_ptr(), seed=100, precision=precision)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        r = lib.pdgesv_mixed(Algo(nb=512).c(), n, x.data_ptr(), seed=100, precision=precision)
        torch.cuda.synchronize()
    print({k: round(v, 2) if isinstance(v, float) else v for k, v in r.items()})
    agg = collections.defaultdict(lambda: [0.0, 0])
    for e in prof.events():
        if e.device_type.name != "CUDA":
            continue
        name = e.name.replace("void ", "").replace("hplb::(anonymous namespace)::", "")
        name = name.split("(")[0][:48]
        agg[name][0] += (e.time_range.end - e.time_range.start) / 1e3
        agg[name][1] += 1
    for name, (ms, cnt) in sorted(agg.items(), key=lambda kv: -kv[1][0])[:24]:
        print(f"{name:50s} {ms:10.1f} ms {cnt:7d}")


def batch(n: int, nb: int = 16, nrhs: int = 16) -> None:
    import numpy as np
    import torch

    from . import library
    from .batch import BatchPlan

    lib = library(0)
    plan = BatchPlan(lib, np.full(148 * 4, n, dtype=np.int32), nrhs, [nb] * 6)
    dA = torch.zeros(plan.a_elems, dtype=torch.float64, device="cuda")
    dB = torch.zeros(plan.b_elems, dtype=torch.float64, device="cuda")
    dP = torch.zeros(plan.p_elems, dtype=torch.int32, device="cuda")
    dI = torch.zeros(plan.count, dtype=torch.int32, device="cuda")
    seeds = np.arange(plan.count, dtype=np.uint64)
    for _ in range(3):
        plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())
        plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    print(f"batch {plan.count} x N={n} NB={int(plan.nb[0])}: {plan.last_ms:.2f} ms, "
          f"{plan.flops() / plan.last_ms / 1e9:.2f} TFLOP/s")


if __name__ == "__main__":
    case = sys.argv[1]
    args = [int(a) for a in sys.argv[2:]]
    {"dgemm": dgemm, "solve": solve, "gemm_lp": gemm_lp, "getrf": getrf, "mixed": mixed,
     "batch": batch}[case](*args)
