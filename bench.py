"""HPL benchmark: FP64 solve throughput on B200 (TFLOP/s, 2/3 N^3 + 2 N^2).

Default workload: N = 131072, NB = 512, NBMIN = 32, NDIV = 2, right-looking
recursion and leaf, look-ahead depth 1, seed 100 -- the plain FP64 HPL at
near-full HBM on one B200 (the [A|b] matrix is 137.5 GB, far larger than L2).

A step is one HPL_pdgesv (LU + back-solve), the region rocHPL times
(src/HPL_pdtest.cpp:132-134); [A|b] is regenerated from the LCG before every
step, outside the timed region, as rocHPL does before each of its `-it`
repeats.  Timing is CUDA events on the launching streams, max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Before the timed steps the generated N = 131072 [A|b] is checked bit for bit
against the oracle's LCG (sampled entries over the whole matrix, column b and
the last 512-column block, LCG state indices up to 1.7e10) and, for seed 100,
against the reference generator's hashes in tests/golden/lcg_c2_golden.json.
After them: the HPL config of N = 4096, NB = 256 ("c1"), and a parity solve at
N = 16384, NB = 512 against the oracle's own solve of the same system (pivot
divergences by column, x error against 64 N eps kappa; "parity").

After the FP64 steps the same system is solved in the mixed-precision form
(16-bit tensor-core LU, BF16 x3 and FP16 x3, + FP64 GMRES refinement to the
same residual threshold); its time to solution, speed-up over the FP64 solve,
iteration counts and distance to the FP64 x go under "mixed" in the line; the
same at N = 32768 and 65536 against FP64 solves of those systems
("mixed.by_n").

Then the batched form (4096 LCG systems, N log-uniform in [32, 1024], nrhs
1 / 16 / 64, one persistent graph-captured launch each) and the
differentiable solve (N = 16384 with 32 RHS, forward and backward; 256
systems with N in [64, 512] through the batched form) go under "batched" and
"autograd" (the N = 16384 gradients are checked against torch's FP64 solve
and against central differences with step 1e-6).

Multi-GPU runs are replicas for the headline (each rank solves its own system,
reported as weak scaling); with --gpus N > 1 a further leg ("grid") solves ONE
N = 131072 system across all N GPUs on a 1 x N process grid (strong scaling).

--impl reference times the reference algorithm's CPU restatement (the oracle,
host OpenBLAS on every host core): N = 16384 on every step and N = 32768 once,
then the N = 131072 time extrapolated from the N = 32768 point as N^3 (the host
cannot hold the 137.5 GB matrix beside the run, and one host solve of it would
take about an hour).

--case NAME runs one small kernel case for profiling and prints its event-timed
rate (dgemm, solve, gemm_lp, getrf, mixed, batch; sizes from --n / --nb / --k /
--prec / --nrhs), so the same command can run plainly before it runs under ncu.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HPL TFLOP/s at N=131072: FP64 LU vs BF16 LU+IR at same residual; % of peak"

# DRAM bytes per algorithmic flop of the trailing-update DGEMM, from an ncu
# capture of one 8192 x 8192 x 512 launch (profiles/dgemm_tma_kernel_8192x8192x512.md):
# (718.5 + 498.3) MB over 68.7 GFLOP.  Its traffic scales with the C-tile count,
# i.e. with the flops at k = 512, so bench lines scale it to their own launches.
DGEMM_DRAM_BYTES_PER_FLOP = 1216.8e6 / (2.0 * 8192 * 8192 * 512)
UNIT = "TFLOP/s"


def hpl_flops(n: int) -> float:
    return 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="hplb_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        loaded = [s for s, p in zip(sm, power) if p > 200] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port with host OpenBLAS
# ---------------------------------------------------------------------------

def host_info() -> dict:
    """CPU model, logical cores and RAM of this host."""
    model, ram = None, None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
        for line in open("/proc/meminfo"):
            if line.startswith("MemTotal:"):
                ram = int(line.split()[1]) * 1024 / 1e9
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count(), "ram_gb": ram}


def oracle_solve(n: int, nb: int, seed: int = 100):
    """One host solve by the oracle (generate, LU, back-solve, check), OpenBLAS
    level 3 on every host core.  Returns (seconds, x, ipiv, resid, blas)."""
    from oracle import oracle as O

    O.lib()
    have_blas = O.use_blas(os.cpu_count())
    t0 = time.perf_counter()
    x, ipiv, info, resid = O.hpl_test(n, nb, 32, 2, seed=seed)
    return time.perf_counter() - t0, x, ipiv, resid, have_blas


def cpu_baseline(n: int, nb: int) -> tuple[dict, object, object]:
    t, x, ipiv, resid, have_blas = oracle_solve(n, nb)
    cb = {"value": hpl_flops(n) / t / 1e12, "unit": UNIT, "cores": os.cpu_count(),
          "kind": "port",
          "sample": f"N={n} NB={nb} NBMIN=32 NDIV=2 R/R seed 100, generate+LU+back-solve+check "
                    f"on the host, {'OpenBLAS' if have_blas else 'scalar'} level-3, "
                    f"{os.cpu_count()} threads; value = (2/3N^3+2N^2)/t",
          "resid": resid, "seconds": t, "host": host_info()}
    return cb, x, ipiv


def run_reference(args):
    """The reference algorithm (its CPU restatement) on the host cores: N =
    cpu_n on every step, N = cpu_n_big once, and the rate at N = args.n
    extrapolated from the largest measured point with t proportional to N^3."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    n_step, n_big, target = args.cpu_n, args.cpu_n_big, args.n
    for _ in range(args.warmup):
        oracle_solve(max(256, n_step // 4), args.nb)
    steps = []
    for _ in range(args.steps):
        t, _x, _p, resid, have_blas = oracle_solve(n_step, args.nb)
        steps.append((t, resid))
    t_step = statistics.median(t for t, _ in steps)
    points = [{"n": n_step, "seconds": t_step, "tflops": hpl_flops(n_step) / t_step / 1e12,
               "steps": args.steps, "resid_max": max(r for _, r in steps)}]
    base_n, base_t = n_step, t_step
    if n_big > n_step:
        t, _x, _p, resid, _b = oracle_solve(n_big, args.nb)
        points.append({"n": n_big, "seconds": t, "tflops": hpl_flops(n_big) / t / 1e12,
                       "steps": 1, "resid_max": resid})
        base_n, base_t = n_big, t
    t_target = base_t * hpl_flops(target) / hpl_flops(base_n)
    v = hpl_flops(target) / t_target / 1e12
    extrapolated = target != base_n
    cb = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
          "sample": (f"N={n_step} x {args.steps} steps" +
                     (f" and N={n_big} once" if n_big > n_step else "") +
                     f", NB={args.nb} NBMIN=32 NDIV=2 R/R seed 100, generate+LU+back-solve+check "
                     f"on the host, {'OpenBLAS' if have_blas else 'scalar'} level-3, "
                     f"{os.cpu_count()} threads" +
                     (f"; N={target} extrapolated from N={base_n} as N^3" if extrapolated else "")),
          "resid": max(p["resid_max"] for p in points), "host": host_info(),
          "measured_points": points}
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_target * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (HPL LCG, seed 100)",
        "config": {"workload": f"HPL FP64 solve N={target} NB={args.nb} NBMIN=32 NDIV=2 "
                               f"PFACT=R RFACT=R depth 1 on the host cores" +
                               (f" (extrapolated as N^3 from measured N={base_n})"
                                if extrapolated else ""),
                   "n": target, "nb": args.nb, "extrapolated": extrapolated,
                   "measured_points": points, "parallelism": "host threads"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch

    from rochpl_b200 import library
    from rochpl_b200.hpl import Algo, default_ld

    from rochpl_b200.ranks import Ranks

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    ranks = Ranks("nccl", timeout_s=1800)
    barrier, max_over_ranks = ranks.barrier, ranks.max

    lib = library(local)
    n, nb = args.n, args.nb
    algo = Algo(nb, 32, 2, 2, 2, 1, 0)
    ld = default_ld(n)
    seed = 100 + rank  # each replica its own system
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP = torch.zeros(n, dtype=torch.int32, device="cuda")

    dmma_peak, dfma_peak = lib.fp64_peak(20000)
    lcg = None if args.no_parity else lcg_check(lib, dA, n, ld, seed, nb)

    def step():
        lib.matgen(n, n + 1, seed, dA.data_ptr(), ld, nb)  # outside the timed region
        torch.cuda.synchronize()
        barrier()
        lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr(), dP.data_ptr())
        torch.cuda.synchronize()
        return lib.last_timing()

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    clocks.start()
    timings = [step() for _ in range(args.steps)]
    clk = clocks.stop()
    barrier()

    solve_ms = sum(t["total_ms"] for t in timings) / len(timings)
    solve_ms_max = max_over_ranks(solve_ms)
    value = world * hpl_flops(n) / (solve_ms_max * 1e-3) / 1e12
    gemm_ms = sum(t["gemm_ms"] for t in timings)
    gemm_flops = sum(t["gemm_flops"] for t in timings)
    gemm_launches = sum(t["gemm_launches"] for t in timings)
    gemm_tf = gemm_flops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else 0.0
    launches = sum(t["kernel_launches"] for t in timings)

    res = lib.residual_lcg(n, seed, dX.data_ptr())

    # End to end through the C ABI with host buffers: [A|b] uploaded from
    # pinned host memory, solve, x read back -- all inside the timed region.
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(lib, algo, n, ld, seed, dA, dX, barrier, max_over_ranks, world)

    # The HPL config N = 4096 (the reference's CPU-runnable case) and the
    # parity solve against the oracle: rank 0, outside every timed region.
    c1 = parity = cb = None
    if rank == 0 and not args.no_c1:
        c1 = c1_leg(lib, dmma_peak)
    if rank == 0 and not (args.no_cpu_baseline and args.no_parity):
        cb, xo, po = cpu_baseline(args.cpu_n, nb)
        if not args.no_parity:
            parity = {"lcg": lcg, "solve": parity_leg(lib, args.cpu_n, nb, xo, po)}
        if args.no_cpu_baseline:
            cb = None

    mixed = None
    if not args.no_mixed:
        x64 = dX.double().cpu().numpy()
        dA = None  # the FP64 [A|b] cannot stay beside the FP32 factors at this N
        torch.cuda.empty_cache()
        mixed = mixed_leg(lib, algo, n, seed, x64, solve_ms, args, barrier, max_over_ranks)
        if args.mixed_sizes:
            mixed["by_n"] = mixed_sizes_leg(lib, args, seed, barrier, max_over_ranks)

    grid = None
    if world > 1 and not args.no_grid:
        dA = None
        torch.cuda.empty_cache()
        grid = grid_leg(lib, args, ranks)

    batched = None if args.no_batched else batched_leg(lib, args, ranks)
    autograd = None if args.no_autograd else autograd_leg(lib, args, max_over_ranks)

    if rank == 0:
        peak = dmma_peak
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": solve_ms_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (HPL LCG matrix, seed 100 + rank, entries in (-0.5, 0.5])",
            "config": {"workload": f"HPL FP64 solve N={n} NB={nb} NBMIN=32 NDIV=2 "
                                   "PFACT=R RFACT=R depth 1, P=Q=1 per GPU",
                       "n": n, "nb": nb, "nbmin": 32, "ndiv": 2,
                       "l2": "inputs larger than L2 ([A|b] is %.1f GB)" % (ld * (n + 1) * 8 / 1e9),
                       "parallelism": f"replicas x{world}"},
            "frac_of_fp64_peak": value / world / peak,
            "resid": res["resid"], "resid_passed": res["resid"] < 16.0,
            "gflops_reference_formula": world * (2 / 3 * n ** 3 + 1.5 * n ** 2)
            / (solve_ms_max * 1e-3) / 1e9,
            "roofline": {"kernel": "dgemm_tma_kernel (trailing-update DMMA DGEMM, TMA-fed)",
                         "bound": "tensor", "achieved": gemm_tf, "peak": peak, "unit": "TFLOP/s",
                         "frac": gemm_tf / peak,
                         "traffic": (args.gemm_traffic if args.gemm_traffic is not None else
                                     DGEMM_DRAM_BYTES_PER_FLOP * gemm_flops / max(gemm_launches, 1)),
                         "traffic_note": "DRAM bytes per DGEMM launch, from the ncu capture in "
                                         "profiles/ scaled by each launch's flops",
                         "peak_source": "FP64 DMMA m16n8k8 issue rate measured live by "
                                        "hplb_fp64_peak (MEASURED_PEAKS.json has no FP64 figure)",
                         "gemm_share_of_solve": gemm_ms / sum(t["total_ms"] for t in timings),
                         "gemm_launches": gemm_launches},
            "fp64_probe": {"dmma_tflops": dmma_peak, "dfma_tflops": dfma_peak},
            "clocks": clk,
            "gpu_launches": launches,
            "timing_ms": {k: statistics.mean(t[k] for t in timings)
                          for k in ("total_ms", "lu_ms", "trsv_ms", "gemm_ms", "panel_ms")},
        }
        if e2e is not None:
            line["e2e"] = e2e
        if mixed is not None:
            line["mixed"] = mixed
        if grid is not None:
            line["grid"] = grid
        if batched is not None:
            line["batched"] = batched
        if autograd is not None:
            line["autograd"] = autograd
        if cb is not None:
            line["cpu_baseline"] = cb
        if c1 is not None:
            line["c1"] = c1
        if parity is not None:
            line["parity"] = parity
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def lcg_check(lib, dA, n, ld, seed, nb, samples=100000) -> dict:
    """The generated [A|b] against the oracle's LCG, bit for bit: `samples`
    entries drawn over the whole matrix, column b and the last 512-column
    block (state indices up to n^2 + n, past 2^32 at N = 131072), and for seed
    100 the reference generator's block hashes from tests/golden/."""
    import numpy as np
    import torch

    from oracle import oracle as O

    lib.matgen(n, n + 1, seed, dA.data_ptr(), ld, nb)
    torch.cuda.synchronize()
    cols = dA.view(n + 1, ld)  # row j of this view is column j of [A|b]
    rng = np.random.default_rng(seed)
    ii = rng.integers(0, n, samples)
    jj = rng.integers(0, n + 1, samples)
    ii[:2], jj[:2] = (0, n - 1), (0, n)
    got = dA[torch.from_numpy(ii + jj * ld).cuda()].cpu().numpy()
    ref = np.array([O.lcg_value(O.lcg_state(seed, n, int(i), int(j))) for i, j in zip(ii, jj)])
    bad = int(np.count_nonzero(got.view(np.uint64) != ref.view(np.uint64)))
    w = min(512, n)
    blocks = {"column b": (n, 1), "last column block": (n - w, w)}
    gold_path = os.path.join(ROOT, "tests", "golden", "lcg_c2_golden.json")
    golden = None
    if seed == 100 and os.path.exists(gold_path):
        g = json.load(open(gold_path))
        if g["n"] == n:
            golden = {b["name"]: b for b in g["blocks"]}
            for b in g["blocks"]:
                blocks[b["name"]] = (b["col0"], b["ncols"])
    out = {"entries_sampled": samples, "sample_mismatches": bad,
           "max_state_index": n * (n + 1), "blocks": {}}
    for name, (c0, wc) in blocks.items():
        A = np.ascontiguousarray(cols[c0:c0 + wc, :n].cpu().numpy()).T  # n x wc, Fortran order
        ref_b = O.matgen_block(n, 0, c0, n, wc, seed)
        ok = bool(np.array_equal(A.view(np.uint64), ref_b.view(np.uint64)))
        rec = {"col0": c0, "ncols": wc, "bit_exact_vs_oracle": ok}
        if golden and name in golden:
            rec["fnv1a"] = f"{O.hash_block(A, n, wc):016x}"
            rec["matches_reference_generator"] = rec["fnv1a"] == golden[name]["fnv1a"]
        out["blocks"][name] = rec
        bad += 0 if ok else 1
    out["bit_exact"] = bad == 0 and all(b.get("matches_reference_generator", True)
                                       for b in out["blocks"].values())
    return out


def parity_leg(lib, n, nb, xo, po, seed=100) -> dict:
    """The GPU solve of the system the oracle just solved on the host (N = n,
    seed 100): pivot divergences by column, ||x - x_oracle||oo / ||x_oracle||oo
    against 64 n eps kappa_oo (kappa from an FP64 inverse on the device, a
    check only), and the HPL residual."""
    import numpy as np
    import torch

    from rochpl_b200.hpl import Algo, default_ld

    ld = default_ld(n)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    dP = torch.zeros(n, dtype=torch.int32, device="cuda")
    lib.matgen(n, n + 1, seed, dA.data_ptr(), ld, nb)
    A = dA.view(n + 1, ld)[:n, :n].t()
    anorm = float(A.abs().sum(dim=1).max())
    ainv = torch.linalg.inv(A)
    kappa = anorm * float(ainv.abs().sum(dim=1).max())
    del ainv, A
    torch.cuda.empty_cache()
    lib.pdgesv(Algo(nb, 32, 2, 2, 2, 1, 0).c(), n, dA.data_ptr(), ld, dX.data_ptr(), dP.data_ptr())
    x, ipiv = dX.cpu().numpy(), dP.cpu().numpy()
    div = np.nonzero(ipiv != np.asarray(po))[0]
    err = float(np.max(np.abs(x - xo)) / np.max(np.abs(xo)))
    tol = 64 * n * 2.0 ** -53 * kappa
    res = lib.residual_lcg(n, seed, dX.data_ptr())
    return {"n": n, "nb": nb, "seed": seed, "pivot_divergences": int(div.size),
            "first_divergent_column": int(div[0]) if div.size else None,
            "x_rel_err_vs_oracle": err, "x_tolerance": tol, "kappa_inf": kappa,
            "x_within_tolerance": err <= tol, "resid": res["resid"],
            "note": "oracle = the C restatement of the reference algorithm on the host "
                    "(OpenBLAS level 3); tolerance 64 N eps kappa_oo"}


def c1_leg(lib, peak, steps=10, warmup=3) -> dict:
    """The HPL config N = 4096, NB = 256, NBMIN = 32, NDIV = 2, R/R, depth 1,
    seed 100: per-solve device time (median of `steps`), rate, residual."""
    import torch

    from rochpl_b200.hpl import Algo, default_ld

    n, nb = 4096, 256
    ld = default_ld(n)
    algo = Algo(nb, 32, 2, 2, 2, 1, 0)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    ts = []
    for it in range(warmup + steps):
        lib.matgen(n, n + 1, 100, dA.data_ptr(), ld, nb)
        lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr())
        if it >= warmup:
            ts.append(lib.last_timing())
    ms = statistics.median(t["total_ms"] for t in ts)
    res = lib.residual_lcg(n, 100, dX.data_ptr())
    v = hpl_flops(n) / (ms * 1e-3) / 1e12
    return {"workload": "HPL FP64 solve N=4096 NB=256 NBMIN=32 NDIV=2 PFACT=R RFACT=R depth 1, "
                        "seed 100", "ms_per_solve": ms, "value": v, "unit": UNIT,
            "frac_of_fp64_peak": v / peak, "resid": res["resid"], "resid_passed": res["resid"] < 16,
            "steps": steps,
            "breakdown_ms": {k: statistics.median(t[k] for t in ts)
                             for k in ("lu_ms", "trsv_ms", "gemm_ms", "panel_ms")}}


def _measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def mixed_one(lib, algo, n, seed, prec, x64, fp64_ms, steps, warmup, barrier, max_over_ranks,
              bf16_peak) -> dict:
    """One precision of the mixed-precision form: low-precision LU + GMRES
    refinement to the HPL residual threshold on the LCG system of `seed`,
    timed on the device (first to last event of hplb_pdgesv_mixed), against
    the FP64 solve of the same system (time fp64_ms, solution x64)."""
    import numpy as np
    import torch

    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    for _ in range(warmup):
        lib.pdgesv_mixed(algo.c(), n, dX.data_ptr(), seed=seed, precision=prec)
    reps = []
    for _ in range(steps):
        torch.cuda.synchronize()
        barrier()
        reps.append(lib.pdgesv_mixed(algo.c(), n, dX.data_ptr(), seed=seed, precision=prec))
    tm = lib.last_timing()
    ms = max_over_ranks(statistics.mean(r["total_ms"] for r in reps))
    r = reps[-1]
    chk = lib.residual_lcg(n, seed, dX.data_ptr())
    x = dX.cpu().numpy()
    gemm_tf = r["gemm_flops"] / (r["gemm_ms"] * 1e-3) / 1e12 if r["gemm_ms"] > 0 else 0.0
    return {
        "time_to_solution_ms": ms, "speedup_vs_fp64": fp64_ms / ms,
        "value": hpl_flops(n) / (ms * 1e-3) / 1e12, "unit": UNIT,
        "converged": bool(r["converged"]), "resid": chk["resid"],
        "resid_passed": chk["resid"] < 16.0, "resid_lu_only": r["resid_lu"],
        "outer_iters": r["outer_iters"], "gmres_iters": r["gmres_iters"],
        "rel_err_vs_fp64_x": float(np.max(np.abs(x - x64)) / np.max(np.abs(x64))),
        "lu_ms": r["lu_ms"], "ir_ms": r["ir_ms"], "panel_ms": r["panel_ms"],
        "roofline": {"kernel": "gemm_lp_kernel (tcgen05 16-bit trailing update" +
                               (", x3 split)" if prec >= 2 else ")"),
                     "bound": "tensor", "achieved": gemm_tf, "peak": bf16_peak,
                     "unit": "TFLOP/s", "frac": gemm_tf / bf16_peak,
                     "gemm_ms": r["gemm_ms"], "gemm_flops": r["gemm_flops"]},
        "gpu_launches": tm["kernel_launches"], "steps": steps,
    }


def _bf16_peak():
    peaks = _measured_peaks()
    if peaks.get("bf16_tflops_sustained"):
        return peaks["bf16_tflops_sustained"], "MEASURED_PEAKS.json bf16_tflops_sustained"
    return 1394.6, "fallback 1394.6"


MIXED_NOTE = ("time to HPL scaled residual < 16 (target 16.0); value = (2/3N^3+2N^2)/t, the "
              "HPL-equivalent rate; speedup = FP64 solve time / mixed time; GMRES-IR in FP64, "
              "A regenerated from the LCG for r = b - Ax")


def mixed_leg(lib, algo, n, seed, x64, fp64_ms, args, barrier, max_over_ranks):
    """The mixed-precision form on the system of the FP64 steps (BF16 x3 and
    FP16 x3), against the FP64 solve just timed.  A is regenerated from the LCG
    for r = b - A x (bit-identical to the stored FP64 A, which does not fit in
    HBM beside the FP32 factors at N = 131072)."""
    from rochpl_b200.lib import PREC_BF16X3, PREC_FP16X3

    peak, src = _bf16_peak()
    out = {"note": MIXED_NOTE, "bf16_peak_tflops": peak, "bf16_peak_source": src}
    for name, prec in (("bf16x3", PREC_BF16X3), ("fp16x3", PREC_FP16X3)):
        out[name] = mixed_one(lib, algo, n, seed, prec, x64, fp64_ms, args.mixed_steps,
                              args.mixed_warmup, barrier, max_over_ranks, peak)
    return out


def mixed_sizes_leg(lib, args, seed, barrier, max_over_ranks) -> dict:
    """The mixed-precision form at the other sizes of its config (N = 32768
    and 65536, NB = 512), each against an FP64 solve of the same system timed
    here; the plain (single-pass) BF16 / FP16 forms at N <= 32768 too, where
    their result (converged or not) is part of the record."""
    import torch

    from rochpl_b200.hpl import Algo, default_ld
    from rochpl_b200.lib import PREC_BF16, PREC_BF16X3, PREC_FP16, PREC_FP16X3

    peak, _ = _bf16_peak()
    algo = Algo(512, 32, 2, 2, 2, 1, 0)
    out = {}
    for n in args.mixed_sizes:
        ld = default_ld(n)
        dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
        dX = torch.zeros(n, dtype=torch.float64, device="cuda")
        ms = []
        for it in range(1 + 2):
            lib.matgen(n, n + 1, seed, dA.data_ptr(), ld, 512)
            torch.cuda.synchronize()
            barrier()
            lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr())
            if it >= 1:
                ms.append(lib.last_timing()["total_ms"])
        fp64_ms = max_over_ranks(statistics.mean(ms))
        res64 = lib.residual_lcg(n, seed, dX.data_ptr())
        x64 = dX.cpu().numpy()
        del dA, dX
        torch.cuda.empty_cache()
        rec = {"fp64": {"ms_per_solve": fp64_ms, "value": hpl_flops(n) / (fp64_ms * 1e-3) / 1e12,
                        "resid": res64["resid"]}}
        precs = [("bf16x3", PREC_BF16X3), ("fp16x3", PREC_FP16X3)]
        if n <= 32768:
            precs += [("bf16", PREC_BF16), ("fp16", PREC_FP16)]
        for name, prec in precs:
            rec[name] = mixed_one(lib, algo, n, seed, prec, x64, fp64_ms,
                                  1 if prec < 2 else args.mixed_steps, 0 if prec < 2 else 1,
                                  barrier, max_over_ranks, peak)
        out[str(n)] = rec
        torch.cuda.empty_cache()
    return out


def grid_leg(lib, args, ranks) -> dict:
    """One system across all ranks: HPL_pdgesv on a 1 x world process grid
    (rochpl_b200.grid; NB-wide column blocks cyclic over the GPUs, the panel
    broadcast over NCCL), N = args.grid_n, seed 100.  Device time from CUDA
    events around the whole solve, max over ranks; the residual against the
    regenerated LCG matrix on rank 0."""
    import torch

    from rochpl_b200.grid import DeviceBackend, DistGroup, Grid1xQ, matgen_local, pdgesv_grid
    from rochpl_b200.hpl import Algo, default_ld

    n, nb = args.grid_n, args.nb
    algo = Algo(nb, 32, 2, 2, 2, 1, 0)
    g = Grid1xQ(n, nb, ranks.rank, ranks.world)
    ld = default_ld(n)
    be, comm = DeviceBackend(lib), DistGroup()
    A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64, device="cuda")
    ms = []
    for it in range(1 + args.grid_steps):
        matgen_local(be, g, 100, A, ld)
        torch.cuda.synchronize()
        ranks.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        x, ipiv, info = pdgesv_grid(be, comm, g, algo, A, ld)
        e1.record()
        torch.cuda.synchronize()
        if it >= 1:
            ms.append(e0.elapsed_time(e1))
    t = ranks.max(statistics.mean(ms))
    res = lib.residual_lcg(n, 100, x.data_ptr()) if ranks.rank == 0 else {"resid": None}
    del A
    torch.cuda.empty_cache()
    return {"workload": f"one HPL system N={n} NB={nb} on a 1 x {ranks.world} process grid "
                        "(column blocks cyclic over the GPUs, panel broadcast over NCCL)",
            "scaling": "strong (one system)", "ms_per_solve": t,
            "value": hpl_flops(n) / (t * 1e-3) / 1e12, "unit": UNIT, "info": info,
            "resid": res["resid"], "steps": args.grid_steps}


def batched_leg(lib, args, ranks):
    """The batched form: 4096 independent LCG systems, N log-uniform in
    [32, 1024], per-system seed 100 + i, nrhs in {1, 16, 64}; one persistent,
    graph-captured launch per solve, panel widths from the autotuner.  Over
    several ranks the systems are split by flops (batch.partition_systems):
    each rank generates and solves only its own, and the per-system residuals
    are assembled once at the end.  value = sum over ALL systems of
    (2/3 N^3 + 2 N^2 nrhs) / the max over ranks of the launch's device time."""
    import numpy as np
    import torch

    from rochpl_b200.batch import BatchShard, autotune, workload_sizes

    torch.cuda.empty_cache()
    n = workload_sizes(args.batch_count)
    out = {"workload": f"{args.batch_count} systems, N log-uniform in [32, 1024] "
                       "(numpy PCG64 seed 20261203), seed_i = 100 + i",
           "scaling": "strong (the systems are split across ranks by flops)"
                      if ranks.world > 1 else "one GPU",
           "by_nrhs": {}}
    for nrhs in (1, 16, 64):
        table = autotune(lib, nrhs=nrhs, use_cache=False)
        shard = BatchShard(lib, n, nrhs, ranks.rank, ranks.world, table)
        plan, seeds = shard.plan, shard.seeds
        dA = torch.zeros(max(plan.a_elems, 1), dtype=torch.float64, device="cuda")
        dB = torch.zeros(max(plan.b_elems, 1), dtype=torch.float64, device="cuda")
        dP = torch.zeros(max(plan.p_elems, 1), dtype=torch.int32, device="cuda")
        dI = torch.zeros(max(plan.count, 1), dtype=torch.int32, device="cuda")
        ms = []
        for it in range(args.warmup + args.steps):
            plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())  # outside the timed launch
            ranks.barrier()
            plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
            if it >= args.warmup:
                ms.append(plan.last_ms if plan.count else 0.0)
        res = torch.zeros(max(plan.count, 1), dtype=torch.float64, device="cuda")
        plan.residual(seeds, dB.data_ptr(), res.data_ptr())
        res_all = ranks.assemble(res.cpu().numpy()[:plan.count], shard.index, shard.total)
        sing = ranks.sum(float((dI[:plan.count] != 0).sum()))
        t = ranks.max(statistics.mean(ms))
        out["by_nrhs"][str(nrhs)] = {
            "ms_per_solve": t, "value": shard.total_flops / (t * 1e-3) / 1e12, "unit": UNIT,
            "resid_max": float(res_all.max()), "resid_passed": bool(float(res_all.max()) < 16.0),
            "singular": int(sing), "nb_by_class": table, "gpu_launches": 1,
            "flops": shard.total_flops, "systems_on_rank0": int(plan.count)}
        del dA, dB, dP, dI, res
        shard.close()
        torch.cuda.empty_cache()
    return out


def autograd_leg(lib, args, max_over_ranks):
    """The differentiable solve X = A^-1 B (FP64): N = 16384 with 32 RHS from
    the LCG (forward: factor + solve; backward: transposed solves on the stored
    factors + the fused rank-32 kernel), and 256 systems with N uniform in
    [64, 512] through the batched form."""
    import numpy as np
    import torch

    from rochpl_b200.autograd import hpl_solve, hpl_solve_batch
    from rochpl_b200.batch import BatchPlan

    torch.cuda.empty_cache()
    n, nrhs = args.ad_n, 32
    M = torch.empty((n + nrhs) * n, dtype=torch.float64, device="cuda")
    lib.matgen(n, n + nrhs, 100, M.data_ptr(), n)
    Mc = M.view(n + nrhs, n)
    A = Mc[:n].t().contiguous().requires_grad_(True)
    B = Mc[n:].t().contiguous().requires_grad_(True)
    del M, Mc
    Xbar = torch.ones(n, nrhs, dtype=torch.float64, device="cuda")
    fwd, bwd = [], []
    for it in range(args.warmup + args.steps):
        A.grad = None
        B.grad = None
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record()
        X = hpl_solve(A, B, nb=512)
        e1.record()
        X.backward(Xbar)
        e2.record()
        torch.cuda.synchronize()
        if it >= args.warmup:
            fwd.append(e0.elapsed_time(e1))
            bwd.append(e1.elapsed_time(e2))
    with torch.no_grad():
        r = (A @ X - B).abs().max().item()
    f_fwd = 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2 * nrhs
    tf, tb = max_over_ranks(statistics.mean(fwd)), max_over_ranks(statistics.mean(bwd))
    single = {"n": n, "nrhs": nrhs, "forward_ms": tf, "backward_ms": tb,
              "forward_tflops": f_fwd / (tf * 1e-3) / 1e12,
              "backward_flops": 4.0 * n ** 2 * nrhs, "abs_residual_max": r,
              "note": "torch CUDA events on the current stream around hpl_solve and backward()"}
    if not args.no_parity:
        single["checks"] = autograd_checks(A, B, X.detach(), Xbar)
    del A, B, X, Xbar
    torch.cuda.empty_cache()
    rng = np.random.default_rng(20261203)
    sizes = rng.integers(64, 513, size=256).astype(np.int32)
    plan = BatchPlan(lib, sizes, nrhs)
    As, Bs = [], []
    for i, m in enumerate(sizes):
        Mi = torch.empty(int(m) * (int(m) + nrhs), dtype=torch.float64, device="cuda")
        lib.matgen(int(m), int(m) + nrhs, 100 + i, Mi.data_ptr(), int(m))
        Mi = Mi.view(int(m) + nrhs, int(m))
        As.append(Mi[:m].t().contiguous().requires_grad_(True))
        Bs.append(Mi[m:].t().contiguous().requires_grad_(True))
    tfb = []
    for it in range(args.warmup + args.steps):
        for T in As + Bs:
            T.grad = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Xs = hpl_solve_batch(plan, As, Bs)
        sum(X.sum() for X in Xs).backward()
        torch.cuda.synchronize()
        if it >= args.warmup:
            tfb.append((time.perf_counter() - t0) * 1e3)
    plan.close()
    batch = {"systems": 256, "n_range": [64, 512], "nrhs": nrhs,
             "forward_backward_ms_wall": max_over_ranks(statistics.mean(tfb)),
             "note": "wall clock incl. packing the 512 tensors into pools"}
    return {"single": single, "batched": batch}


def autograd_checks(A, B, X, Xbar, h=1e-6, fd_tol=1e-4) -> dict:
    """Gradients of L = <Xbar, X(A, B)> after backward(): against an FP64
    reference from torch's own dense solve (a check, not the product path)
    within 64 n eps kappa_oo, and directional derivatives along unit-norm
    directions of A and of B (half seeded-random, half along the computed
    gradient) against central differences with step h."""
    import torch

    from rochpl_b200.autograd import hpl_solve

    n = A.shape[0]
    with torch.no_grad():
        Ad, Bd = A.detach(), B.detach()
        Xr = torch.linalg.solve(Ad, Bd)
        Bbar_r = torch.linalg.solve(Ad.t(), Xbar)
        Abar_r = -Bbar_r @ Xr.t()
        kappa = float(Ad.abs().sum(dim=1).max()) * float(
            torch.linalg.inv(Ad).abs().sum(dim=1).max())

    def rel(a, b):
        return float((a - b).abs().max() / b.abs().max())

    tol = 64 * n * 2.0 ** -53 * kappa
    out = {"kappa_inf": kappa, "tolerance": tol, "x_rel_err": rel(X, Xr),
           "abar_rel_err": rel(A.grad, Abar_r), "bbar_rel_err": rel(B.grad, Bbar_r)}
    out["within_tolerance"] = max(out["x_rel_err"], out["abar_rel_err"], out["bbar_rel_err"]) <= tol
    del Xr, Bbar_r, Abar_r
    g = torch.Generator(device=A.device).manual_seed(n)
    dA = torch.randn(A.shape, generator=g, dtype=torch.float64, device=A.device)
    dB = torch.randn(B.shape, generator=g, dtype=torch.float64, device=A.device)
    # The normalised sum of a random unit direction and the computed
    # gradient's direction: the derivative is then of the order of the
    # gradient's norm, far above the difference quotient's rounding floor.
    dA = dA / dA.norm() + A.grad / A.grad.norm()
    dB = dB / dB.norm() + B.grad / B.grad.norm()
    dA /= dA.norm()
    dB /= dB.norm()

    def L(Ap, Bp):
        with torch.no_grad():
            return float((hpl_solve(Ap, Bp, nb=512) * Xbar).sum())

    fdA = (L(Ad + h * dA, Bd) - L(Ad - h * dA, Bd)) / (2 * h)
    fdB = (L(Ad, Bd + h * dB) - L(Ad, Bd - h * dB)) / (2 * h)
    anA = float((A.grad * dA).sum())
    anB = float((B.grad * dB).sum())
    out["fd"] = {"step": h, "tolerance": fd_tol,
                 "direction": "unit norm: seeded Gaussian + the computed gradient's direction",
                 "dA": {"analytic": anA, "central_difference": fdA,
                        "rel_err": abs(anA - fdA) / abs(fdA)},
                 "dB": {"analytic": anB, "central_difference": fdB,
                        "rel_err": abs(anB - fdB) / abs(fdB)}}
    out["fd"]["passed"] = max(out["fd"]["dA"]["rel_err"], out["fd"]["dB"]["rel_err"]) <= fd_tol
    return out


def _cudart():
    """The CUDA runtime torch has already loaded (for exact-size pinned memory:
    torch's pinned allocator rounds a 137.5 GB request up to 256 GB)."""
    import ctypes

    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    return None


def _mem_available() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def end_to_end(lib, algo, n, ld, seed, dA, dX, barrier, max_over_ranks, world):
    """[A|b] uploaded from pinned host memory, hplb_pdgesv, x read back to the
    host, all inside a wall-clock timed region through the C ABI."""
    import ctypes

    import torch

    nbytes = ld * (n + 1) * 8
    rt = _cudart()
    hptr = ctypes.c_void_p()
    ok = (rt is not None and _mem_available() > nbytes + (24 << 30) and
          rt.cudaHostAlloc(ctypes.byref(hptr), ctypes.c_size_t(nbytes), 0) == 0)
    hX = torch.empty(n, dtype=torch.float64, pin_memory=True)
    if not ok:
        note = "pinned host buffer unavailable: inputs generated from the seed by hplb_matgen"
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        lib.matgen(n, n + 1, seed, dA.data_ptr(), ld, algo.nb)
        lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr())
        hX.copy_(dX)
        torch.cuda.synchronize()
        t = max_over_ranks(time.perf_counter() - t0)
        return {"value": world * hpl_flops(n) / t / 1e12, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": n * 8, "note": note}
    H2D, D2H = 1, 2
    try:
        lib.matgen(n, n + 1, seed, dA.data_ptr(), ld, algo.nb)
        torch.cuda.synchronize()
        # The host copy of [A|b] (the same LCG matrix), made before timing.
        assert rt.cudaMemcpy(hptr, ctypes.c_void_p(dA.data_ptr()), ctypes.c_size_t(nbytes),
                             D2H) == 0
        dA.zero_()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        assert rt.cudaMemcpy(ctypes.c_void_p(dA.data_ptr()), hptr, ctypes.c_size_t(nbytes),
                             H2D) == 0
        t_h2d = time.perf_counter() - t0
        lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr())
        hX.copy_(dX)
        torch.cuda.synchronize()
        t = max_over_ranks(time.perf_counter() - t0)
    finally:
        rt.cudaFreeHost(hptr)
    return {"value": world * hpl_flops(n) / t / 1e12, "unit": UNIT,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": n * 8,
            "h2d_s": t_h2d, "seconds": t,
            "note": "[A|b] from pinned host memory (cudaMemcpy), hplb_pdgesv, x back to the "
                    "host; wall clock"}


# ---------------------------------------------------------------------------
# Small single-kernel cases for profiling (--case)
# ---------------------------------------------------------------------------

def case_dgemm(args) -> None:
    """3 x hplb_dgemm_sub, --n x --n x --nb (k), random operands."""
    import torch

    from rochpl_b200 import library

    lib = library(0)
    m = n = args.n
    k = args.nb
    A = torch.randn(m * k, dtype=torch.float64, device="cuda")
    B = torch.randn(k * n, dtype=torch.float64, device="cuda")
    C = torch.randn(m * n, dtype=torch.float64, device="cuda")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        lib.dgemm_sub(m, n, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(f"dgemm_sub {m}x{n}x{k}: {ms:.3f} ms, {2.0 * m * n * k / ms / 1e9:.2f} TFLOP/s")


def _kernel_split(prof, top=24):
    """Per-kernel device time and launch count from a torch.profiler trace
    (CUPTI activity records: concurrent streams as in production)."""
    import collections

    agg = collections.defaultdict(lambda: [0.0, 0])
    for e in prof.events():
        if e.device_type.name != "CUDA":
            continue
        name = e.name.replace("void ", "").replace("hplb::(anonymous namespace)::", "")
        name = name.split("(")[0][:48]
        agg[name][0] += (e.time_range.end - e.time_range.start) / 1e3
        agg[name][1] += 1
    for name, (ms, cnt) in sorted(agg.items(), key=lambda kv: -kv[1][0])[:top]:
        print(f"{name:50s} {ms:10.2f} ms {cnt:7d}")


def case_solve(args) -> None:
    """generate + hplb_pdgesv (--n, --nb) twice, with the timing split of the
    second; --breakdown adds a per-kernel split of a third solve."""
    import torch

    from rochpl_b200 import library
    from rochpl_b200.hpl import Algo, default_ld

    lib = library(0)
    n, nb = args.n, args.nb
    ld = default_ld(n)
    algo = Algo(nb, 32, 2, 2, 2, 1, 0)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        lib.matgen(n, n + 1, 100, dA.data_ptr(), ld, nb)
        lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr())
    t = lib.last_timing()
    res = lib.residual_lcg(n, 100, dX.data_ptr())
    print(f"solve N={n} NB={nb}: {t['total_ms']:.2f} ms, "
          f"{hpl_flops(n) / t['total_ms'] / 1e9:.2f} TFLOP/s, lu {t['lu_ms']:.2f} ms, "
          f"panel {t['panel_ms']:.2f} ms, gemm {t['gemm_ms']:.2f} ms, trsv {t['trsv_ms']:.3f} ms "
          f"({n * n / 2 * 8 / (t['trsv_ms'] * 1e-3) / 1e9:.0f} GB/s), resid {res['resid']:.3e}")
    if args.breakdown:
        from torch.profiler import ProfilerActivity, profile

        lib.matgen(n, n + 1, 100, dA.data_ptr(), ld, nb)
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            lib.pdgesv(algo.c(), n, dA.data_ptr(), ld, dX.data_ptr())
            torch.cuda.synchronize()
        _kernel_split(prof)


def case_gemm_lp(args) -> None:
    """13 x hplb_gemm_lp_sub (FP16), --n x --n x --k, events over the last 10."""
    import torch

    from rochpl_b200 import library

    lib = library(0)
    m = n = args.n
    k = args.k
    A = (torch.rand(m, k, device="cuda") - 0.5).to(torch.float16)
    B = (torch.rand(n, k, device="cuda") - 0.5).to(torch.float16)
    sA = torch.ones((m + 127) // 128, device="cuda")
    sB = torch.ones((n + 255) // 256, device="cuda")
    C = torch.zeros(n, m, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 13
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


def case_getrf(args) -> None:
    """One hplb_getrf (--n, --nb): the leaves and the panel in context."""
    import torch

    from rochpl_b200 import library
    from rochpl_b200.hpl import Algo

    lib = library(0)
    n, nb = args.n, args.nb
    A = torch.empty(n * n, dtype=torch.float64, device="cuda")
    lib.matgen(n, n, 100, A.data_ptr(), n)
    ip = torch.zeros(n, dtype=torch.int32, device="cuda")
    lib.getrf(Algo(nb, 32, 2, 2, 2, 1, 0).c(), n, A.data_ptr(), n, ip.data_ptr())
    t = lib.last_timing()
    print(f"getrf N={n} NB={nb}: {t['total_ms']:.1f} ms (panels {t['panel_ms']:.1f} ms)")


def case_mixed(args) -> None:
    """hplb_pdgesv_mixed (--n, --prec), with a per-kernel split from the torch
    profiler's CUDA activity records."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    from rochpl_b200 import library
    from rochpl_b200.hpl import Algo

    lib = library(0)
    n = args.n
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    algo = Algo(args.nb, 32, 2, 2, 2, 1, 0)
    lib.pdgesv_mixed(algo.c(), n, x.data_ptr(), seed=100, precision=args.prec)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        r = lib.pdgesv_mixed(algo.c(), n, x.data_ptr(), seed=100, precision=args.prec)
        torch.cuda.synchronize()
    print({k: round(v, 2) if isinstance(v, float) else v for k, v in r.items()})
    _kernel_split(prof)


def case_batch(args) -> None:
    """592 systems of one size (--n) with panel width --nb (64: the recursive
    factorisation) and --nrhs right-hand sides; three launches."""
    import numpy as np
    import torch

    from rochpl_b200 import library
    from rochpl_b200.batch import BatchPlan

    lib = library(0)
    plan = BatchPlan(lib, np.full(148 * 4, args.n, dtype=np.int32), args.nrhs, [args.nb] * 6)
    dA = torch.zeros(plan.a_elems, dtype=torch.float64, device="cuda")
    dB = torch.zeros(plan.b_elems, dtype=torch.float64, device="cuda")
    dP = torch.zeros(plan.p_elems, dtype=torch.int32, device="cuda")
    dI = torch.zeros(plan.count, dtype=torch.int32, device="cuda")
    seeds = np.arange(plan.count, dtype=np.uint64)
    for _ in range(3):
        plan.matgen(seeds, dA.data_ptr(), dB.data_ptr())
        plan.gesv(dA.data_ptr(), dB.data_ptr(), dP.data_ptr(), dI.data_ptr())
    print(f"batch {plan.count} x N={args.n} NB={int(plan.nb[0])} nrhs={args.nrhs}: "
          f"{plan.last_ms:.2f} ms, {plan.flops() / plan.last_ms / 1e9:.2f} TFLOP/s")
    plan.close()


def case_autograd(args) -> None:
    """hpl_solve (--n, --nb, 32 RHS from the LCG) forward and backward, four
    times; CUDA events on the current stream, the mean of the last three."""
    import torch

    from rochpl_b200 import library
    from rochpl_b200.autograd import hpl_solve

    lib = library(0)
    n, nrhs = args.n, 32
    M = torch.empty((n + nrhs) * n, dtype=torch.float64, device="cuda")
    lib.matgen(n, n + nrhs, 100, M.data_ptr(), n)
    A = M.view(n + nrhs, n)[:n].t().contiguous().requires_grad_(True)
    B = M.view(n + nrhs, n)[n:].t().contiguous().requires_grad_(True)
    del M
    Xbar = torch.ones(n, nrhs, dtype=torch.float64, device="cuda")
    fwd, bwd = [], []
    for it in range(4):
        A.grad = B.grad = None
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record()
        X = hpl_solve(A, B, nb=args.nb)
        e1.record()
        X.backward(Xbar)
        e2.record()
        torch.cuda.synchronize()
        if it:
            fwd.append(e0.elapsed_time(e1))
            bwd.append(e1.elapsed_time(e2))
    tf = statistics.mean(fwd)
    f = 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2 * nrhs
    print(f"autograd N={n} NB={args.nb} nrhs={nrhs}: forward {tf:.2f} ms ({f / tf / 1e9:.2f} "
          f"TFLOP/s), backward {statistics.mean(bwd):.2f} ms")


CASES = {"dgemm": case_dgemm, "solve": case_solve, "gemm_lp": case_gemm_lp,
         "getrf": case_getrf, "mixed": case_mixed, "batch": case_batch,
         "autograd": case_autograd}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=131072)
    ap.add_argument("--nb", type=int, default=512)
    ap.add_argument("--cpu-n", type=int, default=16384,
                    help="host sample size for the CPU baseline / reference arm (every step) "
                         "and of the parity solve")
    ap.add_argument("--cpu-n-big", type=int, default=32768,
                    help="reference arm: the larger host sample (once) the N^3 extrapolation "
                         "starts from")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the LCG, parity-solve and gradient checks")
    ap.add_argument("--no-c1", action="store_true", help="skip the N = 4096 config line")
    ap.add_argument("--no-grid", action="store_true",
                    help="skip the one-system-across-all-GPUs leg (runs only with --gpus > 1)")
    ap.add_argument("--grid-n", type=int, default=131072)
    ap.add_argument("--grid-steps", type=int, default=1)
    ap.add_argument("--mixed-sizes", type=lambda v: [int(x) for x in v.split(",") if x],
                    default=[32768, 65536],
                    help="further N of the mixed-precision form (comma list; empty to skip)")
    ap.add_argument("--case", choices=sorted(CASES), default=None,
                    help="run one small profiling case instead of the benchmark")
    ap.add_argument("--k", type=int, default=1536, help="--case gemm_lp: reduction size")
    ap.add_argument("--prec", type=int, default=3, help="--case mixed: precision")
    ap.add_argument("--nrhs", type=int, default=16, help="--case batch: right-hand sides")
    ap.add_argument("--breakdown", action="store_true",
                    help="--case solve: per-kernel split of one more solve (torch profiler)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision (16-bit LU + GMRES-IR) leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-solver leg")
    ap.add_argument("--no-autograd", action="store_true", help="skip the autograd leg")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--ad-n", type=int, default=16384)
    ap.add_argument("--mixed-steps", type=int, default=2)
    ap.add_argument("--mixed-warmup", type=int, default=1)
    ap.add_argument("--gemm-traffic", type=float, default=None,
                    help="DRAM bytes per DGEMM launch from an ncu capture, if known")
    args = ap.parse_args()
    if args.case:
        CASES[args.case](args)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
