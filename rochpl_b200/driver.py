"""The HPL run driver: what rocHPL's xhpl does around the solve.

  sweep       the parameter loops of src/HPL_pddriver.cpp:120-212, in the same
              order: grids, then N, NB, DEPTH, BCAST, RFACT, PFACT, NBMIN, NDIV
  test        src/HPL_pdtest.cpp:105-213 and :425-450: a warm-up (the role of
              src/HPL_pdwarmup.cpp:18-105: every kernel of the solve runs once
              before the timed solves), then `-it` repetitions of generate,
              timed solve, residual check
  output      the reference's lines: the T/V table, the start and end times,
              the residual line with PASSED / FAILED (and the norms when it
              fails), the final tally (src/HPL_pddriver.cpp:226-283)
  progress    the per-step report of src/pgesv/HPL_pdgesv.cpp:136-341
              (HPL_PROGRESS_REPORT), from hplb_last_steps

One process runs the 1 x 1 grids (GpuSolver).  Launched as W processes (one
per GPU, torchrun), the driver runs the P x Q grids with P Q = W as one
distributed solve (GridSolver: rochpl_b200.grid for 1 x W, NB-wide column
blocks cyclic over the GPUs and the panel broadcast over NCCL;
rochpl_b200.grid2d for P > 1, the processes placed in PMAP order); process 0
reads the input for all and writes the output.  Grids of another size are
counted as skipped tests.  The solve itself, the generator and the residual run
on the GPU through libhplb200.so; the driver only formats and counts, so its
loops and output are tested with a stand-in solver on the CPU.

    python -m rochpl_b200.driver [-N 45312] [-NB 384] [-it 1] [-i HPL.dat] [--progress]
    torchrun --nproc-per-node Q -m rochpl_b200.driver -N 65536 -NB 512 -P 1 -Q Q
"""
from __future__ import annotations

import sys
import time

from .hpl import (HPL_ISEED, Algo, HplConfig, HplInputError, default_ld, hpl_flops_reference,
                  parse_cli, parse_hpl_dat)

RULE_EQ = "=" * 80
RULE_DASH = "-" * 80

_FACT = {0: "L", 1: "C", 2: "R"}  # src/HPL_pdtest.cpp:167-176


def tv_code(algo: Algo, bcast: int, pmap: int) -> str:
    """The T/V column: W, grid order, depth, broadcast topology, RFACT, NDIV,
    PFACT, NBMIN (src/HPL_pdtest.cpp:192-206)."""
    return "W%c%1d%c%c%1d%c%1d" % ("C" if pmap == 1 else "R", algo.depth, str(bcast),
                                  _FACT.get(algo.rfact, "R"), algo.ndiv,
                                  _FACT.get(algo.pfact, "R"), algo.nbmin)


def table_header() -> str:
    return (RULE_EQ + "\n"
            "T/V                N    NB     P     Q               Time                 Gflops\n"
            + RULE_DASH + "\n")


def result_lines(algo: Algo, bcast: int, pmap: int, n: int, p: int, q: int, wtime: float,
                 t_start: float, t_end: float) -> str:
    """The result line and the start / end times (src/HPL_pdtest.cpp:161-213).
    Gflops is the reference's count, (2/3 N^3 + 3/2 N^2) / t."""
    if wtime <= 0.0:
        return ""
    gflops = hpl_flops_reference(n) / wtime / 1e9
    return ("%s%12d %5d %5d %5d %18.2f     %18.3e\n" % (tv_code(algo, bcast, pmap), n, algo.nb,
                                                     p, q, wtime, gflops)
            + "HPL_pdgesv() start time %s\n\n" % time.ctime(t_start)
            + "HPL_pdgesv() end time   %s\n\n" % time.ctime(t_end))


def residual_lines(res: dict, thrsh: float) -> str:
    """src/HPL_pdtest.cpp:439-475: the scaled residual against the threshold,
    and the norms behind it when the check fails."""
    r = res["resid"]
    ok = r < thrsh
    out = (RULE_DASH + "\n" + "%s%16.7f%s%s\n" % (
        "||Ax-b||_oo/(eps*(||A||_oo*||x||_oo+||b||_oo)*N)= ", r, " ...... ",
        "PASSED" if ok else "FAILED"))
    if not ok:
        for label, key in (("||Ax-b||_oo  . . . . . . . . . . . . . . . . . = ", "rnorm_inf"),
                           ("||A||_oo . . . . . . . . . . . . . . . . . . . = ", "anorm_inf"),
                           ("||A||_1  . . . . . . . . . . . . . . . . . . . = ", "anorm_1"),
                           ("||x||_oo . . . . . . . . . . . . . . . . . . . = ", "xnorm_inf"),
                           ("||x||_1  . . . . . . . . . . . . . . . . . . . = ", "xnorm_1"),
                           ("||b||_oo . . . . . . . . . . . . . . . . . . . = ", "bnorm_inf")):
            out += "%s%18.6f\n" % (label, res.get(key, 0.0))
    return out


def summary_lines(kpass: int, kfail: int, kskip: int, thrsh: float) -> str:
    """The final tally (src/HPL_pddriver.cpp:226-283)."""
    ktest = kpass + kfail + kskip
    out = RULE_EQ + "\n" + "\n%s %6d %s\n" % ("Finished", ktest, "tests with the following results:")
    if thrsh > 0.0:
        out += "         %6d %s\n" % (kpass, "tests completed and passed residual checks,")
        out += "         %6d %s\n" % (kfail, "tests completed and failed residual checks,")
        out += "         %6d %s\n" % (kskip, "tests skipped because of illegal input values.")
    else:
        out += "         %6d %s\n" % (kpass, "tests completed without checking,")
        out += "         %6d %s\n" % (kskip, "tests skipped because of illegal input values.")
    return out + RULE_DASH + "\n" + "\nEnd of Tests.\n" + RULE_EQ + "\n"


def progress_lines(steps, n: int) -> str:
    """The per-step report (src/pgesv/HPL_pdgesv.cpp:155-160 header, :284-341
    rows without the detailed-timing columns): percent of columns done, the
    step's first column, its time, and the rate so far, counted as the
    reference counts it: (2/3 (N^3 - r^3) - 1/2 (N^2 - r^2) - 1/6 (N - r)) / t
    with r the columns still to factor after the step."""
    out = ("---------------------------------------------------\n"
           "   %   | Column    | Step Time (s) | Overall GFLOPS\n"
           "       |           |               |               \n"
           "---------------------------------------------------\n")
    total = 0.0
    cols = [c for c, _ in steps] + [n]
    for i, (j, ms) in enumerate(steps):
        total += ms * 1e-3
        r = n - cols[i + 1]
        done = (2.0 / 3.0 * (float(n) ** 3 - float(r) ** 3) - 0.5 * (float(n) ** 2 - float(r) ** 2)
                - (n - r) / 6.0)
        gflops = done / (total if total > 0.0 else 1e-6) / 1e9
        out += "%5.1f%% | %09d | " % (j * 100.0 / n if n else 0.0, j)
        out += "   %9.7f  |" % (ms * 1e-3)
        out += "    %9.3e   \n" % gflops
    return out


def sweep(cfg: HplConfig):
    """(n, p, q, bcast, algo) in the reference's loop order."""
    for p, q in zip(cfg.ps, cfg.qs):
        for n in cfg.ns:
            for nb in cfg.nbs:
                for depth in cfg.depths:
                    for bc in cfg.bcasts:
                        for rf in cfg.rfacts:
                            for pf in cfg.pfacts:
                                for nbm in cfg.nbmins:
                                    for nd in cfg.ndivs:
                                        yield n, p, q, bc, Algo(nb, nbm, nd, pf, rf, depth,
                                                                cfg.l1notran)


def skipped(p: int, q: int, algo: Algo, world: int = 1, two_d: bool = False) -> bool:
    """Tests this driver counts as skipped: values the library does not take
    (NBMIN > 128, NB > 2048, DEPTH != 1), and grids it cannot run: P x Q must
    use all the processes, and P must be 1 unless the solver runs 2-D grids
    (`two_d`)."""
    if algo.nbmin > 128 or algo.nb > 2048 or algo.depth != 1 or p * q != world:
        return True
    return p != 1 and not two_d


class GpuSolver:
    """One device, one [A|b] buffer reused while N stays the same.  A call
    generates [A|b] (seed 100), times hplb_pdgesv by the wall clock around the
    synchronous call (as HPL_ptimer does around HPL_pdgesv), checks the residual
    against the regenerated matrix and returns the numbers the driver prints."""

    def __init__(self, device: int = 0):
        import torch

        from .lib import library

        self.torch = torch
        self.device = device
        self.lib = library(device)
        self._key = None
        self._mat = None

    def _buffers(self, n: int):
        if self._key != n:
            self._mat = None
            torch = self.torch
            ld = default_ld(n)
            dev = torch.device("cuda", self.device)
            self._mat = (ld, torch.empty(ld * (n + 1), dtype=torch.float64, device=dev),
                         torch.zeros(max(n, 1), dtype=torch.float64, device=dev))
            self._key = n
        return self._mat

    def warmup(self, algo: Algo, n: int) -> None:
        """Every kernel of the solve once, on a system of at most 2 NB + 1 in
        buffers of its own (the test's [A|b] stays allocated)."""
        torch = self.torch
        m = min(n, 2 * algo.nb + 1)
        ld = default_ld(m)
        dev = torch.device("cuda", self.device)
        A = torch.empty(ld * (m + 1), dtype=torch.float64, device=dev)
        X = torch.zeros(max(m, 1), dtype=torch.float64, device=dev)
        self.lib.matgen(m, m + 1, HPL_ISEED, A.data_ptr(), ld, algo.nb)
        self.lib.pdgesv(algo.c(), m, A.data_ptr(), ld, X.data_ptr(), 0)
        torch.cuda.synchronize(self.device)

    def __call__(self, algo: Algo, n: int, seed: int = HPL_ISEED, progress: bool = False) -> dict:
        ld, A, X = self._buffers(n)
        lib = self.lib
        lib.matgen(n, n + 1, seed, A.data_ptr(), ld, algo.nb)
        self.torch.cuda.synchronize(self.device)
        t_start = time.time()
        t0 = time.perf_counter()
        info = lib.pdgesv(algo.c(), n, A.data_ptr(), ld, X.data_ptr(), 0)
        wtime = time.perf_counter() - t0
        t_end = time.time()
        res = lib.residual_lcg(n, seed, X.data_ptr())
        out = {"wtime": wtime, "t_start": t_start, "t_end": t_end, "info": info, **res}
        if progress:
            out["steps"] = lib.last_steps()
        return out


class GridSolver:
    """This process's part of one system on a P x Q grid of all processes
    (torch.distributed already initialised, one GPU each): the 1 x Q solve of
    rochpl_b200.grid, or the 2-D one of rochpl_b200.grid2d when P > 1.  The
    solve is timed by the wall clock between two barriers, the slowest
    process's time (as HPL_ptimer_combine takes the maximum); the residual is
    computed on rank 0 against the regenerated matrix.  pmap: HPL.dat's PMAP,
    the order of the processes on a P x Q grid (0 row-, 1 column-major)."""

    takes_grid = True  # run() passes each test's (P, Q)

    def __init__(self, device: int = 0, pmap: int = 0, lib=None, backend=None, backend2d=None,
                 dev=None):
        """lib, backend, backend2d and dev, when given, stand in for the GPU's
        library (its residual check), the two grid backends and the device:
        the tests run this solver's orchestration on CPU with host
        backends."""
        import torch
        import torch.distributed as dist

        from .grid import DeviceBackend, DistGroup
        from .grid2d import DeviceBackend2D

        self.torch, self.dist = torch, dist
        self.device = device
        if lib is None:
            from .lib import library

            lib = library(device)
        self.lib = lib
        self.backend = backend if backend is not None else DeviceBackend(lib)
        self.backend2d = backend2d if backend2d is not None else DeviceBackend2D(lib)
        self.dev = dev if dev is not None else torch.device("cuda", device)
        self.comm = DistGroup()
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.pmap = pmap
        self._comms2d = {}  # (P, Q) -> (row, col, world); every rank builds the same groups

    def _run(self, algo: Algo, n: int, seed: int, grid):
        from .grid import Grid1xQ, matgen_local, pdgesv_grid
        from .grid2d import Grid2D, dist_comms, matgen_local_2d, pdgesv_2d

        torch = self.torch
        P, Q = grid if grid is not None else (1, self.world)
        dev = self.dev
        if P == 1:
            g = Grid1xQ(n, algo.nb, self.rank, self.world)
            ld = default_ld(n)
            A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64, device=dev)
            matgen_local(self.backend, g, seed, A, ld)
            solve = lambda: pdgesv_grid(self.backend, self.comm, g, algo, A, ld)  # noqa: E731
        else:
            if (P, Q) not in self._comms2d:
                self._comms2d[(P, Q)] = dist_comms(P, Q, self.pmap)
            p, q = Grid2D.coords(self.rank, P, Q, self.pmap)
            g = Grid2D(n, algo.nb, p, q, P, Q, self.pmap)
            ld = (max(g.mp, 1) + 1) // 2 * 2  # even: the DGEMM's TMA path
            A = torch.zeros(ld * max(g.nq, 1), dtype=torch.float64, device=dev)
            matgen_local_2d(self.backend2d, g, seed, A, ld)
            comms = self._comms2d[(P, Q)]
            solve = lambda: pdgesv_2d(self.backend2d, comms, g, algo, A, ld)  # noqa: E731
        self._sync()
        self.dist.barrier()
        t_start = time.time()
        t0 = time.perf_counter()
        x, ipiv, info = solve()
        self._sync()
        w = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
        self.dist.all_reduce(w, op=self.dist.ReduceOp.MAX)
        return x, info, float(w.item()), t_start, time.time()

    def _sync(self):
        if self.dev.type == "cuda":
            self.torch.cuda.synchronize(self.dev)

    def warmup(self, algo: Algo, n: int, grid=None) -> None:
        self._run(algo, min(n, 2 * algo.nb * self.world + 1), HPL_ISEED, grid)

    def __call__(self, algo: Algo, n: int, seed: int = HPL_ISEED, progress: bool = False,
                 grid=None) -> dict:
        x, info, wtime, t_start, t_end = self._run(algo, n, seed, grid)
        res = (self.lib.residual_lcg(n, seed, x.data_ptr()) if self.rank == 0 else
               {"resid": 0.0})
        return {"wtime": wtime, "t_start": t_start, "t_end": t_end, "info": info, **res}


class _Discard:
    def write(self, s):
        return len(s)

    def flush(self):
        return None


def run(cfg: HplConfig, out=None, solver=None, progress: bool = False, world: int = 1) -> dict:
    """Run every test of the sweep; write the reference's output to `out`
    (default stdout); return the tally.  `solver(algo, n, progress=...)` returns
    a dict with wtime, t_start, t_end, resid and the norms (GpuSolver by
    default); `solver.warmup(algo, n)` runs before each test's repetitions."""
    out = out or sys.stdout
    solver = solver if solver is not None else GpuSolver()
    kpass = kfail = kskip = 0
    first = True
    two_d = getattr(solver, "takes_grid", False)
    for n, p, q, bc, algo in sweep(cfg):
        if skipped(p, q, algo, world, two_d):
            kskip += 1
            continue
        kw = {"grid": (p, q)} if two_d else {}
        warm = getattr(solver, "warmup", None)
        if warm is not None:
            warm(algo, n, **kw)
        for _ in range(max(cfg.iters, 1)):
            r = solver(algo, n, progress=progress, **kw)
            # The table header precedes every result while residuals are
            # checked, only the first without checking (src/HPL_pdtest.cpp:144-158).
            if first:
                out.write(table_header())
                if cfg.thrsh <= 0.0:
                    first = False
            if progress and r.get("steps"):
                out.write(progress_lines(r["steps"], n))
            out.write(result_lines(algo, bc, cfg.pmap, n, p, q, r["wtime"], r["t_start"],
                                   r["t_end"]))
            if cfg.thrsh > 0.0:
                if r["resid"] < cfg.thrsh:
                    kpass += 1
                else:
                    kfail += 1
                out.write(residual_lines(r, cfg.thrsh))
            else:
                kpass += 1
        out.flush()
    out.write(summary_lines(kpass, kfail, kskip, cfg.thrsh))
    out.flush()
    return {"passed": kpass, "failed": kfail, "skipped": kskip}


def config_from_argv(argv) -> HplConfig:
    """The command line, or the HPL.dat that -i names."""
    cfg = parse_cli(argv)
    if cfg is None:
        path = argv[argv.index("-i") + 1] if "-i" in argv else argv[argv.index("--input") + 1]
        with open(path) as f:
            cfg = parse_hpl_dat(f.read())
        if "-it" in argv:  # -it also applies to a run from HPL.dat
            cfg.iters = int(argv[argv.index("-it") + 1])
    return cfg


def shared_config(argv, rank: int):
    """The run's configuration on every process of a torch.distributed job,
    as HPL_pdinfo does it (src/HPL_pdinfo.cpp): process 0 alone reads the
    command line and HPL.dat, and every process takes its values from it.
    Returns the HplConfig, or the message of the input error, the same on
    every process, so a bad input ends every process and none waits for the
    others."""
    import torch.distributed as dist

    box = [None]
    if rank == 0:
        try:
            box[0] = config_from_argv(argv)
        except (HplInputError, OSError) as e:
            box[0] = str(e)
    dist.broadcast_object_list(box, src=0)
    return box[0]


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    progress = "--progress" in argv
    if progress:
        argv.remove("--progress")
    import os

    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world == 1:
        try:
            cfg = config_from_argv(argv)
        except HplInputError as e:
            print(e, file=sys.stderr)
            return 1
    solver, rank = None, 0
    if world > 1:  # one process per GPU under torchrun: the P x Q = world grids
        import torch
        import torch.distributed as dist

        rank, local = int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
        cfg = shared_config(argv, rank)
        if isinstance(cfg, str):
            if rank == 0:
                print(cfg, file=sys.stderr)
            dist.destroy_process_group()
            return 1
        solver = GridSolver(local, pmap=cfg.pmap)
    try:
        if rank != 0:
            tally = run(cfg, _Discard(), solver=solver, world=world)
        elif cfg.outfile:
            with open(cfg.outfile, "w") as f:
                tally = run(cfg, f, solver=solver, progress=progress, world=world)
        else:
            tally = run(cfg, sys.stdout, solver=solver, progress=progress and world == 1,
                        world=world)
    finally:
        if world > 1:
            dist.destroy_process_group()
    return 0 if tally["failed"] == 0 else 2


if __name__ == "__main__":
    sys.exit(main())
