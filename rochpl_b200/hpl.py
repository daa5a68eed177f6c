"""Host-side mirror of rocHPL's interface for the single-process solve path.

Names follow the reference:
  HPL_pdmatgen  allocate [A|b] (padded ld) and the solution vector, fill A
                (src/matgen/HPL_pdmatgen.cpp:85-383 + HPL_pdrandmat)
  HPL_pdgesv    factor and solve (include/hpl_pgesv.hpp:162)
  HPL_pdtest    generate, time the solve, regenerate, check the scaled
                residual against the threshold (src/HPL_pdtest.cpp:21-495)
  parse_hpl_dat the HPL.dat reader of src/HPL_pdinfo.cpp:590-1030, with the
                same rejections and messages
  parse_cli     the rocHPL command-line flags of src/HPL_pdinfo.cpp:251-385

Device memory comes from torch; all compute goes through libhplb200.so.
"""
from __future__ import annotations

import dataclasses
import time

from .lib import Library, hplb_algo, library

HPL_ISEED = 100  # include/hpl_ptest.hpp:57
HPL_MAX_PARAM = 20  # include/hpl_ptest.hpp:56


class HplInputError(ValueError):
    """An HPL.dat / command-line value rocHPL rejects (same message)."""


@dataclasses.dataclass
class Algo:
    """HPL_T_palg fields that reach the solve (include/hpl_pgesv.hpp:63-81)."""
    nb: int = 384
    nbmin: int = 32
    ndiv: int = 2
    pfact: int = 2  # 0 left, 1 Crout, 2 right
    rfact: int = 2
    depth: int = 1
    l1notran: int = 0

    def c(self) -> hplb_algo:
        return hplb_algo(self.nb, self.nbmin, self.ndiv, self.pfact, self.rfact, self.depth,
                         self.l1notran)


@dataclasses.dataclass
class Pmat:
    """HPL_T_pmat at P = Q = 1 (include/hpl_pgesv.hpp:83-109)."""
    n: int
    nb: int
    ld: int
    A: object  # torch.Tensor, float64, ld * (n + 1) elements, column-major
    X: object  # torch.Tensor, float64, n elements
    ipiv: object  # torch.Tensor, int32, n elements
    info: int = 0


def default_ld(n: int) -> int:
    """((max(1,n)+95)/128)*128+32 (src/matgen/HPL_pdmatgen.cpp:109-110)."""
    return ((max(1, n) + 95) // 128) * 128 + 32


def hpl_flops(n: int) -> float:
    """Algorithmic flops of the solve, 2/3 n^3 + 2 n^2."""
    return 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2


def hpl_flops_reference(n: int) -> float:
    """The count rocHPL prints, 2/3 n^3 + 3/2 n^2 (src/HPL_pdtest.cpp:164-165)."""
    return 2.0 / 3.0 * n ** 3 + 3.0 / 2.0 * n ** 2


def HPL_pdmatgen(n: int, nb: int, seed: int = HPL_ISEED, device: int = 0,
                 lib: Library | None = None, ld: int | None = None) -> Pmat:
    """Allocate [A|b] and X on the device and generate A with the LCG."""
    import torch

    lib = lib or library(device)
    ld = ld or default_ld(n)
    dev = torch.device("cuda", device)
    A = torch.empty(ld * (n + 1), dtype=torch.float64, device=dev)
    X = torch.zeros(max(n, 1), dtype=torch.float64, device=dev)
    ipiv = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
    lib.matgen(n, n + 1, seed, A.data_ptr(), ld, nb)
    return Pmat(n=n, nb=nb, ld=ld, A=A, X=X, ipiv=ipiv)


def HPL_pdgesv(algo: Algo, mat: Pmat, lib: Library | None = None) -> int:
    """Factor [A|b] and solve; returns info (first zero-pivot column or 0)."""
    lib = lib or library(mat.A.device.index or 0)
    mat.info = lib.pdgesv(algo.c(), mat.n, mat.A.data_ptr(), mat.ld, mat.X.data_ptr(),
                          mat.ipiv.data_ptr())
    return mat.info


def HPL_pdtest(algo: Algo, n: int, seed: int = HPL_ISEED, thrsh: float = 16.0,
               device: int = 0, lib_fused_residual: bool = False) -> dict:
    """One HPL test at P = Q = 1: generate, time the solve (pdgesv including the
    back-solve, as src/HPL_pdtest.cpp:132-134), regenerate [A|b] and compute
    the scaled residual."""
    import torch

    lib = library(device)
    mat = HPL_pdmatgen(n, algo.nb, seed, device, lib)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    HPL_pdgesv(algo, mat, lib)
    t = time.perf_counter() - t0
    timing = lib.last_timing()
    if lib_fused_residual:
        res = lib.residual_lcg(n, seed, mat.X.data_ptr())
    else:
        lib.matgen(n, n + 1, seed, mat.A.data_ptr(), mat.ld, algo.nb)
        res = lib.residual(n, mat.A.data_ptr(), mat.ld, mat.X.data_ptr())
    out = {
        "n": n, "nb": algo.nb, "time_s": t, "gflops": hpl_flops(n) / t / 1e9 if t > 0 else 0.0,
        "gflops_reference_formula": hpl_flops_reference(n) / t / 1e9 if t > 0 else 0.0,
        "info": mat.info, "passed": res["resid"] < thrsh, **res, "timing": timing,
    }
    out["mat"] = mat
    return out


# ---------------------------------------------------------------------------
# HPL.dat and command line
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class HplConfig:
    """The parameter sweep one HPL.dat (or command line) describes."""
    ns: list
    nbs: list
    ps: list
    qs: list
    thrsh: float = 16.0
    pfacts: list = dataclasses.field(default_factory=lambda: [2])
    nbmins: list = dataclasses.field(default_factory=lambda: [32])
    ndivs: list = dataclasses.field(default_factory=lambda: [2])
    rfacts: list = dataclasses.field(default_factory=lambda: [2])
    depths: list = dataclasses.field(default_factory=lambda: [1])
    l1notran: int = 0
    outfile: str | None = None
    iters: int = 1
    frac: float = 0.3
    pmap: int = 1  # process mapping: 0 row-major, 1 column-major (the command line's)
    bcasts: list = dataclasses.field(default_factory=lambda: [0])  # 0..5: 1rg .. blongM

    def algos(self):
        for nb in self.nbs:
            for pf in self.pfacts:
                for nbm in self.nbmins:
                    for nd in self.ndivs:
                        for rf in self.rfacts:
                            for dp in self.depths:
                                yield Algo(nb, nbm, nd, pf, rf, dp, self.l1notran)


def _fact(j: int) -> int:
    # src/HPL_pdinfo.cpp:840-862: 0 left, 1 Crout, 2 right, anything else right
    return j if j in (0, 1, 2) else 2


def parse_hpl_dat(text: str) -> HplConfig:
    """Read an HPL.dat (src/HPL_pdinfo.cpp:590-1030).  Raises HplInputError with
    the reference's message for the values it rejects."""
    lines = text.splitlines()
    pos = [2]  # the first two lines are free text

    def nxt() -> str:
        if pos[0] >= len(lines):
            raise HplInputError("Illegal input in file HPL.dat. Exiting ...")
        s = lines[pos[0]]
        pos[0] += 1
        return s

    def first_int(line: str) -> int:
        tok = line.split()
        return int(tok[0]) if tok and _isint(tok[0]) else 0

    def ints(line: str, k: int):
        tok = line.split()
        return [int(t) if _isint(t) else 0 for t in (tok + ["0"] * k)[:k]]

    def count(line: str, what: str) -> int:
        k = first_int(line)
        if k < 1 or k > HPL_MAX_PARAM:
            raise HplInputError(f"Number of values of {what} is less than 1 or greater than "
                                f"{HPL_MAX_PARAM}")
        return k

    outtok = nxt().split()
    outname = outtok[0] if outtok else None
    dev = first_int(nxt())  # device out (6 stdout, 7 stderr, else file)
    k = count(nxt(), "N")
    ns = ints(nxt(), k)
    if any(v < 0 for v in ns):
        raise HplInputError("Value of N less than 0")
    k = count(nxt(), "NB")
    nbs = ints(nxt(), k)
    if any(v < 1 for v in nbs):
        raise HplInputError("Value of NB less than 1")
    pmap = 1 if first_int(nxt()) == 1 else 0  # PMAP: 1 column-major, else row-major
    k = count(nxt(), "grids")
    ps = ints(nxt(), k)
    qs = ints(nxt(), k)
    if any(v < 1 for v in ps):
        raise HplInputError("Value of P less than 1")
    if any(v < 1 for v in qs):
        raise HplInputError("Value of Q less than 1")
    tline = nxt().split()
    thrsh = float(tline[0]) if tline else 16.0
    k = count(nxt(), "PFACT")
    pfacts = [_fact(v) for v in ints(nxt(), k)]
    k = count(nxt(), "NBMIN")
    nbmins = ints(nxt(), k)
    if any(v < 1 for v in nbmins):
        raise HplInputError("Value of NBMIN less than 1")
    k = count(nxt(), "NDIV")
    ndivs = ints(nxt(), k)
    if any(v < 2 for v in ndivs):
        raise HplInputError("Value of NDIV less than 2")
    k = count(nxt(), "RFACT")
    rfacts = [_fact(v) for v in ints(nxt(), k)]
    k = count(nxt(), "BCAST")
    # Broadcast topologies: no data moves at Q = 1, but each is a test of its own.
    bcasts = [v if 0 <= v <= 4 else 5 for v in ints(nxt(), k)]
    k = count(nxt(), "DEPTH")
    depths = ints(nxt(), k)
    if any(v < 0 for v in depths):
        raise HplInputError("Value of DEPTH less than 0")
    if any(v != 1 for v in depths):
        raise HplInputError("Value of DEPTH must be 1")
    swap = first_int(nxt())
    if swap != 1:
        raise HplInputError("Value of SWAP must be 1")
    nxt()  # swapping threshold
    l1 = first_int(nxt())
    l1 = l1 if l1 in (0, 1) else 0
    u = first_int(nxt())
    u = u if u in (0, 1) else 0
    if u != 0:
        raise HplInputError("U  in no-transposed form unsupported")
    eq = first_int(nxt())
    eq = eq if eq in (0, 1) else 1
    if eq != 0:
        raise HplInputError("Equilibration currently unsupported")
    return HplConfig(ns=ns, nbs=nbs, ps=ps, qs=qs, thrsh=thrsh, pfacts=pfacts, nbmins=nbmins,
                     ndivs=ndivs, rfacts=rfacts, depths=depths, l1notran=l1,
                     outfile=outname if dev not in (6, 7) else None, pmap=pmap, bcasts=bcasts)


def _isint(s: str) -> bool:
    try:
        int(s)
        return True
    except ValueError:
        return False


def parse_cli(argv) -> HplConfig | None:
    """rocHPL's command line (src/HPL_pdinfo.cpp:251-385): -P -Q -p -q -N -NB
    -f -it -i.  Returns None when -i names an HPL.dat to read instead; the
    command-line run fixes PFACT=R, NBMIN=32, NDIV=2, RFACT=R, DEPTH=1
    (:487-560)."""
    P = Q = 1
    n, nb, it, frac = 45312, 384, 1, 0.3
    i = 0
    inputfile = None
    while i < len(argv):
        a = argv[i]
        val = argv[i + 1] if i + 1 < len(argv) else None
        if a in ("-P", "--ranksP"):
            P = int(val)
            if P < 1:
                raise HplInputError("Illegal value for P. Exiting ...")
            i += 1
        elif a in ("-Q", "--ranksQ"):
            Q = int(val)
            if Q < 1:
                raise HplInputError("Illegal value for Q. Exiting ...")
            i += 1
        elif a in ("-p", "-q"):
            i += 1
        elif a in ("-N", "--sizeN"):
            n = int(val)
            if n < 1:
                raise HplInputError("Illegal value for N. Exiting ...")
            i += 1
        elif a in ("-NB", "--sizeNB"):
            nb = int(val)
            if nb < 1:
                raise HplInputError("Illegal value for NB. Exiting ...")
            i += 1
        elif a in ("-f", "--frac"):
            frac = float(val)
            i += 1
        elif a == "-it":
            it = int(val)
            i += 1
        elif a in ("-i", "--input"):
            inputfile = val
            i += 1
        i += 1
    if inputfile is not None:
        return None
    return HplConfig(ns=[n], nbs=[nb], ps=[P], qs=[Q], iters=it, frac=frac)
