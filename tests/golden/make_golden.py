"""Generates the golden fixtures in this folder from rocHPL's OWN code.

Every number written here comes from the reference sources compiled by
oracle/build_ref.sh into oracle/_ref/libhplref.so:

  lcg_golden.json   -- hpl_randmat / HPL_pdrandmat run on a CUDA device:
                       FNV-1a hash of every generated matrix plus sampled entries
                       (needs a GPU: run as `python tests/golden/make_golden.py --lcg`
                       on the GPU box, copy the json back).
  jump_golden.json  -- HPL_xjumpm constants (host code).
  lcg_c2_golden.json -- the same generator for four blocks of the N = 131072
                       [A|b] (first, middle and last 512-column blocks and b),
                       state indices up to 1.7e10 (GPU: `--lcg-c2`).
  perm_golden.json  -- HPL_pipid + the permU unrolling of HPL_pdpanel_swapids
                       for seeded random pivot vectors (host code).

The CPU tests then check the oracle against these files without needing the
reference tree.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

# (m, n, nb) shapes: the small edge cases and the first config (N=4096, NB=256).
LCG_SHAPES = [(1, 2, 1), (2, 3, 1), (31, 32, 8), (257, 258, 64), (1000, 1001, 256),
              (4096, 4097, 256), (5000, 37, 384)]


def make_lcg(outdir: str) -> None:
    import torch

    R = O.ref()
    assert R is not None, "oracle/_ref/libhplref.so not built"
    rng = np.random.default_rng(12345)
    out = []
    for (m, n, nb) in LCG_SHAPES:
        ld = O.default_ld(m)
        dA = torch.zeros(ld * n, dtype=torch.float64, device="cuda")
        rc = R.ref_pdrandmat(m, n, nb, dA.data_ptr(), ld, 100)
        assert rc == 0, rc
        A = dA.view(n, ld).T.cpu().numpy()  # ld x n, column-major view
        A = np.asfortranarray(A)
        h = O.hash_block(A, m, n)
        ii = rng.integers(0, m, 16)
        jj = rng.integers(0, n, 16)
        samples = [[int(i), int(j), A[i, j].hex()] for i, j in zip(ii, jj)]
        samples += [[0, 0, A[0, 0].hex()], [m - 1, n - 1, A[m - 1, n - 1].hex()]]
        out.append({"m": m, "n": n, "nb": nb, "seed": 100, "fnv1a": f"{h:016x}",
                    "samples": samples})
        print(m, n, nb, f"{h:016x}")
    with open(os.path.join(outdir, "lcg_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


# Blocks of the N = 131072 [A|b] (NB = 512) whose LCG state indices i + j N
# run up to 1.7e10, far past 2^32: as the local columns of processes of a
# 1 x 256 grid, where process q owns column block q and process 0 also owns
# block 256 (the single column b).
C2_N, C2_NB, C2_Q = 131072, 512, 256
C2_BLOCKS = [("first column block", 0, 0, 0, 512), ("column b", 0, 512, 131072, 1),
             ("middle column block", 128, 0, 65536, 512),
             ("last column block", 255, 0, 130560, 512)]


def make_lcg_c2(outdir: str) -> None:
    """The reference's own generator (HPL_pdrandmat on a CUDA device) for the
    N = 131072 blocks above: FNV-1a hash plus sampled entries of each."""
    import torch

    R = O.ref()
    assert R is not None, "oracle/_ref/libhplref.so not built"
    rng = np.random.default_rng(131072)
    n_cols = C2_N + 1
    out = {"n": C2_N, "nb": C2_NB, "seed": 100, "q": C2_Q, "blocks": []}
    local = {}
    for mycol in sorted({b[1] for b in C2_BLOCKS}):
        nq = 513 if mycol == 0 else 512
        dA = torch.zeros(C2_N * nq, dtype=torch.float64, device="cuda")
        rc = R.ref_pdrandmat_grid(C2_N, n_cols, C2_NB, dA.data_ptr(), C2_N, 100, 1, C2_Q, 0,
                                  mycol)
        assert rc == 0, rc
        local[mycol] = np.asfortranarray(dA.view(nq, C2_N).T.cpu().numpy())
        del dA
    for name, mycol, lc0, gc0, w in C2_BLOCKS:
        A = np.asfortranarray(local[mycol][:, lc0:lc0 + w])
        h = O.hash_block(A, C2_N, w)
        ii = rng.integers(0, C2_N, 24)
        jj = rng.integers(0, w, 24)
        samples = [[int(i), int(gc0 + j), A[i, j].hex()] for i, j in zip(ii, jj)]
        samples += [[C2_N - 1, gc0 + w - 1, A[C2_N - 1, w - 1].hex()]]
        out["blocks"].append({"name": name, "col0": gc0, "ncols": w, "fnv1a": f"{h:016x}",
                              "samples": samples})
        print(name, gc0, w, f"{h:016x}")
    with open(os.path.join(outdir, "lcg_c2_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


def make_jump(outdir: str) -> None:
    R = O.ref()
    out = []
    for k in [1, 2, 3, 7, 32, 100, 4096, 4097, 131072, 1000003]:
        m, a, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        R.ref_xjumpm(k, 6364136223846793005, 1, 100, C.byref(m), C.byref(a), C.byref(c))
        out.append({"k": k, "a": f"{a.value:016x}", "c": f"{c.value:016x}",
                    "x_from_100": f"{m.value:016x}"})
    with open(os.path.join(outdir, "jump_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


def make_perm(outdir: str) -> None:
    R = O.ref()
    rng = np.random.default_rng(2024)
    out = []
    for t in range(60):
        jb = int(rng.integers(1, 96))
        ia = int(rng.integers(0, 1000))
        M = jb + int(rng.integers(0, 300))
        ipiv = np.array([ia + i + int(rng.integers(0, M - i)) for i in range(jb)], dtype=np.int32)
        if t % 5 == 0:  # no interchanges at all
            ipiv = np.arange(ia, ia + jb, dtype=np.int32)
        permU = np.zeros(2 * jb, dtype=np.int32)
        R.ref_swapids(ia, jb, ipiv.ctypes.data, permU.ctypes.data)
        out.append({"ia": ia, "ipiv": ipiv.tolist(), "permU": permU.tolist()})
    with open(os.path.join(outdir, "perm_golden.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--lcg", action="store_true", help="also run the reference LCG on a GPU")
    ap.add_argument("--lcg-c2", action="store_true",
                    help="only the N = 131072 blocks of the reference LCG (needs a GPU)")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if a.lcg_c2:
        make_lcg_c2(a.out)
        sys.exit(0)
    make_jump(a.out)
    make_perm(a.out)
    if a.lcg:
        make_lcg(a.out)
