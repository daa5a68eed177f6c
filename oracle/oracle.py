"""ctypes front end of the C oracle (hpl_oracle.c) and of the reference-pinning
library built from rocHPL's own sources (oracle/_ref/libhplref.so).

Test infrastructure only: used by tests/, the smoke check and the CPU-baseline
leg of bench.py, never by the product path.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhpl_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libhplref.so")

_lib = None
_ref = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="F_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile the oracle (and, where the reference tree exists, _ref)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.hplo_jump.argtypes = [C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.hplo_lcg_value.argtypes = [C.c_uint64]
        L.hplo_lcg_value.restype = C.c_double
        L.hplo_lcg_state.argtypes = [C.c_uint64, C.c_int64, C.c_int64, C.c_int64]
        L.hplo_lcg_state.restype = C.c_uint64
        L.hplo_matgen.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_void_p, C.c_int64]
        L.hplo_matgen_block.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int,
                                        C.c_uint64, C.c_void_p, C.c_int64]
        L.hplo_hash.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.hplo_hash.restype = C.c_uint64
        L.hplo_use_blas.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.hplo_use_blas.restype = C.c_int
        L.hplo_pdgesv.argtypes = [C.c_int] * 6 + [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.hplo_pdgesv.restype = C.c_int
        L.hplo_panel_factor.argtypes = [C.c_int] * 7 + [C.c_void_p, C.c_int64, C.c_int,
                                                        C.c_void_p]
        L.hplo_panel_factor.restype = C.c_int
        L.hplo_panel_update.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64,
                                        C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int]
        L.hplo_swapids.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.hplo_residual.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.hplo_hpl_test.argtypes = [C.c_int] * 6 + [C.c_uint64, C.c_void_p, C.c_int64,
                                                    C.c_void_p, C.c_void_p, C.c_void_p]
        L.hplo_hpl_test.restype = C.c_int
        _lib = L
    return _lib


def ref():
    """The reference-pinning library, or None when it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        R = C.CDLL(REF_PATH)
        R.ref_pdrandmat.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
        R.ref_pdrandmat.restype = C.c_int
        R.ref_pdrandmat_grid.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                         C.c_int, C.c_int, C.c_int, C.c_int]
        R.ref_pdrandmat_grid.restype = C.c_int
        R.ref_xjumpm.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                 C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        R.ref_pipid.argtypes = [C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int), C.c_void_p]
        R.ref_swapids.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        R.ref_dlaswp00N.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        R.ref_dlaswp00N.restype = C.c_int
        _ref = R
    return _ref


def default_ld(n: int) -> int:
    """rocHPL's padded leading dimension (src/matgen/HPL_pdmatgen.cpp:109-110)."""
    return ((max(1, n) + 95) // 128) * 128 + 32


def jump(k: int) -> tuple[int, int]:
    a, c = C.c_uint64(), C.c_uint64()
    lib().hplo_jump(k, C.byref(a), C.byref(c))
    return a.value, c.value


def lcg_value(state: int) -> float:
    return lib().hplo_lcg_value(state)


def lcg_state(seed: int, m: int, i: int, j: int) -> int:
    return lib().hplo_lcg_state(seed, m, i, j)


def matgen(m: int, n: int, seed: int = 100, ld: int | None = None) -> np.ndarray:
    """HPL_pdrandmat at P=Q=1: an ld x n Fortran-ordered array, rows >= m zero."""
    ld = ld or m
    A = np.zeros((ld, n), dtype=np.float64, order="F")
    lib().hplo_matgen(m, n, seed, A.ctypes.data, ld)
    return A


def matgen_block(M: int, i0: int, j0: int, m: int, n: int, seed: int = 100) -> np.ndarray:
    """Rows [i0, i0+m) x columns [j0, j0+n) of the M-row LCG matrix (m x n,
    Fortran order)."""
    A = np.zeros((max(m, 1), max(n, 1)), dtype=np.float64, order="F")
    lib().hplo_matgen_block(M, i0, j0, m, n, seed, A.ctypes.data, max(m, 1))
    return A[:m, :n]


def hash_block(A: np.ndarray, m: int, n: int) -> int:
    A = np.asfortranarray(A)
    return lib().hplo_hash(m, n, A.ctypes.data, A.shape[0])


_blas_loaded = None


def use_blas(nthreads: int = 0) -> bool:
    """Route the oracle's dgemm/dtrsm to the host OpenBLAS shipped with scipy
    (LP64, 'scipy_' prefix).  Returns False when no such library is found."""
    global _blas_loaded
    import scipy

    cands = sorted(glob.glob(os.path.join(os.path.dirname(scipy.__file__), os.pardir,
                                          "scipy.libs", "libscipy_openblas-*.so")))
    for c in cands:
        if lib().hplo_use_blas(c.encode(), b"scipy_", nthreads or os.cpu_count()) == 0:
            _blas_loaded = c
            return True
    return False


def no_blas() -> None:
    global _blas_loaded
    lib().hplo_use_blas(None, None, 0)
    _blas_loaded = None


def pdgesv(A: np.ndarray, n: int, nb: int, nbmin: int = 32, ndiv: int = 2,
           pfact: int = 2, rfact: int = 2):
    """Factor [A|b] in place (Fortran array, >= n rows, >= n+1 columns) and
    back-solve.  Returns (x, ipiv, info)."""
    assert A.flags.f_contiguous and A.dtype == np.float64
    x = np.zeros(max(n, 1), dtype=np.float64)
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    info = lib().hplo_pdgesv(n, nb, nbmin, ndiv, pfact, rfact, A.ctypes.data, A.shape[0],
                             x.ctypes.data, ipiv.ctypes.data)
    return x[:n], ipiv[:n], info


def swapids(ia: int, ipiv) -> np.ndarray:
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int32)
    jb = len(ipiv)
    out = np.zeros(2 * max(jb, 1), dtype=np.int32)
    lib().hplo_swapids(ia, jb, ipiv.ctypes.data, out.ctypes.data)
    return out[: 2 * jb]


def residual(A: np.ndarray, n: int, x) -> dict:
    """HPL scaled residual of x against the (regenerated) [A|b]."""
    A = np.asfortranarray(A)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(8)
    r = np.zeros(max(n, 1))
    lib().hplo_residual(n, A.ctypes.data, A.shape[0], x.ctypes.data, out.ctypes.data, r.ctypes.data)
    keys = ["resid", "rnorm_inf", "anorm_1", "anorm_inf", "xnorm_1", "xnorm_inf", "bnorm_inf", "eps"]
    d = dict(zip(keys, out.tolist()))
    d["r"] = r[:n]
    return d


def hpl_test(n: int, nb: int, nbmin: int = 32, ndiv: int = 2, pfact: int = 2, rfact: int = 2,
             seed: int = 100):
    """Generate, solve, regenerate and check, all on the host."""
    ld = default_ld(n)
    A = np.zeros((ld, n + 1), dtype=np.float64, order="F")
    x = np.zeros(max(n, 1))
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    res = np.zeros(8)
    info = lib().hplo_hpl_test(n, nb, nbmin, ndiv, pfact, rfact, seed, A.ctypes.data, ld,
                               x.ctypes.data, ipiv.ctypes.data, res.ctypes.data)
    return x[:n], ipiv[:n], info, float(res[0])
