"""ctypes binding of libhplb200.so (include/hplb.h).

Every entry point declared in the header is bound here with its exact C
signature; device buffers are passed as raw integer addresses (for example a
torch CUDA tensor's data_ptr()).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhplb200.so")

HPLB_OK = 0
HPLB_ERR_ARG = 1
HPLB_ERR_OOM = 2
HPLB_ERR_SINGULAR = 3
HPLB_ERR_TIMEOUT = 4
HPLB_ERR_CUDA = 5
HPLB_ERR_UNSUPPORTED = 6

# Every symbol include/hplb.h declares (checked by the CPU test suite).
EXPORTS = [
    "hplb_create", "hplb_destroy", "hplb_status_string", "hplb_last_error",
    "hplb_default_ld", "hplb_matgen", "hplb_matgen_block", "hplb_pdgesv", "hplb_residual",
    "hplb_residual_lcg", "hplb_last_timing", "hplb_last_steps", "hplb_dgemm_sub", "hplb_laswp_trsm",
    "hplb_fp64_peak", "hplb_selftest_wait_timeout", "hplb_residual_lcg_noalloc",
    "hplb_gemm_lp_sub", "hplb_pdgesv_mixed", "hplb_getrf", "hplb_getrs", "hplb_rank_k",
    "hplb_set_stream", "hplb_set_option", "hplb_batch_create", "hplb_batch_destroy", "hplb_batch_layout",
    "hplb_batch_matgen", "hplb_batch_gesv", "hplb_batch_getrs", "hplb_batch_rank_k",
    "hplb_batch_residual", "hplb_batch_last_ms", "hplb_batch_tune",
    "hplb_panel_factor", "hplb_panel_update", "hplb_trsv_block", "hplb_gesv",
    "hplb_col_argmax", "hplb_col_rank1", "hplb_trsm_lower_unit", "hplb_trsm_upper",
]

HPLB_BATCH_CLASSES = 6
HPLB_BATCH_MAX_N = 2048
HPLB_BATCH_RECURSIVE = 64
HPLB_BATCH_RECURSIVE_MAX_N = 1024


class hplb_algo(C.Structure):
    _fields_ = [("nb", C.c_int), ("nbmin", C.c_int), ("ndiv", C.c_int), ("pfact", C.c_int),
                ("rfact", C.c_int), ("depth", C.c_int), ("l1notran", C.c_int)]


class hplb_resid(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("resid", "rnorm_inf", "anorm_1", "anorm_inf",
                                          "xnorm_1", "xnorm_inf", "bnorm_inf", "eps")]


class hplb_timing(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("lu_ms", C.c_double), ("trsv_ms", C.c_double),
                ("gemm_ms", C.c_double), ("gemm_flops", C.c_double), ("panel_ms", C.c_double),
                ("gemm_launches", C.c_int), ("kernel_launches", C.c_int)]


class hplb_mixed_opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("restart", C.c_int), ("max_outer", C.c_int),
                ("target_resid", C.c_double), ("gmres_tol", C.c_double)]


class hplb_mixed_report(C.Structure):
    _fields_ = [("resid", C.c_double), ("resid_lu", C.c_double), ("outer_iters", C.c_int),
                ("gmres_iters", C.c_int), ("converged", C.c_int), ("info", C.c_int),
                ("lu_ms", C.c_double), ("ir_ms", C.c_double), ("total_ms", C.c_double),
                ("gemm_ms", C.c_double), ("gemm_flops", C.c_double), ("panel_ms", C.c_double)]


# hplb_mixed_opts.precision values
PREC_BF16, PREC_FP16, PREC_BF16X3, PREC_FP16X3 = 0, 1, 2, 3

# hplb_set_option options and values
HPLB_OPT_LEAF = 1
LEAF_AUTO, LEAF_SHARED, LEAF_GLOBAL, LEAF_REGISTERS = 0, 1, 2, 3
HPLB_OPT_PANEL_SMS, PANEL_SMS_AUTO = 2, -1


class HplError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"hplb status {status}: {message}")
        self.status = status


_lib = None


def load() -> C.CDLL:
    """Load libhplb200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m rochpl_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, u64 = C.c_void_p, C.c_int64, C.c_int, C.c_uint64
    L.hplb_create.argtypes = [i32, C.POINTER(C.c_int)]
    L.hplb_create.restype = vp
    L.hplb_destroy.argtypes = [vp]
    L.hplb_destroy.restype = None
    L.hplb_status_string.argtypes = [i32]
    L.hplb_status_string.restype = C.c_char_p
    L.hplb_last_error.argtypes = [vp]
    L.hplb_last_error.restype = C.c_char_p
    L.hplb_default_ld.argtypes = [i32]
    L.hplb_default_ld.restype = i64
    L.hplb_matgen.argtypes = [vp, i32, i32, i32, u64, vp, i64]
    L.hplb_matgen_block.argtypes = [vp, i64, i64, i64, i64, i32, i32, u64, vp, i64]
    L.hplb_matgen_block.restype = i32
    L.hplb_pdgesv.argtypes = [vp, C.POINTER(hplb_algo), i32, vp, i64, vp, vp, C.POINTER(C.c_int)]
    L.hplb_residual.argtypes = [vp, i32, vp, i64, vp, C.POINTER(hplb_resid)]
    L.hplb_residual_lcg.argtypes = [vp, i32, u64, vp, C.POINTER(hplb_resid)]
    L.hplb_last_timing.argtypes = [vp, C.POINTER(hplb_timing)]
    L.hplb_last_steps.argtypes = [vp, i32, C.POINTER(C.c_int), vp, vp]
    L.hplb_last_steps.restype = i32
    L.hplb_dgemm_sub.argtypes = [vp, i32, i32, i32, vp, i64, vp, i64, vp, i64]
    L.hplb_laswp_trsm.argtypes = [vp, vp, i64, i32, i32, i32, vp, i32, i32]
    L.hplb_fp64_peak.argtypes = [vp, i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.hplb_selftest_wait_timeout.argtypes = [vp, u64]
    L.hplb_residual_lcg_noalloc.argtypes = [i32, u64, vp, vp, C.POINTER(hplb_resid)]
    L.hplb_residual_lcg_noalloc.restype = i32
    L.hplb_gemm_lp_sub.argtypes = [vp, i32, i32, i32, i32, vp, i64, vp, i64, vp, vp, vp, i64]
    L.hplb_gemm_lp_sub.restype = i32
    L.hplb_pdgesv_mixed.argtypes = [vp, C.POINTER(hplb_algo), C.POINTER(hplb_mixed_opts), i32, vp,
                                    i64, u64, vp, vp, C.POINTER(hplb_mixed_report)]
    L.hplb_pdgesv_mixed.restype = i32
    ip, i64p, u64p, dp = (C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_uint64),
                          C.POINTER(C.c_double))
    L.hplb_batch_create.argtypes = [vp, i32, ip, ip, ip, C.POINTER(vp)]
    L.hplb_batch_destroy.argtypes = [vp]
    L.hplb_batch_destroy.restype = None
    L.hplb_batch_layout.argtypes = [vp, i64p, i64p, i64p, i64p, i64p, i64p, ip]
    L.hplb_batch_matgen.argtypes = [vp, u64p, vp, vp]
    L.hplb_batch_gesv.argtypes = [vp, vp, vp, vp, vp]
    L.hplb_batch_getrs.argtypes = [vp, i32, vp, vp, vp]
    L.hplb_batch_rank_k.argtypes = [vp, C.c_double, vp, vp, vp]
    L.hplb_batch_residual.argtypes = [vp, u64p, vp, vp]
    L.hplb_batch_last_ms.argtypes = [vp, dp]
    L.hplb_batch_tune.argtypes = [vp, i32, ip, dp]
    for name in ("hplb_batch_create", "hplb_batch_layout", "hplb_batch_matgen", "hplb_batch_gesv",
                 "hplb_batch_getrs", "hplb_batch_rank_k", "hplb_batch_residual",
                 "hplb_batch_last_ms", "hplb_batch_tune"):
        getattr(L, name).restype = i32
    L.hplb_set_stream.argtypes = [vp, vp]
    L.hplb_set_stream.restype = i32
    L.hplb_set_option.argtypes = [vp, i32, i32]
    L.hplb_set_option.restype = i32
    L.hplb_getrf.argtypes = [vp, C.POINTER(hplb_algo), i32, vp, i64, vp, C.POINTER(C.c_int)]
    L.hplb_getrf.restype = i32
    L.hplb_getrs.argtypes = [vp, i32, i32, i32, i32, vp, i64, vp, vp, i64]
    L.hplb_getrs.restype = i32
    L.hplb_gesv.argtypes = [vp, C.POINTER(hplb_algo), i32, i32, vp, i64, vp, i64, vp,
                            C.POINTER(C.c_int)]
    L.hplb_gesv.restype = i32
    L.hplb_col_argmax.argtypes = [vp, vp, i64, i32, i32, i32, C.POINTER(C.c_double),
                                  C.POINTER(C.c_int)]
    L.hplb_col_rank1.argtypes = [vp, vp, i64, i32, i32, i32, i32, i32, C.c_double, vp]
    L.hplb_trsm_lower_unit.argtypes = [vp, i32, i32, vp, i64, vp, i64]
    L.hplb_trsm_upper.argtypes = [vp, i32, i32, vp, i64, vp, i64, vp, i64]
    for name in ("hplb_col_argmax", "hplb_col_rank1", "hplb_trsm_lower_unit", "hplb_trsm_upper"):
        getattr(L, name).restype = i32
    L.hplb_panel_factor.argtypes = [vp, C.POINTER(hplb_algo), i32, i32, i32, vp, i64, i32, vp,
                                    C.POINTER(C.c_int)]
    L.hplb_panel_factor.restype = i32
    L.hplb_panel_update.argtypes = [vp, i32, i32, i32, vp, i64, vp, vp, i64, i32, i32]
    L.hplb_panel_update.restype = i32
    L.hplb_trsv_block.argtypes = [vp, i32, i32, i32, vp, i64, i32, vp, vp, vp, vp]
    L.hplb_trsv_block.restype = i32
    L.hplb_rank_k.argtypes = [vp, i32, i32, i32, C.c_double, vp, i64, vp, i64, vp, i64, i32]
    L.hplb_rank_k.restype = i32
    for name in ("hplb_fp64_peak", "hplb_selftest_wait_timeout", "hplb_matgen", "hplb_pdgesv", "hplb_residual", "hplb_residual_lcg",
                 "hplb_last_timing", "hplb_dgemm_sub", "hplb_laswp_trsm"):
        getattr(L, name).restype = i32
    _lib = L
    return L


class Library:
    """One hplb context (device, streams, workspaces) on one CUDA device."""

    def __init__(self, device: int = 0):
        self.L = load()
        st = C.c_int(0)
        self.ctx = self.L.hplb_create(device, C.byref(st))
        if not self.ctx:
            raise HplError(st.value, "hplb_create failed: "
                           + self.L.hplb_status_string(st.value).decode())
        self.device = device

    def close(self):
        if getattr(self, "ctx", None):
            self.L.hplb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, allow=(HPLB_OK,)) -> int:
        if st not in allow:
            raise HplError(st, self.L.hplb_last_error(self.ctx).decode())
        return st

    def matgen(self, m: int, n: int, seed: int, A: int, ld: int, nb: int = 0):
        self._check(self.L.hplb_matgen(self.ctx, m, n, nb, seed, A, ld))

    def matgen_block(self, mg: int, ng: int, i0: int, j0: int, m: int, n: int, seed: int,
                     A: int, ld: int):
        """Rows [i0, i0+m) x columns [j0, j0+n) of the mg x ng LCG matrix."""
        self._check(self.L.hplb_matgen_block(self.ctx, mg, ng, i0, j0, m, n, seed, A, ld))

    def pdgesv(self, algo: hplb_algo, n: int, A: int, ld: int, X: int, ipiv: int | None = None):
        info = C.c_int(0)
        st = self.L.hplb_pdgesv(self.ctx, C.byref(algo), n, A, ld, X, ipiv or None,
                                C.byref(info))
        self._check(st, allow=(HPLB_OK, HPLB_ERR_SINGULAR))
        return info.value

    def gesv(self, algo: hplb_algo, n: int, nrhs: int, A: int, ld: int, X: int, ldx: int,
             ipiv: int | None = None) -> int:
        """hplb_gesv: factor [A | B] (B in columns n .. n + nrhs - 1 of A) and
        write X = A^-1 B (n x nrhs, leading dimension ldx); returns info."""
        info = C.c_int(0)
        st = self.L.hplb_gesv(self.ctx, C.byref(algo), n, nrhs, A, ld, X, ldx, ipiv or None,
                              C.byref(info))
        self._check(st, allow=(HPLB_OK, HPLB_ERR_SINGULAR))
        return info.value

    def col_argmax(self, A: int, ld: int, r0: int, r1: int, col: int) -> tuple[float, int]:
        """hplb_col_argmax: (value, row) of the largest |A[r, col]|, r in [r0, r1)."""
        v, r = C.c_double(0.0), C.c_int(-1)
        self._check(self.L.hplb_col_argmax(self.ctx, A, ld, r0, r1, col, C.byref(v), C.byref(r)))
        return v.value, r.value

    def col_rank1(self, A: int, ld: int, r0: int, r1: int, c0: int, k: int, kend: int,
                  piv: float, u: int):
        self._check(self.L.hplb_col_rank1(self.ctx, A, ld, r0, r1, c0, k, kend, piv, u))

    def trsm_lower_unit(self, n: int, nrhs: int, L: int, ldl: int, X: int, ldx: int):
        self._check(self.L.hplb_trsm_lower_unit(self.ctx, n, nrhs, L, ldl, X, ldx))

    def trsm_upper(self, n: int, nrhs: int, U: int, ldu: int, Y: int, ldy: int, X: int,
                   ldx: int):
        self._check(self.L.hplb_trsm_upper(self.ctx, n, nrhs, U, ldu, Y, ldy, X, ldx))

    def pdgesv_mixed(self, algo: hplb_algo, n: int, X: int, seed: int = 100, A: int | None = None,
                     ld: int = 0, precision: int = PREC_BF16X3, restart: int = 20,
                     max_outer: int = 20, target_resid: float = 16.0, gmres_tol: float = 1e-6,
                     ipiv: int | None = None) -> dict:
        """hplb_pdgesv_mixed: low-precision LU + GMRES refinement.  A None
        solves the LCG system of `seed` without a stored FP64 matrix.  Returns
        the report as a dict (plus "status"); a zero pivot is reported, not
        raised."""
        o = hplb_mixed_opts(precision, restart, max_outer, target_resid, gmres_tol)
        r = hplb_mixed_report()
        st = self.L.hplb_pdgesv_mixed(self.ctx, C.byref(algo), C.byref(o), n, A or None, ld,
                                      seed, X, ipiv or None, C.byref(r))
        self._check(st, allow=(HPLB_OK, HPLB_ERR_SINGULAR))
        out = {k: getattr(r, k) for k, _ in hplb_mixed_report._fields_}
        out["status"] = st
        return out

    def set_stream(self, stream: int | None):
        """Order later calls after the work queued on `stream` (a raw
        cudaStream_t, e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self.L.hplb_set_stream(self.ctx, stream or None))

    def set_leaf(self, kind: int):
        """hplb_set_option(HPLB_OPT_LEAF): LEAF_AUTO, LEAF_REGISTERS, LEAF_SHARED or
        LEAF_GLOBAL."""
        self._check(self.L.hplb_set_option(self.ctx, HPLB_OPT_LEAF, int(kind)))

    def set_panel_sms(self, sms: int):
        """hplb_set_option(HPLB_OPT_PANEL_SMS): PANEL_SMS_AUTO (-1), 0, or the
        SMs the trailing-update DGEMM leaves to the panel stream."""
        self._check(self.L.hplb_set_option(self.ctx, HPLB_OPT_PANEL_SMS, int(sms)))

    def getrf(self, algo: hplb_algo, n: int, A: int, ld: int, ipiv: int | None = None) -> int:
        """hplb_getrf: factor A alone; returns info (0, or the first zero pivot)."""
        info = C.c_int(0)
        st = self.L.hplb_getrf(self.ctx, C.byref(algo), n, A, ld, ipiv or None, C.byref(info))
        self._check(st, allow=(HPLB_OK, HPLB_ERR_SINGULAR))
        return info.value

    def getrs(self, trans: int, n: int, nb: int, nrhs: int, LU: int, ld: int, ipiv: int, B: int,
              ldb: int):
        self._check(self.L.hplb_getrs(self.ctx, int(trans), n, nb, nrhs, LU, ld, ipiv, B, ldb))

    def rank_k(self, m: int, n: int, k: int, alpha: float, A: int, lda: int, B: int, ldb: int,
               Cp: int, ldc: int, accumulate: bool = False):
        self._check(self.L.hplb_rank_k(self.ctx, m, n, k, float(alpha), A, lda, B, ldb, Cp, ldc,
                                       int(bool(accumulate))))

    def residual(self, n: int, A: int, ld: int, X: int) -> dict:
        r = hplb_resid()
        self._check(self.L.hplb_residual(self.ctx, n, A, ld, X, C.byref(r)))
        return {k: getattr(r, k) for k, _ in hplb_resid._fields_}

    def residual_lcg(self, n: int, seed: int, X: int) -> dict:
        r = hplb_resid()
        self._check(self.L.hplb_residual_lcg(self.ctx, n, seed, X, C.byref(r)))
        return {k: getattr(r, k) for k, _ in hplb_resid._fields_}

    def panel_factor(self, algo: hplb_algo, n: int, j: int, jb: int, A: int, ld: int, lc: int,
                     ipiv: int) -> int:
        """hplb_panel_factor; returns info (0, or the zero pivot's global column)."""
        info = C.c_int(0)
        st = self.L.hplb_panel_factor(self.ctx, C.byref(algo), n, j, jb, A, ld, lc, ipiv,
                                      C.byref(info))
        self._check(st, allow=(HPLB_OK, HPLB_ERR_SINGULAR))
        return info.value

    def panel_update(self, n: int, j: int, jb: int, Lp: int, ldl: int, ipiv: int, A: int,
                     ld: int, c0: int, ncols: int):
        self._check(self.L.hplb_panel_update(self.ctx, n, j, jb, Lp, ldl, ipiv, A, ld, c0,
                                             ncols))

    def trsv_block(self, n: int, j: int, jb: int, A: int, ld: int, lc: int, y: int, s: int,
                   x: int, z: int):
        self._check(self.L.hplb_trsv_block(self.ctx, n, j, jb, A, ld, lc, y, s, x, z))

    def last_timing(self) -> dict:
        t = hplb_timing()
        self._check(self.L.hplb_last_timing(self.ctx, C.byref(t)))
        return {k: getattr(t, k) for k, _ in hplb_timing._fields_}

    def last_steps(self) -> list:
        """[(first column, ms), ...] per step of the last pdgesv / getrf."""
        cnt = C.c_int(0)
        self._check(self.L.hplb_last_steps(self.ctx, 0, C.byref(cnt), None, None))
        n = cnt.value
        cols = (C.c_int * max(n, 1))()
        ms = (C.c_double * max(n, 1))()
        self._check(self.L.hplb_last_steps(self.ctx, n, C.byref(cnt), cols, ms))
        return [(int(cols[i]), float(ms[i])) for i in range(min(n, cnt.value))]

    def dgemm_sub(self, m, n, k, A, lda, B, ldb, Cp, ldc):
        self._check(self.L.hplb_dgemm_sub(self.ctx, m, n, k, A, lda, B, ldb, Cp, ldc))

    def laswp_trsm(self, A, ld, ia, jb, lc, ipiv_host, c0, n):
        arr = None
        if ipiv_host is not None:
            arr = (C.c_int * len(ipiv_host))(*[int(v) for v in ipiv_host])
        self._check(self.L.hplb_laswp_trsm(self.ctx, A, ld, ia, jb, lc, arr, c0, n))


    def gemm_lp_sub(self, bf16, m, n, k, A16, lda, B16, ldb, sA, sB, Cp, ldc):
        self._check(self.L.hplb_gemm_lp_sub(self.ctx, int(bf16), m, n, k, A16, lda, B16, ldb,
                                            sA, sB, Cp, ldc))

    def fp64_peak(self, iters: int = 20000) -> tuple[float, float]:
        a, b = C.c_double(0), C.c_double(0)
        self._check(self.L.hplb_fp64_peak(self.ctx, iters, C.byref(a), C.byref(b)))
        return a.value, b.value

    def selftest_wait_timeout(self, budget_ns: int) -> int:
        """Returns the status of a bounded wait that is made to expire."""
        return self.L.hplb_selftest_wait_timeout(self.ctx, budget_ns)


def residual_lcg_noalloc(n: int, seed: int, X: int, stream: int = 0):
    """hplb_residual_lcg_noalloc: (status, results dict); needs no context."""
    L = load()
    r = hplb_resid()
    st = L.hplb_residual_lcg_noalloc(n, seed, X, stream or None, C.byref(r))
    return st, {k: getattr(r, k) for k, _ in hplb_resid._fields_}


_default = {}


def library(device: int = 0) -> Library:
    """The process's shared context on `device` (a process drives one device:
    hplb_create refuses a second)."""
    if device not in _default:
        _default[device] = Library(device)
    return _default[device]
