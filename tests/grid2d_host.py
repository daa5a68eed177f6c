"""A host backend for rochpl_b200.grid2d (test infrastructure): each
process's local work on CPU torch tensors with numpy / scipy -- the LCG block
generator of the oracle, the column arg-max and rank-1 step of the HPL leaf,
GEMM, and the triangular solves -- so the P x Q driver runs with gloo ranks or
threads on a machine without a GPU."""
import numpy as np
from numpy.lib.stride_tricks import as_strided
from scipy.linalg import solve_triangular


def _mat(t, off, m, n, ld):
    a = t.numpy()
    return as_strided(a[off:], shape=(m, n), strides=(8, 8 * ld))


class HostBackend2D:
    def __init__(self, oracle):
        self.L = oracle.lib()

    def matgen_block(self, n, i0, j0, m, w, seed, A, ld, lr, lc):
        a = A.numpy()
        self.L.hplo_matgen_block(n, i0, j0, m, w, seed, a.ctypes.data + 8 * (lr + lc * ld), ld)

    def col_argmax(self, A, ld, r0, r1, c):
        if r1 <= r0:
            return 0.0, -1
        col = A.numpy()[r0 + c * ld: r1 + c * ld]
        i = int(np.argmax(np.abs(col)))  # the first (lowest) row among equal maxima
        return float(col[i]), r0 + i

    def col_rank1(self, A, ld, r0, r1, c0, k, kend, piv, u):
        if r1 <= r0:
            return
        M = _mat(A, r0 + c0 * ld, r1 - r0, kend, ld)
        uu = u.numpy()
        lcol = M[:, k] / piv
        M[:, k] = lcol
        for c in range(k + 1, kend):
            M[:, c] -= lcol * uu[c]

    def gemm_sub(self, m, n, k, A, lda, ao, B, ldb, bo, C, ldc, co):
        if m > 0 and n > 0 and k > 0:
            Cm = _mat(C, co, m, n, ldc)
            Cm -= _mat(A, ao, m, k, lda) @ _mat(B, bo, k, n, ldb)

    def trsm_lower_unit(self, n, nrhs, L, ldl, lo, X, ldx, xo):
        if n > 0 and nrhs > 0:
            Xm = _mat(X, xo, n, nrhs, ldx)
            Xm[:] = solve_triangular(_mat(L, lo, n, n, ldl), Xm, lower=True, unit_diagonal=True)

    def upper_solve(self, U, ldu, uo, n, y, x):
        x.numpy()[:n] = solve_triangular(_mat(U, uo, n, n, ldu), y.numpy()[:n], lower=False)


def local_to_global_2d(grid, A, ld):
    """The n x (n+1) blocks this process holds, at their global positions
    (other entries NaN)."""
    out = np.full((grid.n, grid.n + 1), np.nan)
    a = A.numpy()
    for lr, i0, h in grid.row_blocks():
        for lc, j0, w in grid.col_blocks():
            out[i0:i0 + h, j0:j0 + w] = _mat(A, lr + lc * ld, h, w, ld)
    return out


class FakeDeviceLib:
    """The Library methods DeviceBackend2D calls, with the C ABI's pointer
    arguments, done on host memory with numpy: runs the device backend's
    argument mapping (offsets, leading dimensions, sizes) on CPU tensors."""

    def __init__(self, oracle):
        self.L = oracle.lib()

    @staticmethod
    def _mat(ptr, m, n, ld):
        import ctypes

        size = (n - 1) * ld + m if m > 0 and n > 0 else 0
        if size == 0:
            return np.zeros((max(m, 0), max(n, 0)))
        a = np.ctypeslib.as_array((ctypes.c_double * size).from_address(ptr))
        return as_strided(a, shape=(m, n), strides=(8, 8 * ld))

    def matgen_block(self, mg, ng, i0, j0, m, n, seed, A, ld):
        self.L.hplo_matgen_block(mg, i0, j0, m, n, seed, A, ld)

    def col_argmax(self, A, ld, r0, r1, col):
        if r1 <= r0:
            return 0.0, -1
        c = self._mat(A + 8 * (col * ld + r0), r1 - r0, 1, ld)[:, 0]
        i = int(np.argmax(np.abs(c)))
        return float(c[i]), r0 + i

    def col_rank1(self, A, ld, r0, r1, c0, k, kend, piv, u):
        M = self._mat(A + 8 * (r0 + c0 * ld), r1 - r0, kend, ld)
        uu = self._mat(u, kend, 1, kend)[:, 0]
        lcol = M[:, k] / piv
        M[:, k] = lcol
        for c in range(k + 1, kend):
            M[:, c] -= lcol * uu[c]

    def dgemm_sub(self, m, n, k, A, lda, B, ldb, C, ldc):
        Cm = self._mat(C, m, n, ldc)
        Cm -= self._mat(A, m, k, lda) @ self._mat(B, k, n, ldb)

    def trsm_lower_unit(self, n, nrhs, L, ldl, X, ldx):
        Xm = self._mat(X, n, nrhs, ldx)
        Xm[:] = solve_triangular(self._mat(L, n, n, ldl), Xm, lower=True, unit_diagonal=True)

    def trsm_upper(self, n, nrhs, U, ldu, Y, ldy, X, ldx):
        self._mat(X, n, nrhs, ldx)[:] = solve_triangular(self._mat(U, n, n, ldu),
                                                          self._mat(Y, n, nrhs, ldy), lower=False)
