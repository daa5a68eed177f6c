"""A host backend for rochpl_b200.grid (test infrastructure): each process's
local work done by the oracle's restatement of the reference's building blocks
(hplo_matgen_block, hplo_panel_factor = HPL_pdfact, hplo_panel_update =
HPL_pdupdateTT) and a numpy back-solve block, on CPU torch tensors.  With it the
1 x Q driver runs with gloo ranks or threads on a machine without a GPU."""
import numpy as np


def _np(t):
    return t.numpy()


class HostBackend:
    def __init__(self, oracle):
        self.L = oracle.lib()

    def matgen_block(self, n, g0, w, seed, A, ld, lc):
        a = _np(A)
        self.L.hplo_matgen_block(n, 0, g0, n, w, seed, a.ctypes.data + 8 * lc * ld, ld)

    def panel_factor(self, algo, n, j, jb, A, ld, lc, ipiv):
        return self.L.hplo_panel_factor(n, j, jb, algo.nbmin, algo.ndiv, algo.pfact, algo.rfact,
                                        _np(A).ctypes.data, ld, lc, _np(ipiv).ctypes.data)

    def update(self, n, j, jb, Lp, ldl, ipiv, A, ld, c0, ncols):
        if ncols > 0:
            self.L.hplo_panel_update(n, j, jb, _np(Lp).ctypes.data, ldl, _np(ipiv).ctypes.data,
                                     _np(A).ctypes.data, ld, c0, ncols)

    def trsv_block(self, n, j, jb, A, ld, lc, y, s, x, z):
        a = _np(A)
        nq = a.size // ld
        F = a[: ld * nq].reshape(nq, ld).T  # ld x nq, column-major view
        U = np.triu(F[j:j + jb, lc:lc + jb])
        xb = np.linalg.solve(U, _np(y)[j:j + jb] - _np(s)[:jb])
        _np(x)[j:j + jb] = xb
        if j > 0:
            _np(z)[:j] += F[:j, lc:lc + jb] @ xb


def local_to_global(grid, A, ld):
    """The n x (n+1) block of this process's columns, placed at their global
    column positions (other columns NaN)."""
    a = _np(A)
    nq = grid.nq
    F = a[: ld * nq].reshape(nq, ld).T
    out = np.full((grid.n, grid.n + 1), np.nan)
    for lc, g0, w in grid.local_blocks():
        out[:, g0:g0 + w] = F[:grid.n, lc:lc + w]
    return out
