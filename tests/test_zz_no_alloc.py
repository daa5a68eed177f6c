"""The allocation-free residual check, hplb_residual_lcg_noalloc.

It serves callers that must not allocate device memory (all of it handed to
their own pool, or a check between solves where cudaMalloc's implicit
synchronisation is not allowed): its scratch is a fixed array in the library
image.  Compared through the C ABI with the context-based hplb_residual_lcg on
the same solution, twice in a row (the array keeps the previous call's
contents), and checked to reject n above its limit.  The file name sorts last
so a run stopping at the first failure has run every other test first.
"""
import pytest

pytestmark = pytest.mark.gpu


def _solution(n, nb=128):
    import torch

    from rochpl_b200 import library
    from rochpl_b200.hpl import Algo, default_ld

    lib = library(0)
    ld = default_ld(n)
    dA = torch.empty(ld * (n + 1), dtype=torch.float64, device="cuda")
    dX = torch.zeros(n, dtype=torch.float64, device="cuda")
    lib.matgen(n, n + 1, 100, dA.data_ptr(), ld, nb)
    lib.pdgesv(Algo(nb, 32, 2, 2, 2, 1, 0).c(), n, dA.data_ptr(), ld, dX.data_ptr())
    return lib, dX


@pytest.mark.parametrize("n", [1000, 4096, 16384])
def test_noalloc_matches_context_residual_twice(n):
    """n = 16384 is the limit itself: every chunk of the array's layout, the
    table block and the output slot at its end are in use."""
    from rochpl_b200.lib import HPLB_OK, residual_lcg_noalloc

    lib, dX = _solution(n)
    ref = lib.residual_lcg(n, 100, dX.data_ptr())
    for _ in range(2):
        st, got = residual_lcg_noalloc(n, 100, dX.data_ptr())
        assert st == HPLB_OK
        for k in ref:
            # Same kernels in the same order: equal to rounding (bit-equal in practice).
            assert got[k] == pytest.approx(ref[k], rel=1e-13, abs=1e-300), k
        assert got["resid"] < 16.0


def test_noalloc_after_a_different_size_call():
    from rochpl_b200.lib import HPLB_OK, residual_lcg_noalloc

    lib, dX = _solution(2048)
    _, big = _solution(4096)
    assert residual_lcg_noalloc(4096, 100, big.data_ptr())[0] == HPLB_OK
    ref = lib.residual_lcg(2048, 100, dX.data_ptr())
    st, got = residual_lcg_noalloc(2048, 100, dX.data_ptr())
    assert st == HPLB_OK
    for k in ref:
        assert got[k] == pytest.approx(ref[k], rel=1e-13, abs=1e-300), k


def test_noalloc_rejects_sizes_above_its_limit():
    import torch

    from rochpl_b200.lib import HPLB_ERR_ARG, load, residual_lcg_noalloc

    load()
    x = torch.zeros(16385, dtype=torch.float64, device="cuda")
    assert residual_lcg_noalloc(16385, 100, x.data_ptr())[0] == HPLB_ERR_ARG
