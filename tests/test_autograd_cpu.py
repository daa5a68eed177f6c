"""The differentiable solve's host-side logic on CPU: the adjoint's
Abar = -Bbar X^T split into hplb_rank_k calls of at most 64 right-hand sides
(pointer offsets, leading dimensions, store then accumulate), through a
stand-in for the library that does each call's arithmetic on host memory."""
import pytest
import torch

from rochpl_b200.autograd import RANK_K_MAX, _rank_k_chunks


class FakeRankK:
    """hplb_rank_k on CPU tensors: C = alpha A B^T (or C += ...), A m x k,
    B n x k, C m x n, column-major at raw addresses inside the given tensors."""

    def __init__(self, *tensors):
        self.tensors = tensors
        self.calls = []

    def _cols(self, ptr, rows, cols, ld):
        """(cols, rows) view: [c, r] = element (r, c) of the matrix at ptr."""
        for t in self.tensors:
            flat = t.view(-1)
            base = flat.data_ptr()
            if base <= ptr < base + 8 * flat.numel():
                off = (ptr - base) // 8
                assert (ptr - base) % 8 == 0
                assert off + (cols - 1) * ld + rows <= flat.numel()
                return flat.as_strided((cols, rows), (ld, 1), flat.storage_offset() + off)
        raise AssertionError(f"address {ptr:#x} is in none of the tensors")

    def rank_k(self, m, n, k, alpha, A, lda, B, ldb, C, ldc, accumulate=False):
        assert 0 <= k <= RANK_K_MAX and lda >= m and ldb >= n and ldc >= m
        self.calls.append((k, bool(accumulate)))
        Cv = self._cols(C, m, n, ldc)
        if k == 0:
            prod = torch.zeros(n, m, dtype=torch.float64)
        else:
            prod = alpha * (self._cols(B, n, k, ldb).T @ self._cols(A, m, k, lda))
        if accumulate:
            Cv += prod
        else:
            Cv.copy_(prod)


@pytest.mark.parametrize("nrhs", [0, 1, 63, 64, 65, 128, 150])
def test_adjoint_rank_k_in_chunks_of_64(nrhs):
    n = 37
    g = torch.Generator().manual_seed(nrhs)
    Bc = torch.rand(nrhs, n, generator=g, dtype=torch.float64)  # Bbar, column by column
    Xc = torch.rand(nrhs, n, generator=g, dtype=torch.float64)  # X, column by column
    Ac = torch.full((n, n), float("nan"), dtype=torch.float64)
    lib = FakeRankK(Bc, Xc, Ac)
    _rank_k_chunks(lib, n, nrhs, Bc, Xc, Ac)
    want = -(Bc.T @ Xc)  # Abar = -Bbar X^T, n x n
    assert torch.allclose(Ac.t(), want, rtol=1e-13, atol=1e-13)
    chunks = max(1, -(-nrhs // RANK_K_MAX))
    assert len(lib.calls) == chunks
    assert [a for _, a in lib.calls] == [False] + [True] * (chunks - 1)
    assert sum(k for k, _ in lib.calls) == nrhs
