"""Kernel-level parity of the CUDA path against the oracle and against
rocHPL's own matgen / row-swap code (oracle/_ref), through the C ABI."""
import json
import os

import numpy as np
import pytest

from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n", [(1, 2), (2, 3), (31, 32), (257, 258), (1000, 1001),
                                 (4096, 4097), (5000, 37), (513, 7)])
def test_matgen_bit_exact_vs_oracle(hlib, oracle, m, n):
    import torch

    ld = oracle.default_ld(m)
    dA = torch.full((ld * n,), np.nan, dtype=torch.float64, device="cuda")
    hlib.matgen(m, n, 100, dA.data_ptr(), ld)
    got = from_dev(dA, ld, n)
    ref = oracle.matgen(m, n, 100, ld=ld)
    assert np.array_equal(got[:m].view(np.uint64), ref[:m].view(np.uint64))
    assert np.all(np.isnan(got[m:]))  # padding rows untouched


@pytest.mark.parametrize("m,n,nb", [(4096, 4097, 256), (1000, 1001, 64), (33, 34, 32)])
def test_matgen_bit_exact_vs_reference_kernel(hlib, oracle, m, n, nb):
    import torch

    R = oracle.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    ld = oracle.default_ld(m)
    d1 = torch.zeros(ld * n, dtype=torch.float64, device="cuda")
    d2 = torch.zeros(ld * n, dtype=torch.float64, device="cuda")
    hlib.matgen(m, n, 100, d1.data_ptr(), ld, nb)
    assert R.ref_pdrandmat(m, n, nb, d2.data_ptr(), ld, 100) == 0
    assert torch.equal(d1.view(torch.int64), d2.view(torch.int64))


@pytest.mark.parametrize("mg,ng,i0,j0,m,n", [(1000, 1001, 0, 0, 1000, 1001),
                                              (1000, 1001, 17, 300, 500, 400),
                                              (4096, 4097, 4095, 4096, 1, 1),
                                              (5000, 37, 1234, 5, 3000, 32)])
def test_matgen_block_equals_full_matrix(hlib, oracle, mg, ng, i0, j0, m, n):
    """hplb_matgen_block is the sub-block of hplb_matgen, bit for bit, and the
    oracle's block generator agrees."""
    import torch

    ld = m + 3
    dA = torch.full((ld * n,), np.nan, dtype=torch.float64, device="cuda")
    hlib.matgen_block(mg, ng, i0, j0, m, n, 100, dA.data_ptr(), ld)
    got = from_dev(dA, ld, n)
    full = oracle.matgen(mg, ng, 100)
    assert np.array_equal(got[:m].view(np.uint64), full[i0:i0 + m, j0:j0 + n].view(np.uint64))
    assert np.array_equal(got[:m].view(np.uint64),
                          oracle.matgen_block(mg, i0, j0, m, n, 100).view(np.uint64))
    assert np.all(np.isnan(got[m:]))


def test_matgen_block_rejects_blocks_outside_the_matrix(hlib):
    from rochpl_b200.lib import HplError

    with pytest.raises(HplError):
        hlib.matgen_block(100, 101, 90, 0, 20, 1, 100, 0, 20)
    with pytest.raises(HplError):
        hlib.matgen_block(100, 101, 0, 100, 100, 2, 100, 0, 100)


C2_GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lcg_c2_golden.json")


@pytest.mark.skipif(not os.path.exists(C2_GOLD),
                    reason="made on a GPU by tests/golden/make_golden.py --lcg-c2")
def test_matgen_c2_blocks_match_reference_kernel(hlib, oracle):
    """The N = 131072 [A|b] (LCG state indices up to 1.7e10, past 2^32): the
    first, middle and last 512-column blocks and b, generated here as blocks of
    the full matrix, against the reference generator's own output (hashes and
    samples in the golden file) and against the oracle, bit for bit."""
    import torch

    g = json.load(open(C2_GOLD))
    n = g["n"]
    for b in g["blocks"]:
        c0, w = b["col0"], b["ncols"]
        dA = torch.empty(n * w, dtype=torch.float64, device="cuda")
        hlib.matgen_block(n, n + 1, 0, c0, n, w, g["seed"], dA.data_ptr(), n)
        A = from_dev(dA, n, w)
        del dA
        assert f"{oracle.hash_block(A, n, w):016x}" == b["fnv1a"], b["name"]
        for i, j, hx in b["samples"]:
            assert A[i, j - c0].hex() == hx, (b["name"], i, j)
        ref = oracle.matgen_block(n, 0, c0, n, w, g["seed"])
        assert np.array_equal(A.view(np.uint64), ref.view(np.uint64)), b["name"]


DGEMM_SHAPES = [(1, 1, 1), (7, 5, 3), (128, 128, 16), (200, 300, 512), (1000, 513, 512),
                (4097, 129, 256), (130, 4100, 33), (2048, 512, 512), (777, 1031, 64),
                (129, 129, 17)]


@pytest.mark.parametrize("m,n,k", DGEMM_SHAPES)
@pytest.mark.parametrize("offset,pad", [(0, 16), (0, 3), (1, 3)])
def test_dgemm_sub(hlib, m, n, k, offset, pad):
    """offset 0 with an even, padded leading dimension takes the TMA kernel;
    odd leading dimensions or an 8-byte offset take the cp.async kernel."""
    import torch

    g = torch.Generator(device="cpu").manual_seed(m * 7 + n + k)
    lda = m + pad + offset
    lda += lda % 2 if pad == 16 else 0
    A = torch.rand(k * lda + offset, generator=g, dtype=torch.float64) - 0.5
    B = torch.rand(n * (k + 2) + offset, generator=g, dtype=torch.float64) - 0.5
    Cm = torch.rand(n * lda + offset, generator=g, dtype=torch.float64) - 0.5
    dA, dB, dC = A.cuda(), B.cuda(), Cm.cuda()
    ldb = k + (1 if pad != 16 else 2)
    hlib.dgemm_sub(m, n, k, dA.data_ptr() + 8 * offset, lda, dB.data_ptr() + 8 * offset, ldb,
                   dC.data_ptr() + 8 * offset, lda)
    Am = A[offset:offset + k * lda].view(k, lda).T[:m]
    Bm = B[offset:offset + n * ldb].view(n, ldb).T[:k]
    Cr = Cm[offset:offset + n * lda].view(n, lda).T.clone()
    Cr[:m] -= Am @ Bm
    got = dC.cpu()[offset:offset + n * lda].view(n, lda).T
    err = (got - Cr).abs().max().item()
    assert err <= 1e-14 * k + 1e-15
    # padding rows of C untouched
    assert torch.equal(got[m:], Cm[offset:offset + n * lda].view(n, lda).T[m:])


@pytest.mark.parametrize("jb,n,rows", [(1, 3, 10), (32, 40, 200), (256, 257, 600),
                                       (512, 100, 2000), (300, 65, 900)])
def test_laswp_trsm_vs_oracle(hlib, oracle, jb, n, rows):
    """Row interchanges + unit-lower TRSM on a block of trailing columns."""
    rng = np.random.default_rng(jb + n)
    ld = rows + 5
    ia = 3
    ncols = ia + jb + n
    A = np.asfortranarray(rng.uniform(-0.5, 0.5, (ld, ncols)))
    # A well-conditioned unit-lower L11 at (ia, ia): small multipliers.
    A[ia:ia + jb, ia:ia + jb] *= 0.02
    ipiv = np.array([ia + i + int(rng.integers(0, rows - ia - i)) for i in range(jb)], np.int32)
    dA = to_dev(A)
    hlib.laswp_trsm(dA.data_ptr(), ld, ia, jb, ia, ipiv, ia + jb, n)
    got = from_dev(dA, ld, ncols)
    ref = A.copy(order="F")
    cols = slice(ia + jb, ia + jb + n)
    for i in range(jb):
        p = ipiv[i]
        ref[[ia + i, p], cols] = ref[[p, ia + i], cols]
    L = np.tril(ref[ia:ia + jb, ia:ia + jb], -1) + np.eye(jb)
    ref[ia:ia + jb, cols] = np.linalg.solve(L, ref[ia:ia + jb, cols])
    assert np.allclose(got[:, cols], ref[:, cols], rtol=0, atol=1e-12)
    # columns outside the block untouched
    assert np.array_equal(got[:, :ia + jb], A[:, :ia + jb])


def test_row_swap_matches_reference_dlaswp00N(hlib, oracle):
    """The swap half of laswp_trsm against rocHPL's own HPL_dlaswp00N, with an
    identity L11 so the TRSM leaves the rows as they are."""
    import torch

    R = oracle.ref()
    if R is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(5)
    jb, n, rows = 64, 50, 400
    ld = rows
    A = np.asfortranarray(rng.uniform(-0.5, 0.5, (ld, jb + n)))
    A[:jb, :jb] = np.eye(jb)  # L11 = I below the diagonal
    ipiv = np.array([i + int(rng.integers(0, rows - i)) for i in range(jb)], np.int32)
    dA = to_dev(A)
    hlib.laswp_trsm(dA.data_ptr(), ld, 0, jb, 0, ipiv, jb, n)
    ours = from_dev(dA, ld, jb + n)[:, jb:]
    permU = oracle.swapids(0, ipiv)
    dB = to_dev(np.asfortranarray(A[:, jb:]))
    dperm = torch.from_numpy(permU).cuda()
    assert R.ref_dlaswp00N(jb, n, dB.data_ptr(), ld, dperm.data_ptr()) == 0
    theirs = from_dev(dB, ld, n)
    assert np.array_equal(ours, theirs)
