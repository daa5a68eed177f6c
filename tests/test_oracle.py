"""CPU checks of the oracle: pinned to rocHPL's own code through the golden
fixtures (made by tests/golden/make_golden.py from the reference sources), and
its LU checked by the HPL residual at small sizes."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_jump_matches_reference_xjumpm(oracle):
    for e in json.load(open(os.path.join(GOLD, "jump_golden.json"))):
        a, c = oracle.jump(e["k"])
        assert f"{a:016x}" == e["a"] and f"{c:016x}" == e["c"], e["k"]
        assert f"{(a * 100 + c) % 2**64:016x}" == e["x_from_100"]


def test_swapids_matches_reference_pipid(oracle):
    for e in json.load(open(os.path.join(GOLD, "perm_golden.json"))):
        got = oracle.swapids(e["ia"], np.array(e["ipiv"], dtype=np.int32))
        assert got.tolist() == e["permU"]


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "lcg_golden.json")),
                    reason="LCG fixture is produced on a GPU by make_golden.py --lcg")
def test_lcg_matches_reference_kernel(oracle):
    for e in json.load(open(os.path.join(GOLD, "lcg_golden.json"))):
        m, n = e["m"], e["n"]
        if m * n > 5_000_000:
            A = oracle.matgen(m, n, e["seed"], ld=oracle.default_ld(m))
        else:
            A = oracle.matgen(m, n, e["seed"], ld=oracle.default_ld(m))
        assert f"{oracle.hash_block(A, m, n):016x}" == e["fnv1a"], (m, n)
        for i, j, hx in e["samples"]:
            assert A[i, j].hex() == hx


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "lcg_c2_golden.json")),
                    reason="made on a GPU by make_golden.py --lcg-c2")
def test_lcg_c2_blocks_match_reference_kernel(oracle):
    """The oracle's generator at N = 131072, where the state index i + j N
    passes 2^32, against the reference generator's own blocks."""
    g = json.load(open(os.path.join(GOLD, "lcg_c2_golden.json")))
    n = g["n"]
    for b in g["blocks"]:
        A = oracle.matgen_block(n, 0, b["col0"], n, b["ncols"], g["seed"])
        assert f"{oracle.hash_block(A, n, b['ncols']):016x}" == b["fnv1a"], b["name"]
        for i, j, hx in b["samples"]:
            assert A[i, j - b["col0"]].hex() == hx
            assert oracle.lcg_value(oracle.lcg_state(g["seed"], n, i, j)).hex() == hx


def test_matgen_block_is_a_block_of_matgen(oracle):
    A = oracle.matgen(300, 301, 7)
    for (i0, j0, m, n) in [(0, 0, 300, 301), (5, 9, 100, 200), (299, 300, 1, 1)]:
        assert np.array_equal(oracle.matgen_block(300, i0, j0, m, n, 7), A[i0:i0 + m, j0:j0 + n])


def test_lcg_value_range_and_state_index(oracle):
    # Entry (i, j) of an m-row matrix is state X(1 + i + j m) (P = Q = 1).
    A = oracle.matgen(37, 5, 100)
    for (i, j) in [(0, 0), (36, 0), (0, 4), (17, 3)]:
        assert A[i, j] == oracle.lcg_value(oracle.lcg_state(100, 37, i, j))
    assert np.all(A > -0.5) and np.all(A <= 0.5)


def test_ld_padding(oracle):
    from rochpl_b200.hpl import default_ld

    for n in [1, 31, 4096, 131072]:
        assert oracle.default_ld(n) == default_ld(n)
    assert default_ld(131072) == 131104 and default_ld(4096) == 4128


@pytest.mark.parametrize("n,nb,nbmin", [(1, 1, 1), (2, 1, 1), (31, 8, 4), (100, 32, 8),
                                        (257, 64, 16), (1000, 256, 32)])
def test_oracle_solve_residual(oracle, n, nb, nbmin):
    x, ipiv, info, resid = oracle.hpl_test(n, nb, nbmin, 2)
    assert info == 0
    assert resid < 16.0
    assert all(ipiv[j] >= j for j in range(n))


def test_oracle_variants_same_pivots(oracle):
    ref = None
    for pf in (0, 1, 2):
        for rf in (0, 1, 2):
            x, ipiv, info, resid = oracle.hpl_test(300, 64, 8, 2, pf, rf)
            assert resid < 16.0
            if ref is None:
                ref = (x, ipiv)
            assert np.array_equal(ipiv, ref[1])
            assert np.max(np.abs(x - ref[0])) <= 1e-10 * np.max(np.abs(ref[0]))


def test_oracle_matches_numpy_solve(oracle):
    n = 200
    A = oracle.matgen(n, n + 1, 7, ld=oracle.default_ld(n))
    M = A[:n, :n].copy()
    b = A[:n, n].copy()
    x, ipiv, info = oracle.pdgesv(A, n, 32, 8, 2)
    xr = np.linalg.solve(M, b)
    assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) < 1e-10


def test_oracle_zero_pivot_reports_info(oracle):
    n = 40
    A = oracle.matgen(n, n + 1, 100, ld=oracle.default_ld(n))
    A[:, 5] = 0.0  # column 5 identically zero
    _, _, info = oracle.pdgesv(A, n, 16, 4, 2)
    assert info == 6
