"""The oracle pinned against the reference's own tests (CPU only).

Golden data come from blockdaglu/apps/tests/main.cpp: the 3x3 system with
duplicate entries (:85-91, :111-128), cache_matrix's all-ones solutions
(:130-168, :197-204) and the export identity (:170-195).  Tolerance: the
reference's close(), relative 1e-9 (:71-73).
"""
import numpy as np
import pytest
import scipy.linalg

import oracle

from reference_cases import GOLDEN_X, cache_matrix, close_vec, dense, export_matrix, small_matrix


def test_canonicalize_duplicates_sum_to_zero_and_drop():
    coo = small_matrix() + [(0, 0, 1.0), (0, 0, -1.0)]
    code, n, canon = oracle.canonicalize_small(coo, 3)
    assert code == 0 and n == 3
    assert canon == sorted(small_matrix())


def test_canonicalize_error_codes():
    # main.cpp:93-109
    assert oracle.canonicalize_small([(-1, 0, 1.0)])[0] == oracle.INVALID_INDEX
    assert oracle.canonicalize_small([(0, 0, float("inf"))])[0] == oracle.NON_FINITE
    assert oracle.canonicalize_small([(2, 2, 1.0)], 2)[0] == oracle.INVALID_INDEX


def test_golden_3x3_through_oracle():
    coo = small_matrix() + [(0, 0, 1.0), (0, 0, -1.0)]
    _, n, canon = oracle.canonicalize_small(coo, 3)
    rows, cols, vals = (np.array(t) for t in zip(*canon))
    ident = np.arange(n, dtype=np.int32)
    sysm = oracle.System(n, rows, cols, vals, ident, ident, np.array([0, n], np.int32))
    assert sysm.factor()
    x = sysm.solve(np.array([1.0, 2.0, 3.0]))
    assert close_vec(x, GOLDEN_X)


@pytest.mark.parametrize("changed", [1100 // 2 + 1, 1100 // 2 + 2])
def test_cache_matrix_all_ones(changed):
    n = 1100
    _, _, canon = oracle.canonicalize_small(cache_matrix(n, changed), n)
    rows, cols, vals = (np.array(t) for t in zip(*canon))
    # cache_matrix is upper triangular: identity permutations with 1x1 BTF
    # blocks are a valid block triangular form; merge as the reference does.
    ident = np.arange(n, dtype=np.int32)
    R = oracle.merge_block_boundaries(np.arange(n + 1, dtype=np.int32), n, 64)
    for scale in (1.0, 2.0):  # main.cpp:162-167 also solves the values x 2
        sysm = oracle.System(n, rows, cols, vals * scale, ident, ident, R)
        assert sysm.factor()
        b = np.zeros(n)
        np.add.at(b, rows, vals * scale)
        assert close_vec(sysm.solve(b), np.ones(n))


def test_dense_lu_pivots_match_lapack_getrf():
    # LAPACK's idamax also takes the first maximal entry, so the pivot
    # sequence of the reference micro-kernel equals getrf's.
    rng = np.random.default_rng(7)
    for m in (1, 2, 5, 17, 64, 90):
        a = rng.standard_normal((m, m))
        ok, lu, piv = oracle.dense_lu(a)
        assert ok
        lu_ref, piv_ref = scipy.linalg.lu_factor(a)
        assert np.array_equal(piv, piv_ref)
        np.testing.assert_allclose(lu, lu_ref, rtol=1e-10, atol=1e-12)


def test_dense_lu_zero_pivot_fails():
    a = np.array([[1.0, 2.0], [2.0, 4.0]])
    ok, _, _ = oracle.dense_lu(a)
    assert not ok


def test_dense_lu_tie_takes_first_row():
    a = np.array([[1.0, 0.0, 0.0], [-3.0, 1.0, 0.0], [3.0, 0.0, 1.0]])
    ok, _, piv = oracle.dense_lu(a)
    assert ok and piv[0] == 1


def test_export_identity_4x4_global_lu():
    # main.cpp:170-195 matrix: the oracle's global dense LU satisfies P*A = L*U.
    a = dense(export_matrix(), 4)
    ok, lu, piv = oracle.dense_lu(a)
    assert ok
    L = np.tril(lu, -1) + np.eye(4)
    U = np.triu(lu)
    pa = a.copy()
    for k, p in enumerate(piv):
        pa[[k, p]] = pa[[p, k]]
    assert close_vec((L @ U).ravel(), pa.ravel())
