"""Host integer analysis (CPU only): canonicalisation, BTF, merge, UBTF split
and block DAG, checked against the oracle and against scipy's strong
components.  Integer results must be identical."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

import blockdaglu as bd
import oracle

from reference_cases import cache_matrix, small_matrix


def analysed(rows, cols, vals, n=-1, mode=None, monkeypatch=None):
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix((rows, cols, vals), n)
    ok = s.analyze()
    return s, ok


def synth(family, seed, n, param=0):
    return bd.Synth(family, seed, n, param)


@pytest.fixture(autouse=True)
def _block_mode(monkeypatch):
    monkeypatch.delenv("BLOCKDAGLU_MODE", raising=False)
    monkeypatch.delenv("USERALGO_MODE", raising=False)


def test_error_codes_match_reference():
    # apps/tests/main.cpp:93-109: storage-only set_matrix, errors at analyze.
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix([(-1, 0, 1.0)])
    assert not s.analyze() and s.last_error() == bd.SolverError.InvalidIndex
    assert s.set_matrix([(0, 0, float("inf"))])
    assert not s.analyze() and s.last_error() == bd.SolverError.NonFiniteValue
    assert s.set_matrix([(2, 2, 1.0)], 2)
    assert not s.analyze() and s.last_error() == bd.SolverError.InvalidIndex
    assert s.last_error_message() == "matrix entry lies outside the declared dimension"


def test_stage_order_enforced():
    s = bd.Solver()
    assert not s.analyze() and s.last_error() == bd.SolverError.NotPrepared
    assert not s.factor() and s.last_error() == bd.SolverError.NotPrepared
    b = np.ones(3)
    assert not s.solve_in_place(b) and s.last_error() == bd.SolverError.NotPrepared


def test_canonical_pattern_matches_oracle():
    coo = small_matrix() + [(0, 0, 1.0), (0, 0, -1.0), (2, 0, 0.0), (1, 2, 0.5)]
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix(coo, 3) and s.analyze()
    r, c = s.canonical_pattern()
    _, n, canon = oracle.canonicalize_small(coo, 3)
    assert n == 3 and list(zip(r.tolist(), c.tolist())) == [(a, b) for a, b, _ in canon]


def _btf_checks(rows, cols, n):
    a = sp.csc_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    nb, P, Q, R, nmatch = bd.btf_order(n, a.indptr, a.indices)
    assert nmatch == n
    assert sorted(P.tolist()) == list(range(n)) and sorted(Q.tolist()) == list(range(n))
    B = a.tocsr()[P][:, Q].tocoo()
    block_of = np.repeat(np.arange(nb), np.diff(R))
    # Upper block triangular and zero-free diagonal.
    assert np.all(block_of[B.col] >= block_of[B.row])
    assert np.all(B.tocsr().diagonal() != 0)
    # The blocks are exactly the strongly connected components.
    ncomp, labels = connected_components(B.tocsr(), directed=True, connection="strong")
    assert ncomp == nb
    for b in range(nb):
        assert len(set(labels[R[b]:R[b + 1]].tolist())) == 1
    return nb, P, Q, R


@pytest.mark.parametrize("seed", [bd.config_seed(0), bd.config_seed(0, 1)])
def test_btf_block_family(seed):
    g = synth(bd.FAMILY_BLOCK, seed, 2000, 40)
    nb, _, _, R = _btf_checks(g.rows, g.cols, g.n)
    # The generator's 40 irreducible blocks are recovered.
    assert nb == 40
    assert sorted(np.diff(R).tolist()) == sorted(g.block_sizes.tolist())


def test_btf_circuit_family_small():
    g = synth(bd.FAMILY_CIRCUIT, bd.config_seed(1, 7), 20000)
    nb, _, _, R = _btf_checks(g.rows, g.cols, g.n)
    assert sorted(np.diff(R).tolist()) == sorted(g.block_sizes.tolist())


def test_btf_structurally_singular_flags_unmatched():
    # Column 1 is empty: maximum matching has size 2 and Q carries a flip.
    n = 3
    rows = np.array([0, 1, 2, 2], np.int32)
    cols = np.array([0, 0, 2, 0], np.int32)
    a = sp.csc_matrix((np.ones(4), (rows, cols)), shape=(n, n))
    nb, P, Q, R, nmatch = bd.btf_order(n, a.indptr, a.indices)
    assert nmatch == 2
    assert np.any(Q < -1)


def test_merge_matches_oracle_random():
    rng = np.random.default_rng(3)
    for trial in range(200):
        sizes = rng.choice([1, 1, 1, 2, 5, 17, 31, 32, 33, 40, 64, 65, 100], size=rng.integers(1, 60))
        R = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
        n = int(R[-1])
        for mm in (1, 8, 32, 64, 100):
            assert np.array_equal(bd.merge_block_boundaries(R, n, mm), oracle.merge_block_boundaries(R, n, mm))


@pytest.mark.parametrize("family,seed,n", [
    (bd.FAMILY_BLOCK, bd.config_seed(0), 2000),
    (bd.FAMILY_CIRCUIT, bd.config_seed(1, 3), 20000),
])
def test_split_and_levels_match_oracle(family, seed, n):
    g = synth(family, seed, n)
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze(), s.last_error_message()
    d = s.decomposition()
    sysm = oracle.System(g.n, g.rows, g.cols, g.vals, d["P"], d["Q"], d["R"])
    optr, ocol, oval = sysm.offdiag()
    assert np.array_equal(d["off_ptr"], optr)
    assert np.array_equal(d["off_col"], ocol)
    assert np.array_equal(g.vals[d["off_src"]], oval)
    lev, mx = sysm.levels()
    assert np.array_equal(d["level"], lev)
    assert s.stats()["max_level"] == mx
    # Merged boundaries are the reference's merge of the raw BTF blocks.
    a = sp.csc_matrix((np.ones(g.nnz), (g.rows, g.cols)), shape=(g.n, g.n))
    _, _, _, Rraw, _ = bd.btf_order(g.n, a.indptr, a.indices)
    assert np.array_equal(d["R"], oracle.merge_block_boundaries(Rraw, g.n, 64))


def test_cache_matrix_decomposition():
    n = 1100
    coo = cache_matrix(n, n // 2 + 1)
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix(coo, n) and s.analyze()
    st = s.stats()
    assert st["nblocks_raw"] == n  # upper triangular: every row its own SCC
    assert st["nblocks"] == (n + 63) // 64


def test_merge_env_knob(monkeypatch):
    monkeypatch.setenv("BLOCKDAGLU_BLOCK_MERGE", "0")
    n = 1100
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix(cache_matrix(n, n // 2 + 1), n) and s.analyze()
    assert s.stats()["nblocks"] == n
