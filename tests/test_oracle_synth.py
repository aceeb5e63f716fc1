"""The oracle's input generator (oracle/synth_oracle.c) and block triangular
form (oracle/btf_oracle.c) against the engine's.  The CPU baseline and the
benchmark's reference arm build their inputs and orderings with the oracle's
code, so they load no engine library; these tests show that they see the
same systems and the same block partition.  CPU only."""
import numpy as np
import pytest
import scipy.sparse as sp

import blockdaglu as bd
import oracle


@pytest.mark.parametrize("family,config,instance,n", [
    (bd.FAMILY_BLOCK, 0, 0, 2000),
    (bd.FAMILY_BLOCK, 2, 5, 37000),
    (bd.FAMILY_CIRCUIT, 1, 3, 20000),
    (bd.FAMILY_CIRCUIT, 1, 0, 200000),
])
def test_oracle_generator_equals_engine_generator(family, config, instance, n):
    seed = bd.config_seed(config, instance)
    assert oracle.config_seed(config, instance) == seed
    a = oracle.Synth(family, seed, n, nrhs=2)
    b = bd.Synth(family, seed, n, nrhs=2)
    assert a.n == b.n and a.nnz == b.nnz
    for key in ("rows", "cols", "vals", "x_true", "b"):
        assert np.array_equal(getattr(a, key), getattr(b, key)), key
    assert np.array_equal(a.perturbed(1_000_003), b.perturbed(1_000_003))


def _csc(g):
    a = sp.csc_matrix((np.ones(g.nnz), (g.rows, g.cols)), shape=(g.n, g.n))
    a.sort_indices()
    return a


def _check_btf(rows, cols, n, nb, P, Q, R, nmatch):
    assert R[0] == 0 and R[-1] == n and len(R) == nb + 1 and np.all(np.diff(R) > 0)
    assert np.array_equal(np.sort(P), np.arange(n))
    Qu = np.where(Q < -1, -Q - 2, Q)
    assert np.array_equal(np.sort(Qu), np.arange(n))
    blk = np.repeat(np.arange(nb), np.diff(R))
    rpos, cpos = np.empty(n, np.int64), np.empty(n, np.int64)
    rpos[P] = np.arange(n)
    cpos[Qu] = np.arange(n)
    # Block upper triangular: no entry below the diagonal blocks.
    assert np.all(blk[rpos[rows]] <= blk[cpos[cols]])
    # Matched diagonal: every unflipped position holds an entry.
    diag = set(zip(rpos[rows].tolist(), cpos[cols].tolist()))
    assert sum(1 for k in range(n) if (k, k) in diag) >= nmatch
    return sorted(tuple(sorted(P[R[i]:R[i + 1]].tolist())) for i in range(nb))


@pytest.mark.parametrize("family,config,instance,n", [
    (bd.FAMILY_BLOCK, 0, 0, 2000),
    (bd.FAMILY_CIRCUIT, 1, 3, 20000),
    (bd.FAMILY_CIRCUIT, 1, 0, 200000),
])
def test_oracle_btf_partition_equals_engine(family, config, instance, n):
    g = oracle.Synth(family, bd.config_seed(config, instance), n)
    a = _csc(g)
    nb, P, Q, R, nm = oracle.btf_order(n, a.indptr, a.indices)
    nb2, P2, Q2, R2, nm2 = bd.btf_order(n, a.indptr, a.indices)
    assert nm == nm2 == n and nb == nb2
    # Any maximum matching gives the same blocks as sets of rows.
    assert _check_btf(g.rows, g.cols, n, nb, P, Q, R, nm) == _check_btf(g.rows, g.cols, n, nb2, P2, Q2, R2, nm2)
    # The strongly connected components of the matched graph (scipy).
    qu = np.where(Q < -1, -Q - 2, Q)
    cpos = np.empty(n, np.int64)
    cpos[qu] = np.arange(n)
    rpos = np.empty(n, np.int64)
    rpos[P] = np.arange(n)
    gph = sp.csr_matrix((np.ones(g.nnz), (rpos[g.rows], cpos[g.cols])), shape=(n, n))
    ncomp, _ = sp.csgraph.connected_components(gph, directed=True, connection="strong")
    assert ncomp == nb


def test_oracle_btf_structurally_singular():
    # Columns 1 and 2 share one row: the maximum matching has size n - 1.
    rows = np.array([0, 0, 1, 2, 3, 3], np.int32)
    cols = np.array([0, 3, 1, 1, 2, 3], np.int32)
    n = 4
    a = sp.csc_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    a.sort_indices()
    nb, P, Q, R, nm = oracle.btf_order(n, a.indptr, a.indices)
    nb2, _, Q2, _, nm2 = bd.btf_order(n, a.indptr, a.indices)
    assert nm == nm2 == 3
    assert np.sum(Q < -1) == np.sum(Q2 < -1) == 1
    _check_btf(rows, cols, n, nb, P, Q, R, 0)
