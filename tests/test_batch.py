"""Batches of independent systems (bdlu_batch_*): the stand-in for the
reference's one-Solver-per-system loop (apps/benchmark/main.cpp:271-297).

Each system keeps its own semantics (validation errors name the system,
canonicalisation, block route), and its solution in the batch must match the
same system solved alone by a Solver: relative residual <= 1e-12 per system
and per right-hand side, and agreement with the single-system solution to the
reference tests' tolerance (1e-9, apps/tests/main.cpp:71-73).
"""
import numpy as np
import pytest

import blockdaglu as bd


def _systems(count, nmin, nmax, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        out.append(bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(2, i), n))
    return out


def _relres(g, vals, x, b):
    r = b.copy()
    np.subtract.at(r, g.rows, vals * x[g.cols])
    arow = np.zeros(g.n)
    np.add.at(arow, g.rows, np.abs(vals))
    return np.max(np.abs(r)) / (arow.max() * np.max(np.abs(x)) + np.max(np.abs(b)))


def test_batch_rejects_bad_systems():
    b = bd.Batch()
    assert b.add(([0], [0], [1.0]), 0) == -1
    assert b.last_error() == bd.SolverError.InvalidDimension
    assert b.add(([0, 1], [0, 1], [1.0, 2.0]), 2) == 0
    assert b.add(([0, 5], [0, 1], [1.0, 2.0]), 2) == 1       # row 5 outside n = 2
    assert not b.analyze()
    assert b.last_error() == bd.SolverError.InvalidIndex
    assert "system 1" in b.last_error_message()
    c = bd.Batch()
    assert not c.analyze() and c.last_error() == bd.SolverError.NotPrepared
    assert not c.factor() and c.last_error() == bd.SolverError.NotPrepared
    d = bd.Batch()
    assert d.add(([0], [0], [float("nan")]), 1) == 0
    assert not d.analyze() and d.last_error() == bd.SolverError.NonFiniteValue


@pytest.mark.gpu
def test_batch_matches_single_solvers(cuda_device):
    systems = _systems(8, 1000, 6000, 7)
    nrhs = 8
    rng = np.random.default_rng(11)
    batch = bd.Batch()
    for k, g in enumerate(systems):
        assert batch.add((g.rows, g.cols, g.vals), g.n) == k
    assert batch.analyze(), batch.last_error_message()
    assert batch.factor(), batch.last_error_message()
    N = batch.rows()
    assert N == sum(g.n for g in systems)
    B = np.asfortranarray(rng.uniform(-1.0, 1.0, (N, nrhs)))
    X = B.copy(order="F")
    assert batch.solve_in_place(X), batch.last_error_message()
    for k, g in enumerate(systems):
        o = batch.row_offset(k)
        assert o == sum(s.n for s in systems[:k])
        s = bd.Solver()
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
        Xs = np.asfortranarray(B[o:o + g.n].copy())
        assert s.solve_in_place(Xs), s.last_error_message()
        for j in range(nrhs):
            x = X[o:o + g.n, j]
            assert _relres(g, g.vals, x, B[o:o + g.n, j]) <= 1e-12, (k, j)
            assert np.allclose(x, Xs[:, j], rtol=1e-9, atol=1e-9), (k, j)


@pytest.mark.gpu
def test_batch_value_refactor(cuda_device):
    systems = _systems(6, 1000, 4000, 8)
    batch = bd.Batch()
    for g in systems:
        batch.add((g.rows, g.cols, g.vals), g.n)
    assert batch.analyze() and batch.factor(), batch.last_error_message()
    for it in range(2):
        vals = [g.perturbed(100 + it) for g in systems]
        for k, g in enumerate(systems):
            assert batch.nnz_offset(k + 1) - batch.nnz_offset(k) == g.nnz
        assert batch.refactor_values(np.concatenate(vals)), batch.last_error_message()
        B = np.concatenate([g.b[:, 0] for g in systems])
        X = B.copy()
        assert batch.solve_in_place(X), batch.last_error_message()
        for k, g in enumerate(systems):
            o = batch.row_offset(k)
            assert _relres(g, vals[k], X[o:o + g.n], B[o:o + g.n]) <= 1e-12, (it, k)
    assert not batch.refactor_values(np.ones(3))
    assert batch.last_error() == bd.SolverError.InvalidIndex


@pytest.mark.gpu
def test_batch_wrong_rhs_rows(cuda_device):
    systems = _systems(2, 1000, 1500, 9)
    batch = bd.Batch()
    for g in systems:
        batch.add((g.rows, g.cols, g.vals), g.n)
    assert batch.analyze() and batch.factor()
    bad = np.ones(batch.rows() - 1)
    assert not batch.solve_in_place(bad)
    assert batch.last_error() == bd.SolverError.InvalidRightHandSide
