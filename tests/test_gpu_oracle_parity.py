"""GPU parity against the oracle for the paths the reference micro-kernel
tests do not reach: large units (the blocked LU above the shared-memory
limit), the global route, value-only refactors that reuse the pivot order,
the mixed-precision route, batches of systems; and the bounded waits between
tiles, made to run out on purpose.

The oracle (oracle/bdlu_oracle.c, the reference's dense micro-kernel and
reverse block solve) factors every block unblocked with partial pivoting;
the engine's large units use a blocked right-looking LU with the same pivot
rule (first strict maximum), so pivots agree and the factors agree to
rounding.  Tolerances: solutions within the reference's close() (relative
1e-9, apps/tests/main.cpp:71-73) on these well-conditioned families; large
factors within 1e-11 of the largest entry; residual
|Ax-b|_inf / (|A|_inf |x|_inf + |b|_inf) <= 1e-12.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import blockdaglu as bd
import oracle

from reference_cases import close_vec

pytestmark = pytest.mark.gpu

RESID_TOL = 1e-12


@pytest.fixture(autouse=True)
def _env(monkeypatch, cuda_device):
    for k in ("BLOCKDAGLU_MODE", "USERALGO_MODE", "BLOCKDAGLU_REFINE_ITERS", "USERALGO_REFINE_ITERS"):
        monkeypatch.delenv(k, raising=False)


def _rhs(g, vals, x):
    b = np.zeros(g.n)
    np.add.at(b, g.rows, vals * x[g.cols])
    return b


def _resid(g, vals, x, b):
    r = b.copy()
    np.subtract.at(r, g.rows, vals * x[g.cols])
    arow = np.zeros(g.n)
    np.add.at(arow, g.rows, np.abs(vals))
    return np.max(np.abs(r)) / (arow.max() * np.max(np.abs(x)) + np.max(np.abs(b)))


def _oracle_own_ordering(g, vals):
    """The oracle's system under its own BTF (btf_oracle.c) and merge: shares
    nothing with the engine's analysis."""
    a = sp.csc_matrix((np.ones(g.nnz), (g.rows, g.cols)), shape=(g.n, g.n))
    a.sort_indices()
    _, P, Q, R, _ = oracle.btf_order(g.n, a.indptr, a.indices)
    Q = np.where(Q < -1, -Q - 2, Q)
    sysm = oracle.System(g.n, g.rows, g.cols, vals, P, Q, oracle.merge_block_boundaries(R, g.n))
    assert sysm.factor()
    return sysm


def _large_system():
    # 3,000 rows in 6 irreducible blocks of 274-741 rows: every block is a
    # large unit (above the 169-row shared-memory limit).
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 31), 3000, 6)
    assert g.block_sizes.min() > 169
    return g


def test_large_units_match_oracle_factors_and_solution():
    g = _large_system()
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    assert s.stats()["max_unit"] > 169
    d = s.decomposition()
    ref = oracle.System(g.n, g.rows, g.cols, g.vals, d["P"], d["Q"], d["R"])
    assert ref.factor()
    R = d["R"]
    for b in range(len(R) - 1):
        lu, piv = s.block_lu(b)
        lu_ref, piv_ref = ref.block_lu(b)
        assert np.array_equal(piv, piv_ref), b
        scale = np.max(np.abs(lu_ref))
        assert np.max(np.abs(lu - lu_ref)) <= 1e-11 * scale, b
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert close_vec(x, ref.solve(g.b[:, 0]))
    assert close_vec(x, _oracle_own_ordering(g, g.vals).solve(g.b[:, 0]))
    assert _resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL


def test_value_refactor_reusing_pivots_matches_oracle():
    # The engine keeps the large units' pivot order (klu_refactor semantics);
    # the oracle pivots anew on the perturbed values.
    g = _large_system()
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    for k in range(2):
        v = g.perturbed(410 + k)
        b = _rhs(g, v, g.x_true[:, 0])
        assert s.refactor_values(v), s.last_error_message()
        x = b.copy()
        assert s.solve_in_place(x), s.last_error_message()
        assert close_vec(x, _oracle_own_ordering(g, v).solve(b))
        assert _resid(g, v, x, b) <= RESID_TOL


def test_global_route_matches_oracle(monkeypatch):
    # MODE=klu: the whole matrix is one 1,500-row unit (no BTF).
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 32), 1500, 30)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    assert s.stats()["max_unit"] == 1500
    d = s.decomposition()
    ref = oracle.System(g.n, g.rows, g.cols, g.vals, d["P"], d["Q"], d["R"])
    assert ref.factor()
    lu, piv = s.block_lu(0)
    lu_ref, piv_ref = ref.block_lu(0)
    assert np.array_equal(piv, piv_ref)
    assert np.max(np.abs(lu - lu_ref)) <= 1e-11 * np.max(np.abs(lu_ref))
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert close_vec(x, ref.solve(g.b[:, 0]))


def test_mixed_route_matches_oracle():
    # Tensor-core trailing updates + FP64 refinement: the refined solution
    # must agree with the oracle's FP64 solution.
    g = _large_system()
    rng = np.random.default_rng(5)
    B = np.asfortranarray(rng.uniform(-1.0, 1.0, (g.n, 4)))
    s = bd.Solver()
    assert s.set_option("precision", 1)
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    X = B.copy(order="F")
    assert s.solve_in_place(X), s.last_error_message()
    assert s.stats()["residual_inf"] <= RESID_TOL
    ref = _oracle_own_ordering(g, g.vals)
    # Refinement stops at the residual bound (1e-12), so the forward error is
    # up to cond(A) * 1e-12 (the units here have condition numbers up to about
    # 1e5), not the FP64 route's rounding level: relative 1e-6.
    for j in range(B.shape[1]):
        assert close_vec(X[:, j], ref.solve(np.ascontiguousarray(B[:, j])), 1e-6), j


def test_batch_systems_match_oracle():
    sizes = [1200, 2600, 4100, 1800]
    systems = [bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(2, 40 + i), n) for i, n in enumerate(sizes)]
    systems.append(bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(2, 45), 2000, 8))  # large units in a batch
    nrhs = 3
    batch = bd.Batch()
    for k, g in enumerate(systems):
        assert batch.add((g.rows, g.cols, g.vals), g.n) == k
    assert batch.analyze() and batch.factor(), batch.last_error_message()
    rng = np.random.default_rng(9)
    B = np.asfortranarray(rng.uniform(-1.0, 1.0, (batch.rows(), nrhs)))
    X = B.copy(order="F")
    assert batch.solve_in_place(X), batch.last_error_message()
    for k, g in enumerate(systems):
        off = batch.row_offset(k)
        ref = _oracle_own_ordering(g, g.vals)
        for j in range(nrhs):
            xr = ref.solve(np.ascontiguousarray(B[off:off + g.n, j]))
            assert close_vec(X[off:off + g.n, j], xr), (k, j)


def test_solve_waits_run_out_and_report_an_error(monkeypatch):
    # One 3,000-row unit is swept in 47 tiles, each waiting for the ready
    # flags of the tiles before it.  With one poll per wait the waits run out:
    # the solve reports an error status and the context stays usable.
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 33), 3000, 60)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    failed = False
    for _ in range(5):
        assert s.set_option("wait_limit", 1)
        x = g.b[:, 0].copy()
        if not s.solve_in_place(x):
            assert s.last_error() == bd.SolverError.SolveFailed
            assert "bounded wait" in s.last_error_message()
            failed = True
            break
    assert failed
    assert s.set_option("wait_limit", 0)
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert _resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL


def test_tile_graph_refactor_wait_runs_out_and_falls_back(monkeypatch):
    # The tile task graph refactor (refactor_schedule 1) with one poll per
    # wait: a wait runs out, the refactor reports it and is redone with
    # pivoting; the solution still meets the bound.
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 34), 3000, 60)
    s = bd.Solver()
    assert s.set_option("refactor_schedule", 1)
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    v = g.perturbed(501)
    b = _rhs(g, v, g.x_true[:, 0])
    assert s.set_option("wait_limit", 1)
    assert s.refactor_values(v), s.last_error_message()
    assert s.set_option("wait_limit", 0)
    x = b.copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert _resid(g, v, x, b) <= RESID_TOL
