"""GPU parity: the engine through the C ABI against the reference's own test
cases and the oracle.

Tolerances: solutions within the reference's close() (relative 1e-9,
apps/tests/main.cpp:71-73); the normwise residual
|Ax-b|_inf / (|A|_inf |x|_inf + |b|_inf) <= 1e-12; dense-block factors and
pivots of the reference micro-kernel path bit-identical (==).
"""
import threading

import numpy as np
import pytest

import blockdaglu as bd
import oracle

from reference_cases import (GOLDEN_X, cache_matrix, close_vec, dense, export_matrix, multiply,
                             small_matrix)

pytestmark = pytest.mark.gpu

RESID_TOL = 1e-12


@pytest.fixture(autouse=True)
def _env(monkeypatch, cuda_device):
    for k in ("BLOCKDAGLU_MODE", "USERALGO_MODE", "BLOCKDAGLU_REFINE_ITERS", "USERALGO_REFINE_ITERS"):
        monkeypatch.delenv(k, raising=False)


def solve_known_ones(coo, n):
    """main.cpp:145-154."""
    rhs = multiply(coo, n, np.ones(n))
    s = bd.Solver()
    assert s.set_matrix(coo, n)
    assert s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    assert s.solve_in_place(rhs), s.last_error_message()
    assert close_vec(rhs, np.ones(n))
    return s


def test_invalid_inputs():
    # main.cpp:93-109
    s = bd.Solver()
    assert s.set_matrix([(-1, 0, 1.0)])
    assert not s.analyze() and s.last_error() == bd.SolverError.InvalidIndex
    s = bd.Solver()
    assert s.set_matrix([(0, 0, float("inf"))])
    assert not s.analyze() and s.last_error() == bd.SolverError.NonFiniteValue
    s = bd.Solver()
    assert s.set_matrix([(2, 2, 1.0)], 2)
    assert not s.analyze() and s.last_error() == bd.SolverError.InvalidIndex


@pytest.mark.parametrize("mode", ["klu", "block"])
def test_solve_and_duplicates(monkeypatch, mode):
    # main.cpp:111-128 (run by the reference in KLU mode; both routes here).
    monkeypatch.setenv("BLOCKDAGLU_MODE", mode)
    s = bd.Solver()
    coo = small_matrix() + [(0, 0, 1.0), (0, 0, -1.0)]
    rhs = np.array([1.0, 2.0, 3.0])
    assert s.set_matrix(coo, 3)
    assert s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    assert s.solve_in_place(rhs), s.last_error_message()
    assert close_vec(rhs, GOLDEN_X)
    assert s.selected_mode() == ("KLU" if mode == "klu" else "BLOCK")
    bad = np.array([1.0, 2.0])
    assert not s.solve_in_place(bad)
    assert s.last_error() == bd.SolverError.InvalidRightHandSide


def test_cache_isolation(monkeypatch):
    # main.cpp:156-168
    monkeypatch.setenv("BLOCKDAGLU_MODE", "block")
    monkeypatch.setenv("BLOCKDAGLU_CACHE", "1")
    n = 1100
    solve_known_ones(cache_matrix(n, n // 2 + 1), n)
    solve_known_ones(cache_matrix(n, n // 2 + 2), n)
    original = cache_matrix(n, n // 2 + 1)
    scaled = [(r, c, 2.0 * v) for r, c, v in original]
    solve_known_ones(original, n)
    solve_known_ones(scaled, n)


def test_compatibility_export(monkeypatch):
    # main.cpp:170-195
    monkeypatch.setenv("BLOCKDAGLU_MODE", "block")
    s = bd.Solver()
    assert s.set_matrix(export_matrix(), 4)
    assert s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    rearranged = s.get_rearranged_matrix()
    L = s.getL()
    U = s.getU()
    assert rearranged and L and U
    assert close_vec(dense(rearranged, 4).ravel(), (dense(L, 4) @ dense(U, 4)).ravel())
    # P and Q are the permutations of the identity rearranged = P A Q.
    P = dense(s.getP(), 4)
    Q = dense(s.getQ(), 4)
    assert close_vec((P @ dense(export_matrix(), 4) @ Q).ravel(), dense(rearranged, 4).ravel())


def test_concurrent_solvers(monkeypatch):
    # main.cpp:197-204
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    errors = []

    def worker():
        try:
            solve_known_ones(cache_matrix(256, 129), 256)
        except AssertionError as e:  # pragma: no cover - reported below
            errors.append(e)

    ts = [threading.Thread(target=worker) for _ in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors


def _engine_and_oracle(g):
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n)
    assert s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    d = s.decomposition()
    ref = oracle.System(g.n, g.rows, g.cols, g.vals, d["P"], d["Q"], d["R"])
    assert ref.factor()
    return s, d, ref


def _inf_resid(g, vals, x, b):
    return oracle.metrics(g.rows, g.cols, vals, x, b, n=g.n)[0]


@pytest.mark.parametrize("instance", [0, 1, 2])
def test_block_family_matches_oracle(instance):
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, instance), 2000, 40)
    s, d, ref = _engine_and_oracle(g)
    # Factors of every merged block equal the reference micro-kernel's, bit for bit.
    for b in range(len(d["R"]) - 1):
        lu, piv = s.block_lu(b)
        lu_ref, piv_ref = ref.block_lu(b)
        assert np.array_equal(piv, piv_ref), b
        assert np.array_equal(lu, lu_ref), b
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x)
    x_ref = ref.solve(g.b[:, 0])
    assert close_vec(x, x_ref)
    assert _inf_resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL
    assert s.stats()["residual_inf"] <= RESID_TOL


def test_value_only_refactor_matches_fresh_factor():
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 5), 2000, 40)
    s, d, _ = _engine_and_oracle(g)
    for k in range(3):
        v = g.perturbed(1000 + k)
        assert s.refactor_values(v), s.last_error_message()
        ref = oracle.System(g.n, g.rows, g.cols, v, d["P"], d["Q"], d["R"])
        assert ref.factor()
        b = multiply(list(zip(g.rows, g.cols, v)), g.n, g.x_true[:, 0])
        x = b.copy()
        assert s.solve_in_place(x)
        assert close_vec(x, ref.solve(b))
        for blk in (0, len(d["R"]) // 2, len(d["R"]) - 2):
            assert np.array_equal(s.block_lu(blk)[0], ref.block_lu(blk)[0])


def test_multi_rhs_columns_equal_single_solves():
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(2, 0), 3000, 60, nrhs=8)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor()
    X = np.asfortranarray(g.b.copy())
    assert s.solve_in_place(X), s.last_error_message()
    for k in range(8):
        x = np.ascontiguousarray(g.b[:, k])
        assert s.solve_in_place(x)
        assert close_vec(X[:, k], x, 1e-12)
        assert close_vec(X[:, k], g.x_true[:, k], 1e-8)


def test_global_route_large_dense_unit(monkeypatch):
    # MODE=klu: one 2000x2000 unit through the blocked multi-CTA LU.
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0), 2000, 40)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    assert s.stats()["max_unit"] == 2000
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x)
    assert _inf_resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL
    assert close_vec(x, g.x_true[:, 0], 1e-8)


def test_refinement_option_keeps_solution():
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 9), 2000, 40)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor()
    assert s.set_option("refine_iters", 2)
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x)
    assert s.stats()["refine_iters"] == 2
    assert _inf_resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL


def test_singular_block_reports_factorization_failed():
    # Two identical rows inside one irreducible block.
    coo = [(0, 0, 1.0), (0, 1, 2.0), (1, 0, 1.0), (1, 1, 2.0), (2, 2, 3.0), (0, 2, 1.0)]
    s = bd.Solver()
    assert s.set_matrix(coo, 3) and s.analyze()
    assert not s.factor()
    assert s.last_error() == bd.SolverError.FactorizationFailed


def test_circuit_full_size_residual():
    # The 200k-row circuit configuration at full size: size-independent
    # properties (normwise residual, agreement with x_true to the conditioning).
    g = bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(1), 200000)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert _inf_resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL
    st = s.stats()
    assert st["residual_inf"] <= RESID_TOL
    assert st["max_unit"] == int(g.block_sizes.max())
    # Value-only refactor + solve stays on the same bound.
    v = g.perturbed(77)
    assert s.refactor_values(v)
    b = multiply(list(zip(g.rows, g.cols, v)), g.n, g.x_true[:, 0])
    x = b.copy()
    assert s.solve_in_place(x)
    assert _inf_resid(g, v, x, b) <= RESID_TOL


def test_circuit_small_matches_oracle():
    g = bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(1, 3), 20000)
    s, d, ref = _engine_and_oracle(g)
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x)
    assert close_vec(x, ref.solve(g.b[:, 0]))
    R = d["R"]
    for b in range(len(R) - 1):
        if R[b + 1] - R[b] <= 64:
            lu, piv = s.block_lu(b)
            lu_ref, piv_ref = ref.block_lu(b)
            assert np.array_equal(piv, piv_ref) and np.array_equal(lu, lu_ref), b


def test_global_route_tall_unit_fallback_panel(monkeypatch):
    # MODE=klu on 7000 rows: one unit taller than a thread-block cluster holds,
    # factored by the single-CTA global-memory panel and solved tile by tile.
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 11), 7000, 140)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    assert s.stats()["max_unit"] == 7000
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x)
    assert _inf_resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL


def test_refactor_reusing_pivot_order_matches_pivoting_refactor(monkeypatch):
    # MODE=klu: one 2000-row block factored across CTAs.  A value-only refactor
    # keeps the block's pivot order (klu_refactor semantics); the result must
    # agree with a refactor that pivots again.
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 21), 2000, 40)
    s1, s2 = bd.Solver(), bd.Solver()
    for s, piv in ((s1, 0), (s2, 1)):
        assert s.set_option("refactor_pivoting", piv)
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    for k in range(3):
        v = g.perturbed(300 + k)
        b = multiply(list(zip(g.rows, g.cols, v)), g.n, g.x_true[:, 0])
        xs = []
        for s in (s1, s2):
            assert s.refactor_values(v), s.last_error_message()
            x = b.copy()
            assert s.solve_in_place(x), s.last_error_message()
            assert _inf_resid(g, v, x, b) <= RESID_TOL
            xs.append(x)
        assert close_vec(xs[0], xs[1], 1e-8)


def test_refactor_reused_zero_pivot_falls_back_to_pivoting(monkeypatch):
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 22), 400, 1)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    first_row = s.getP()[0][1]      # original row chosen as the first pivot
    v = g.vals.copy()
    hit = np.nonzero((g.rows == first_row) & (g.cols == 0))[0]
    assert len(hit) == 1
    v[hit[0]] = 0.0                 # the reused first pivot is now exactly zero
    assert s.refactor_values(v), s.last_error_message()
    assert s.getP()[0][1] != first_row
    b = multiply(list(zip(g.rows, g.cols, v)), g.n, g.x_true[:, 0])
    x = b.copy()
    assert s.solve_in_place(x)
    assert _inf_resid(g, v, x, b) <= RESID_TOL
