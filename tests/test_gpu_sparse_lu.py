"""Sparse-LU route (option "sparse_lu", the reference's USERALGO_SPARSE_LU_KERNEL
=gp route, gp_lu.cpp:84-306 with the gate of ubtf_block_solver.cpp:197-235)
against the oracle (or_factor_gp, itself bit-identical to the reference's own
gp_lu.cpp, tests/test_gp_oracle.py), on the engine's own ordering.

CPU: the host symbolic analysis against a dense boolean elimination
(tests/cpp/gp_symbolic_test.cpp) and the plan's routing of sparse units
(tests/cpp/gp_plan_test.cpp).
GPU: the same blocks take the sparse route; accepted sparse factors are
bit-identical (==) to the oracle's, rejected blocks are factored dense
(bit-identical up to 169 rows, pivots equal and within 1e-11 above); the
solution is within 1e-9 of the oracle's and the residual within 1e-12, also
after value-only refactors, after a refactor whose values make a block fail
the test (also through the refactor + solve call that queues the refactor
with no status wait), and with 8 right-hand sides; the export identity holds; the fill
limit of option 2 selects the blocks it names; the kernels' bounded waits
run out under a one-poll limit and the handle recovers."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import blockdaglu as bd
import oracle
from conftest import ROOT
from gp_cases import no_pivot_fill, sparse_block_system

SIZES = [70, 30, 90, 120, 20, 100, 66, 200, 300, 500]
X_TOL = 1e-9
RESID_TOL = 1e-12
LARGE_TOL = 1e-11
SPARSE = 3  # bdlu_get_unit_routes route of a sparse unit


def run_cpp_check(tmp_path, name):
    lib = os.path.join(ROOT, "block-daglu_b200", "lib")
    exe = str(tmp_path / name)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "block-daglu_b200", "csrc"), "-I/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L" + lib, "-lbdlu", "-Wl,-rpath," + lib, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip().splitlines()[-1] == "ok", r.stdout + r.stderr


def test_symbolic_matches_dense_elimination(tmp_path):
    """gp_symbolic against a dense boolean elimination, the kernels' index
    arithmetic emulated with bounds checks, and the environment knobs."""
    run_cpp_check(tmp_path, "gp_symbolic_test")


def test_plan_routes_sparse_units(tmp_path):
    """build_plan with the route on: sparse units leave the dense tables and
    arena, appear once per level, and map back to the canonical entries; the
    fill limit, earlier rejections and an unsupported setting keep units
    dense."""
    run_cpp_check(tmp_path, "gp_plan_test")


def engine(n, r, c, v, mode=1, fill_max=None):
    s = bd.Solver()
    s.set_option("sparse_lu", mode)
    if fill_max is not None:
        s.set_option("sparse_fill_max", fill_max)
    assert s.set_matrix((r, c, v), n), s.last_error_message()
    assert s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    return s


def route_of_blocks(s):
    """Per merged block b: (route, reason) of the unit starting at R[b], or
    None when the block is not one unit."""
    R = s.decomposition()["R"]
    start, route, reason = s.unit_routes()
    at = {int(a): (int(b), int(c)) for a, b, c in zip(start, route, reason)}
    return [at.get(int(R[b])) if R[b + 1] - R[b] > 1 else None for b in range(len(R) - 1)]


def check_against_oracle(s, n, r, c, v, check_sparse_only=False):
    d = s.decomposition()
    R = d["R"]
    o = oracle.System(n, r, c, v, d["P"], d["Q"], R)
    ok, reason = o.factor_gp()
    assert ok
    routes = route_of_blocks(s)
    counts = {"sparse": 0, "rejected": 0}
    for b in range(len(R) - 1):
        m = int(R[b + 1] - R[b])
        lu, piv = s.block_lu(b)
        lu_o, piv_o = o.block_lu(b)
        if routes[b] is not None and routes[b][0] == SPARSE:
            assert reason[b] == 0, (b, m, reason[b])
            assert np.array_equal(piv, np.arange(m))
            assert np.array_equal(lu, lu_o), (b, m, np.abs(lu - lu_o).max())
            counts["sparse"] += 1
            continue
        if check_sparse_only:
            continue
        if reason[b] > 0:
            assert routes[b][1] in (1, 2, 3, 4), (b, routes[b])
            counts["rejected"] += 1
        if m <= 169:
            assert np.array_equal(piv, piv_o) and np.array_equal(lu, lu_o), b
        else:
            assert np.array_equal(piv, piv_o), b
            assert np.abs(lu - lu_o).max() <= LARGE_TOL * max(1.0, np.abs(lu_o).max()), b
    return o, counts


def check_solution(s, o, n, r, c, v, nrhs=1, seed=9):
    B = np.asfortranarray(np.random.default_rng(seed).uniform(-1, 1, (n, nrhs)))
    X = B.copy(order="F")
    assert s.solve_in_place(X if nrhs > 1 else X[:, 0]), s.last_error_message()
    for k in range(nrhs):
        x_o = o.solve(B[:, k])
        assert np.max(np.abs(X[:, k] - x_o) / np.maximum(1.0, np.abs(x_o))) <= X_TOL
        assert oracle.metrics(r, c, v, X[:, k], B[:, k])[0] <= RESID_TOL


@pytest.mark.gpu
def test_sparse_route_matches_oracle():
    n, r, c, v = sparse_block_system(0, SIZES, 0.5)
    s = engine(n, r, c, v)
    o, counts = check_against_oracle(s, n, r, c, v)
    assert counts["sparse"] >= 4 and counts["rejected"] >= 1, counts
    check_solution(s, o, n, r, c, v)


@pytest.mark.gpu
def test_sparse_route_refactors_match_oracle():
    n, r, c, v = sparse_block_system(1, SIZES, 1.0)
    s = engine(n, r, c, v)
    rng = np.random.default_rng(3)
    for step in range(3):
        v2 = v * (1.0 + rng.uniform(-0.05, 0.05, len(v)))
        assert s.refactor_values(v2), s.last_error_message()
        o, counts = check_against_oracle(s, n, r, c, v2, check_sparse_only=True)
        assert counts["sparse"] >= 4, counts
        check_solution(s, o, n, r, c, v2, seed=10 + step)


@pytest.mark.gpu
def test_refactor_that_fails_the_pivot_test_moves_the_block_dense():
    n, r, c, v = sparse_block_system(0, SIZES, 0.5)
    s = engine(n, r, c, v)
    d = s.decomposition()
    R, P, Q = d["R"], d["P"], d["Q"]
    routes = route_of_blocks(s)
    b = max((b for b in range(len(R) - 1) if routes[b] and routes[b][0] == SPARSE),
            key=lambda b: R[b + 1] - R[b])
    # Shrink the block's first diagonal entry: column 0 of the block then
    # wants a row swap, which the gate refuses.
    k = np.nonzero((r == P[R[b]]) & (c == Q[R[b]]))[0]
    assert k.size == 1
    v2 = v.copy()
    v2[k] *= 1e-9
    assert s.refactor_values(v2), s.last_error_message()
    after = route_of_blocks(s)
    assert after[b][0] != SPARSE and after[b][1] == 2, after[b]
    o, _ = check_against_oracle(s, n, r, c, v2)
    check_solution(s, o, n, r, c, v2)
    # The block stays dense for the handle, with the original values too.
    assert s.refactor_values(v), s.last_error_message()
    assert route_of_blocks(s)[b][0] != SPARSE


@pytest.mark.gpu
def test_refactor_solve_without_status_wait_moves_the_failing_block_dense():
    """bdlu_refactor_solve queues the refactor with no status wait of its own;
    the solve finds the failed pivot test after its first sweep, factors
    again with the block on the dense route (a re-plan that replaces every
    engine buffer) and solves from the caller's right-hand sides."""
    n, r, c, v = sparse_block_system(0, SIZES, 0.5)
    s = engine(n, r, c, v)
    d = s.decomposition()
    R, P, Q = d["R"], d["P"], d["Q"]
    routes = route_of_blocks(s)
    b = max((b for b in range(len(R) - 1) if routes[b] and routes[b][0] == SPARSE),
            key=lambda b: R[b + 1] - R[b])
    k = np.nonzero((r == P[R[b]]) & (c == Q[R[b]]))[0]
    v2 = v.copy()
    v2[k] *= 1e-9
    rhs = np.asfortranarray(np.random.default_rng(21).uniform(-1, 1, (n, 2)))
    X = rhs.copy(order="F")
    lib = s._lib
    assert lib.bdlu_refactor_solve(s._h, v2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(v2),
                                   X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n, 2) == 0, \
        s.last_error_message()
    assert route_of_blocks(s)[b][0] != SPARSE
    o, _ = check_against_oracle(s, n, r, c, v2)
    for col in range(2):
        x_o = o.solve(rhs[:, col])
        assert np.max(np.abs(X[:, col] - x_o) / np.maximum(1.0, np.abs(x_o))) <= X_TOL
        assert oracle.metrics(r, c, v2, X[:, col], rhs[:, col])[0] <= RESID_TOL


@pytest.mark.gpu
def test_sparse_route_multi_rhs_and_export():
    n, r, c, v = sparse_block_system(2, [90, 40, 120, 75], 0.5)
    s = engine(n, r, c, v)
    o, counts = check_against_oracle(s, n, r, c, v)
    assert counts["sparse"] >= 1
    check_solution(s, o, n, r, c, v, nrhs=8)

    def dense(coo, shape):
        rr, cc, vv = (np.array(t) for t in zip(*coo))
        return sp.csr_matrix((vv, (rr, cc)), shape=shape).toarray()

    L = dense(s.getL(), (n, n))
    U = dense(s.getU(), (n, n))
    A = dense(s.get_rearranged_matrix(), (n, n))
    assert np.abs(L @ U - A).max() <= 1e-12 * max(1.0, np.abs(A).max())


@pytest.mark.gpu
def test_fill_limit_selects_sparse_blocks():
    n, r, c, v = sparse_block_system(0, SIZES, 0.5)
    limit = 0.085
    s = engine(n, r, c, v, mode=2, fill_max=limit)
    d = s.decomposition()
    R, P, Q = d["R"], d["P"], d["Q"]
    Ap = sp.csr_matrix((v, (r, c)), shape=(n, n)).toarray()[P][:, Q]
    o = oracle.System(n, r, c, v, P, Q, R)
    ok, reason = o.factor_gp()
    routes = route_of_blocks(s)
    over = 0
    for b in range(len(R) - 1):
        m = int(R[b + 1] - R[b])
        if m <= 64:
            continue
        fill = no_pivot_fill(Ap[R[b]:R[b + 1], R[b]:R[b + 1]])
        if fill > limit * m * m:
            assert routes[b][0] != SPARSE and routes[b][1] == 5, (b, m, routes[b])
            over += 1
        else:
            assert (routes[b][0] == SPARSE) == (reason[b] == 0), (b, m, routes[b], reason[b])
    assert over >= 1
    check_against_oracle(s, n, r, c, v, check_sparse_only=True)


@pytest.mark.gpu
def test_bounded_waits_run_out_and_recover():
    """A one-poll wait limit makes the columns' and rows' waits on each other
    run out: the factor and the solve return errors, and the same handle
    works again with the default limit."""
    n, r, c, v = sparse_block_system(0, SIZES, 0.5)
    s = engine(n, r, c, v)
    x = np.ones(n)
    s.set_option("wait_limit", 1)
    assert not s.solve_in_place(x.copy())
    assert "bounded wait" in s.last_error_message()
    assert not s.refactor_values(v)
    assert "bounded wait between columns" in s.last_error_message()
    s.set_option("wait_limit", 0)
    assert s.refactor_values(v), s.last_error_message()
    o, counts = check_against_oracle(s, n, r, c, v, check_sparse_only=True)
    assert counts["sparse"] >= 4
    check_solution(s, o, n, r, c, v)


@pytest.mark.gpu
def test_environment_selects_the_route(monkeypatch):
    n, r, c, v = sparse_block_system(0, SIZES, 0.5)

    def routes():
        s = bd.Solver()
        assert s.set_matrix((r, c, v), n) and s.analyze() and s.factor(), s.last_error_message()
        return s.unit_routes()[1]

    assert SPARSE not in routes()
    monkeypatch.setenv("USERALGO_SPARSE_LU_KERNEL", "gp")
    assert SPARSE in routes()
    monkeypatch.setenv("USERALGO_GP_MAX_N", "80")
    on = routes()
    start = bd.Solver()
    assert start.set_matrix((r, c, v), n) and start.analyze()
    sizes = np.diff(np.append(start.unit_routes()[0], n))
    assert all(sizes[on == SPARSE] <= 80)
    monkeypatch.delenv("USERALGO_GP_MAX_N")
    # Row scaling is not implemented on the device: the route turns off.
    monkeypatch.setenv("USERALGO_GP_SCALE", "1")
    assert SPARSE not in routes()
