"""The oracle's restatement of the reference's sparse-LU route (gp_oracle.c,
or_factor_gp) against the reference's own gp_lu.cpp and factor_one_block,
compiled here under oracle/_ref.  CPU only; skipped without that build."""
import ctypes
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libbdlu_ref.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build (oracle/_ref) not present")

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def p32(a):
    return a.ctypes.data_as(_i32p)


def p64(a):
    return a.ctypes.data_as(_f64p)


def ref_lib():
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_gp_lu.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, ctypes.c_double, _f64p, _i32p, _f64p, _i32p]
    lib.ref_gp_solve.argtypes = [ctypes.c_int32, _i32p, _i32p, _f64p, _f64p]
    lib.ref_decompose.restype = ctypes.c_void_p
    lib.ref_decompose.argtypes = [_i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32]
    lib.ref_nblocks.restype = ctypes.c_int32
    lib.ref_nblocks.argtypes = [ctypes.c_void_p]
    lib.ref_get_decomposition.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p, _i32p, _f64p, _i32p]
    lib.ref_factor.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    lib.ref_block_route.restype = ctypes.c_int32
    lib.ref_block_route.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p]
    lib.ref_block_gp.restype = ctypes.c_int32
    lib.ref_block_gp.argtypes = [ctypes.c_void_p, ctypes.c_int32, _f64p, _i32p]
    lib.ref_block_lu.restype = ctypes.c_int32
    lib.ref_block_lu.argtypes = [ctypes.c_void_p, ctypes.c_int32, _f64p, _i32p]
    lib.ref_block_solve.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int32, ctypes.c_int32]
    lib.ref_run_free.argtypes = [ctypes.c_void_p]
    return lib


def ref_gp(lib, A, **opts):
    o = dict(oracle.GP_DEFAULTS, **opts)
    m = A.shape[0]
    lu = np.zeros((m, m))
    perm = np.zeros(m, np.int32)
    rs = np.ones(m)
    st = np.zeros(4, np.int32)
    ip = np.ascontiguousarray(A.indptr, np.int32)
    ix = np.ascontiguousarray(A.indices, np.int32)
    dv = np.ascontiguousarray(A.data, np.float64)
    ok = lib.ref_gp_lu(m, p32(ip), p32(ix), p64(dv), o["scale"], o["diag_prefer_tol"], o["pivot_tol"], o["perturb"],
                       o["drop_tol"], p64(lu), p32(perm), p64(rs), p32(st))
    return bool(ok), lu, perm, rs, st


def perm_of(piv):
    """Row order after LAPACK-style sequential swaps."""
    order = np.arange(len(piv))
    for k, p in enumerate(piv):
        order[[k, p]] = order[[p, k]]
    return order


def block_matrix(rng, m, density, diag_scale, cyclic=True, zero_diag=()):
    """An m x m sparse block: optional cyclic chain i -> i+1 (irreducible),
    random entries N(0,1), diagonal diag_scale * row sum of |off-diagonals|
    + N(0, 0.1); rows in zero_diag get no diagonal entry."""
    A = sp.random(m, m, density=density, random_state=rng, data_rvs=rng.standard_normal, format="lil")
    if cyclic:
        for i in range(m):
            A[i, (i + 1) % m] = rng.standard_normal()
    A = A.tocsr()
    A.setdiag(0.0)
    A.eliminate_zeros()
    d = diag_scale * np.asarray(abs(A).sum(axis=1)).ravel() + 0.1 * rng.standard_normal(m)
    A = A + sp.diags(d)
    A = A.tolil()
    for i in zero_diag:
        A[i, i] = 0.0
    A = A.tocsc()
    A.eliminate_zeros()
    A.sort_indices()
    return A


CASES = [
    # (m, density, diagonal scale, options)
    (70, 0.05, 1.5, {}),                                  # dominant: no swaps
    (90, 0.06, 0.3, {}),                                  # weak diagonal: swaps
    (120, 0.03, 0.5, {"diag_prefer_tol": 0.5}),           # stricter diagonal preference
    (60, 0.08, 0.2, {"scale": 1}),                        # row scaling by sums
    (75, 0.05, 0.2, {"scale": 2, "drop_tol": 1e-3}),      # max scaling and dropping
    (50, 0.10, 1.0, {"pivot_tol": 0.5, "perturb": 0.0}),  # tiny pivots perturbed by pivot_tol
    (40, 0.10, 1.0, {"pivot_tol": 0.5, "perturb": 1e-3}),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_gp_lu_bit_identical_to_reference(case):
    m, dens, dsc, opts = CASES[case]
    lib = ref_lib()
    rng = np.random.default_rng(100 + case)
    A = block_matrix(rng, m, dens, dsc)
    ok_r, lu_r, perm_r, rs_r, st_r = ref_gp(lib, A, **opts)
    ok_o, lu_o, piv_o, rs_o, st_o = oracle.gp_lu(m, A.indptr, A.indices, A.data, **opts)
    assert ok_r == ok_o
    assert [st_o["ok"], st_o["row_swaps"], st_o["tiny_pivots"], st_o["zero_pivots"]] == list(st_r)
    if ok_r:
        assert np.array_equal(perm_of(piv_o), perm_r)
        assert np.array_equal(rs_o, rs_r)
        assert np.array_equal(lu_o, lu_r), np.abs(lu_o - lu_r).max()
        if opts.get("drop_tol", 0.0) > 0.0 or st_o["tiny_pivots"]:
            return  # dropped entries and perturbed pivots make L U an approximation
        # L U = P D A for the restatement too.
        L = np.tril(lu_o, -1) + np.eye(m)
        U = np.triu(lu_o)
        PA = (sp.diags(rs_o) @ A).toarray()[perm_of(piv_o)]
        assert np.abs(L @ U - PA).max() <= 1e-10 * max(1.0, np.abs(PA).max())


def test_gp_cases_cover_swaps_tiny_pivots_and_failures():
    lib = ref_lib()
    seen = set()
    for case, (m, dens, dsc, opts) in enumerate(CASES):
        A = block_matrix(np.random.default_rng(100 + case), m, dens, dsc)
        ok, _, _, _, st = ref_gp(lib, A, **opts)
        if st[1]:
            seen.add("swaps")
        if st[2]:
            seen.add("tiny")
        if ok and not st[1] and not st[2]:
            seen.add("clean")
    assert seen == {"swaps", "tiny", "clean"}
    # A structurally singular column fails in both.
    A = block_matrix(np.random.default_rng(7), 30, 0.1, 1.0).tolil()
    A[:, 5] = 0.0
    A = A.tocsc()
    A.eliminate_zeros()
    A.sort_indices()
    ok_r, *_, st_r = ref_gp(lib, A)
    ok_o, *_, st_o = oracle.gp_lu(30, A.indptr, A.indices, A.data)
    assert not ok_r and not ok_o and st_r[3] == st_o["zero_pivots"] == 1


@pytest.mark.parametrize("stats,m,opts,want", [
    (dict(ok=0, row_swaps=0, tiny_pivots=0, zero_pivots=1, min_abs_diag=0.0), 80, {}, 1),
    (dict(ok=1, row_swaps=2, tiny_pivots=0, zero_pivots=0, min_abs_diag=1.0), 80, {}, 2),
    (dict(ok=1, row_swaps=2, tiny_pivots=0, zero_pivots=0, min_abs_diag=1.0), 80, {"swap_max": 2}, 0),
    (dict(ok=1, row_swaps=2, tiny_pivots=0, zero_pivots=0, min_abs_diag=1.0), 300, {"swap_max": 2}, 2),
    (dict(ok=1, row_swaps=0, tiny_pivots=1, zero_pivots=0, min_abs_diag=1.0), 80, {}, 3),
    (dict(ok=1, row_swaps=0, tiny_pivots=0, zero_pivots=0, min_abs_diag=1e-13), 80, {}, 4),
    (dict(ok=1, row_swaps=0, tiny_pivots=0, zero_pivots=0, min_abs_diag=1e-12), 80, {}, 0),
])
def test_gp_gate_reasons(stats, m, opts, want):
    st = oracle._GpStats(**stats)
    assert oracle.gp_gate({"_c": st}, m, **opts) == want


def gp_system(seed, sizes, scales):
    """Upper block triangular system of irreducible blocks (sizes, diagonal
    scales) with coupling above the blocks, randomly permuted."""
    rng = np.random.default_rng(seed)
    n = sum(sizes)
    blocks = [block_matrix(rng, m, min(0.5, 4.0 / m), s) for m, s in zip(sizes, scales)]
    A = sp.block_diag(blocks, format="lil")
    off = 0
    for m in sizes[:-1]:
        for i in range(off, off + m):
            j = rng.integers(off + m, n)
            A[i, j] = 0.1 * rng.standard_normal()
        off += m
    A = A.tocsr()
    p, q = rng.permutation(n), rng.permutation(n)
    A = A[p][:, q].tocoo()
    return n, A.row.astype(np.int32), A.col.astype(np.int32), A.data.astype(np.float64)


def canonical(n, r, c, v):
    A = sp.csr_matrix((v, (r, c)), shape=(n, n))
    A.sum_duplicates()
    A.eliminate_zeros()
    A = A.tocoo()
    order = np.lexsort((A.col, A.row))
    return A.row[order].astype(np.int32), A.col[order].astype(np.int32), A.data[order].astype(np.float64)


def test_block_route_matches_reference(monkeypatch):
    """factor_one_block with USERALGO_SPARSE_LU_KERNEL=gp: the same blocks
    take the sparse-LU route, with bit-identical factors; dense blocks stay
    bit-identical; the solution agrees."""
    monkeypatch.setenv("USERALGO_SPARSE_LU_KERNEL", "gp")
    lib = ref_lib()
    sizes = [70, 30, 90, 120, 20, 100, 66]
    scales = [1.5, 1.0, 0.3, 2.0, 1.0, 0.4, 1.2]
    n, r, c, v = gp_system(5, sizes, scales)
    r, c, v = canonical(n, r, c, v)
    run = lib.ref_decompose(p32(r), p32(c), p64(v), len(r), n)
    assert run
    try:
        nb = lib.ref_nblocks(run)
        P, Q, R = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(nb + 1, np.int32)
        lib.ref_get_decomposition(run, p32(P), p32(Q), p32(R), None, None, None, None)
        assert lib.ref_factor(run, 1) == 0
        s = oracle.System(n, r, c, v, P, Q, R)
        ok, reason = s.factor_gp()
        assert ok
        kinds = {0: 0, 1: 0, 2: 0}
        for b in range(nb):
            m = R[b + 1] - R[b]
            rr = np.zeros(1, np.int32)
            route = lib.ref_block_route(run, b, p32(rr))
            kinds[route] += 1
            lu_o, piv_o = s.block_lu(b)
            if route == 1:
                assert reason[b] == 0
                lu = np.zeros((m, m))
                perm = np.zeros(m, np.int32)
                assert lib.ref_block_gp(run, b, p64(lu), p32(perm)) == m
                assert np.array_equal(perm, np.arange(m))
                assert np.array_equal(lu, lu_o)
            elif route == 2:
                assert reason[b] == rr[0] and reason[b] > 0
            else:
                assert reason[b] == -1
                lu = np.zeros(m * m)
                piv = np.zeros(m, np.int32)
                assert lib.ref_block_lu(run, b, p64(lu), p32(piv)) == m
                assert np.array_equal(lu.reshape(m, m), lu_o) and np.array_equal(piv, piv_o)
        assert kinds[1] >= 1 and kinds[2] >= 1, kinds
        b = np.random.default_rng(9).uniform(-1, 1, n)
        x_ref = b.copy()
        assert lib.ref_block_solve(run, p64(x_ref), n, 1) == 0
        x = s.solve(b)
        assert np.max(np.abs(x - x_ref) / np.maximum(1.0, np.abs(x_ref))) <= 1e-9
    finally:
        lib.ref_run_free(run)


def test_gp_solve_matches_reference():
    """or_dense_solve on an accepted sparse factor (identity pivots) follows
    gp_lu_solve_inplace_strided's order: the same x bit for bit."""
    lib = ref_lib()
    A = block_matrix(np.random.default_rng(3), 150, 0.03, 2.0)
    ok, lu, piv, _, st = oracle.gp_lu(150, A.indptr, A.indices, A.data)
    assert ok and st["row_swaps"] == 0
    b = np.random.default_rng(4).uniform(-1, 1, 150)
    x_ref = b.copy()
    assert lib.ref_gp_solve(150, p32(A.indptr.astype(np.int32)), p32(A.indices.astype(np.int32)),
                            p64(A.data.astype(np.float64)), p64(x_ref)) == 1
    x = b.copy()
    olib = oracle.load()
    assert olib.or_dense_solve(p64(np.ascontiguousarray(lu)), p32(piv), 150, p64(x)) == 1
    assert np.array_equal(x, x_ref)
