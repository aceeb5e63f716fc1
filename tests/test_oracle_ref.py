"""The oracle restatement against the reference's own sources compiled here
(oracle/_ref, see oracle/Makefile), CPU only.  Skipped when the reference
build is absent (it needs the reference sources at build time)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import blockdaglu as bd
import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
REF_LIB = os.path.join(REF_DIR, "libbdlu_ref.so")
REF_TESTS = os.path.join(REF_DIR, "blockdaglu_tests")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build (oracle/_ref) not present")

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def ref_lib():
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_decompose.restype = ctypes.c_void_p
    lib.ref_decompose.argtypes = [_i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32]
    for name in ("ref_nblocks", "ref_max_level", "ref_offdiag_nnz"):
        getattr(lib, name).restype = ctypes.c_int32
        getattr(lib, name).argtypes = [ctypes.c_void_p]
    lib.ref_get_decomposition.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p, _i32p, _f64p, _i32p]
    lib.ref_factor.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    lib.ref_block_lu.restype = ctypes.c_int32
    lib.ref_block_lu.argtypes = [ctypes.c_void_p, ctypes.c_int32, _f64p, _i32p]
    lib.ref_block_solve.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int32, ctypes.c_int32]
    lib.ref_run_free.argtypes = [ctypes.c_void_p]
    return lib


def p32(a):
    return a.ctypes.data_as(_i32p)


def p64(a):
    return a.ctypes.data_as(_f64p)


def test_reference_test_program_passes():
    # apps/tests/main.cpp, built against the reference sources + stand-in.
    r = subprocess.run([REF_TESTS], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "All BlockDAGLU tests passed" in r.stdout


@pytest.mark.parametrize("family,seed,n", [
    (bd.FAMILY_BLOCK, bd.config_seed(0), 2000),
    (bd.FAMILY_BLOCK, bd.config_seed(0, 1), 2000),
    (bd.FAMILY_CIRCUIT, bd.config_seed(1, 3), 20000),
])
def test_oracle_and_engine_analysis_equal_reference(monkeypatch, family, seed, n):
    # BLOCK_SCHED=level makes the reference build its DAG levels.  The
    # reference's env.h:15-25 compares only 8 characters of "USERALGO_" and
    # then looks up "BLOCKDAGLU__X", so only the USERALGO_ name reaches it.
    monkeypatch.setenv("USERALGO_BLOCK_SCHED", "level")
    g = bd.Synth(family, seed, n)
    lib = ref_lib()
    # The reference build's btf_order is the oracle's own BTF; here it is
    # handed the engine's ordering of the same pattern (n < 50,000: no small
    # entries dropped) so both sides start from one permutation.
    a = sp.csc_matrix((np.ones(g.nnz), (g.rows, g.cols)), shape=(g.n, g.n))
    a.sort_indices()
    nb_e, P_e, Q_e, R_e, nm_e = bd.btf_order(g.n, a.indptr, a.indices)
    oracle.inject_reference_btf(g.n, P_e, Q_e, R_e, nm_e)
    try:
        run = lib.ref_decompose(p32(g.rows), p32(g.cols), p64(g.vals), g.nnz, g.n)
    finally:
        oracle.inject_reference_btf(g.n)
    assert run
    try:
        nb, noff = lib.ref_nblocks(run), lib.ref_offdiag_nnz(run)
        P, Q = np.empty(g.n, np.int32), np.empty(g.n, np.int32)
        R = np.empty(nb + 1, np.int32)
        optr, ocol = np.empty(g.n + 1, np.int32), np.empty(noff, np.int32)
        oval, lev = np.empty(noff), np.empty(nb, np.int32)
        lib.ref_get_decomposition(run, p32(P), p32(Q), p32(R), p32(optr), p32(ocol), p64(oval), p32(lev))
        # Engine host analysis == reference (same BTF permutation by construction).
        s = bd.Solver()
        s.set_option("analysis_only", 1)
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze()
        d = s.decomposition()
        for key, ref_val in (("P", P), ("Q", Q), ("R", R), ("off_ptr", optr), ("off_col", ocol), ("level", lev)):
            assert np.array_equal(d[key], ref_val), key
        assert np.array_equal(g.vals[d["off_src"]], oval)
        # Oracle restatement == reference: split and levels.
        sysm = oracle.System(g.n, g.rows, g.cols, g.vals, P, Q, R)
        o_ptr, o_col, o_val = sysm.offdiag()
        assert np.array_equal(o_ptr, optr) and np.array_equal(o_col, ocol) and np.array_equal(o_val, oval)
        o_lev, o_mx = sysm.levels()
        assert np.array_equal(o_lev, lev) and o_mx == lib.ref_max_level(run)
        # Dense micro-kernel factors: oracle == reference bit for bit.
        assert lib.ref_factor(run, 4) == 0
        assert sysm.factor()
        for b in range(nb):
            m = R[b + 1] - R[b]
            if m > 64:
                continue  # the reference sends these to KLU (stand-in here)
            lu = np.empty(m * m)
            piv = np.empty(m, np.int32)
            assert lib.ref_block_lu(run, b, p64(lu), p32(piv)) == m
            o_lu, o_piv = sysm.block_lu(b)
            assert np.array_equal(piv, o_piv), b
            assert np.array_equal(lu.reshape(m, m), o_lu), b
        # Reverse block solve.  Blocks above 64 rows go to the KLU stand-in,
        # whose threshold pivoting (tol 1e-3, KLU's default rule) is less
        # backward stable than partial pivoting: the bound is looser there.
        x = g.b[:, 0].copy()
        assert lib.ref_block_solve(run, p64(x), g.n, 1) == 0
        assert oracle.metrics(g.rows, g.cols, g.vals, x, g.b[:, 0])[0] <= 1e-9
        xo = sysm.solve(g.b[:, 0])
        assert oracle.metrics(g.rows, g.cols, g.vals, xo, g.b[:, 0])[0] <= 1e-12
    finally:
        lib.ref_run_free(run)


@pytest.mark.parametrize("family,seed,n,mode", [
    (bd.FAMILY_BLOCK, bd.config_seed(0), 2000, "KLU"),
    (bd.FAMILY_CIRCUIT, bd.config_seed(1, 3), 20000, "KLU"),
    (bd.FAMILY_CIRCUIT, bd.config_seed(1, 4), 60000, "BLOCK"),
    (bd.FAMILY_BLOCK, bd.config_seed(2, 7), 45000, "KLU"),
])
def test_auto_route_and_signatures_equal_reference(monkeypatch, family, seed, n, mode):
    """selected_mode() under AUTO and the three matrix signatures, engine vs the
    reference's own code (solver.cpp:96-136, :448-506, :846-861).  The
    reference build analyses with the oracle's BTF; no engine code there."""
    monkeypatch.delenv("BLOCKDAGLU_MODE", raising=False)
    monkeypatch.delenv("USERALGO_MODE", raising=False)
    g = oracle.Synth(family, seed, n)
    # Shuffled input order with a duplicate pair, so canonicalisation matters.
    rng = np.random.default_rng(n)
    perm = rng.permutation(g.nnz)
    rows = np.concatenate([g.rows[perm], g.rows[:1]])
    cols = np.concatenate([g.cols[perm], g.cols[:1]])
    vals = np.concatenate([g.vals[perm], [g.vals[0] * 0.5]])
    vals[np.argsort(perm)[0]] = g.vals[0] * 0.5
    lib = oracle.load_reference()
    lib.ref_matrix_sigs.restype = ctypes.c_int
    lib.ref_matrix_sigs.argtypes = [_i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64)]
    sigs = (ctypes.c_uint64 * 3)()
    nref = ctypes.c_int32()
    assert lib.ref_matrix_sigs(p32(rows), p32(cols), p64(vals), len(rows), -1, ctypes.byref(nref), sigs) == 0
    s = bd.Solver()
    s.set_option("analysis_only", 1)
    assert s.set_matrix((rows, cols, vals), -1) and s.analyze(), s.last_error_message()
    assert s.n() == nref.value == g.n
    assert s.signatures() == tuple(int(v) for v in sigs)
    ref = oracle.RefSolver()
    assert ref.set_matrix(rows, cols, vals, -1) and ref.analyze(), ref.last_error_message()
    assert s.selected_mode() == ref.selected_mode() == mode
