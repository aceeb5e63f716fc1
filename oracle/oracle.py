"""ctypes access to the oracle (test infrastructure: only tests/, the smoke check
and bench.py's cpu_baseline leg use it, always as the checker).

liboracle.so is the C restatement in bdlu_oracle.c; canonicalize_small is a
pure-Python restatement of validate_and_canonicalize_matrix
(blockdaglu/src/solver.cpp:642-722) for small inputs.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libbdlu_ref.so")
_lib = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    srcs = ("bdlu_oracle.c", "btf_oracle.c", "synth_oracle.c", "gp_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(os.path.join(HERE, f)) for f in srcs):
        build()
    lib = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    sig = {
        "or_merge_block_boundaries": (ctypes.c_int32, [_i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p]),
        "or_dense_lu": (ctypes.c_int, [_f64p, _i32p, ctypes.c_int32]),
        "or_dense_solve": (ctypes.c_int, [_f64p, _i32p, ctypes.c_int32, _f64p]),
        "or_split": (vp, [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _f64p, _i32p, _i32p, _i32p, ctypes.c_int32,
                          ctypes.c_double]),
        "or_free": (None, [vp]),
        "or_levels": (None, [vp, _i32p, _i32p]),
        "or_factor": (ctypes.c_int, [vp]),
        "or_block_lu": (_f64p, [vp, ctypes.c_int32, ctypes.POINTER(_i32p), _i32p]),
        "or_block_solve": (ctypes.c_int, [vp, _f64p]),
        "or_solve_system": (ctypes.c_int, [vp, _f64p, ctypes.c_int]),
        "or_metrics": (None, [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p]),
        "or_failed_block": (ctypes.c_int32, [vp]),
        "or_nblocks": (ctypes.c_int32, [vp]),
        "or_offdiag_nnz": (ctypes.c_int32, [vp]),
        "or_get_offdiag": (None, [vp, _i32p, _i32p, _f64p]),
        "or_btf_order": (ctypes.c_int32, [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "or_synth_create": (vp, [ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
        "or_synth_free": (None, [vp]),
        "or_synth_n": (ctypes.c_int32, [vp]),
        "or_synth_nnz": (ctypes.c_int64, [vp]),
        "or_synth_copy": (None, [vp, _i32p, _i32p, _f64p, _f64p, _f64p]),
        "or_synth_perturb": (None, [vp, ctypes.c_uint64, _f64p]),
        "or_gp_lu": (ctypes.c_int, [ctypes.c_int32, _i32p, _i32p, _f64p, ctypes.c_int32, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double, _f64p, _i32p, _f64p,
                                    ctypes.c_void_p]),
        "or_gp_gate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_double]),
        "or_factor_gp": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, _i32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p32(a):
    return a.ctypes.data_as(_i32p) if a is not None else None


def _p64(a):
    return a.ctypes.data_as(_f64p) if a is not None else None


def merge_block_boundaries(R, n, merge_max=64):
    lib = load()
    r = np.ascontiguousarray(R, np.int32)
    out = np.empty(len(r) + 2, np.int32)
    k = lib.or_merge_block_boundaries(_p32(r), len(r), int(n), int(merge_max), _p32(out))
    return out[:k].copy()


def dense_lu(a):
    """Reference micro-kernel on a row-major copy; returns (ok, lu, piv)."""
    lib = load()
    m = a.shape[0]
    lu = np.ascontiguousarray(a, np.float64).copy()
    piv = np.zeros(m, np.int32)
    ok = lib.or_dense_lu(_p64(lu), _p32(piv), m)
    return bool(ok), lu, piv


class _GpStats(ctypes.Structure):
    _fields_ = [("ok", ctypes.c_int32), ("row_swaps", ctypes.c_int32), ("tiny_pivots", ctypes.c_int32),
                ("zero_pivots", ctypes.c_int32), ("min_abs_diag", ctypes.c_double)]


# GpLuOptions defaults (blockdaglu/src/gp_lu.h:43-49) and the gate's defaults
# (blockdaglu/src/ubtf_block_solver.cpp:118-157).
GP_DEFAULTS = dict(scale=0, diag_prefer_tol=1e-3, pivot_tol=1e-12, perturb=1e-12, drop_tol=0.0)
GP_GATE_DEFAULTS = dict(require_no_swaps=1, swap_max_n=256, swap_max=0, require_no_tiny=1, min_abs_diag=1e-12)


def gp_lu(m, col_ptr, row_ind, val, **opts):
    """Restated gp_lu_factor on an m x m CSC (gp_oracle.c).  Returns (ok, lu,
    piv, row_scale, stats): lu row-major with L multipliers below the
    diagonal, piv LAPACK style, stats a dict of the diagnostics."""
    lib = load()
    o = dict(GP_DEFAULTS, **opts)
    cp = np.ascontiguousarray(col_ptr, np.int32)
    ri = np.ascontiguousarray(row_ind, np.int32)
    v = np.ascontiguousarray(val, np.float64)
    lu = np.zeros((m, m))
    piv = np.zeros(m, np.int32)
    rs = np.ones(m)
    st = _GpStats()
    ok = lib.or_gp_lu(int(m), _p32(cp), _p32(ri), _p64(v), int(o["scale"]), float(o["diag_prefer_tol"]),
                      float(o["pivot_tol"]), float(o["perturb"]), float(o["drop_tol"]), _p64(lu), _p32(piv), _p64(rs),
                      ctypes.byref(st))
    stats = {f: getattr(st, f) for f, _ in _GpStats._fields_}
    stats["_c"] = st
    return bool(ok), lu, piv, rs, stats


def gp_gate(stats, m, **opts):
    """Restated gp_gate_eval: 0 accepted, else the reject reason (1-4)."""
    o = dict(GP_GATE_DEFAULTS, **opts)
    return int(load().or_gp_gate(ctypes.byref(stats["_c"]), int(m), int(o["require_no_swaps"]), int(o["swap_max_n"]),
                                 int(o["swap_max"]), int(o["require_no_tiny"]), float(o["min_abs_diag"])))


def metrics(rows, cols, vals, x, b, x_true=None, n=None):
    """(inf-norm relative residual, l2 relative residual, l2 relative error)."""
    lib = load()
    r = np.ascontiguousarray(rows, np.int32)
    c = np.ascontiguousarray(cols, np.int32)
    v = np.ascontiguousarray(vals, np.float64)
    xx = np.ascontiguousarray(x, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    xt = np.ascontiguousarray(x_true, np.float64) if x_true is not None else None
    out = np.zeros(3)
    lib.or_metrics(int(n if n is not None else len(xx)), len(r), _p32(r), _p32(c), _p64(v), _p64(xx), _p64(bb), _p64(xt),
                   _p64(out))
    return float(out[0]), float(out[1]), float(out[2])


def btf_order(n, col_ptr, row_ind):
    """The oracle's block triangular form (btf_oracle.c), SuiteSparse btf_order
    conventions: (nblocks, P, Q, R, nmatch)."""
    lib = load()
    ap = np.ascontiguousarray(col_ptr, np.int32)
    ai = np.ascontiguousarray(row_ind, np.int32)
    P, Q, R = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n + 1, np.int32)
    nm = np.zeros(1, np.int32)
    nb = lib.or_btf_order(int(n), _p32(ap), _p32(ai), _p32(P), _p32(Q), _p32(R), _p32(nm))
    if nb < 0:
        raise MemoryError("or_btf_order failed")
    return nb, P, Q, R[: nb + 1].copy(), int(nm[0])


FAMILY_BLOCK, FAMILY_CIRCUIT = 0, 1


def config_seed(config, instance=0):
    """Seeds of the synthetic configurations: 20261203 + 1000*config + instance."""
    return 20261203 + 1000 * config + instance


class Synth:
    """Seeded synthetic system from the oracle's generator (synth_oracle.c):
    canonical COO, x_true, b; same draws as the benchmark's generator."""

    def __init__(self, family, seed, n, param=0, nrhs=1):
        self._lib = load()
        self._s = self._lib.or_synth_create(int(family), int(seed), int(n), int(param), int(nrhs))
        if not self._s:
            raise ValueError("unknown synthetic family %r" % family)
        self.n = self._lib.or_synth_n(self._s)
        self.nnz = self._lib.or_synth_nnz(self._s)
        self.nrhs = max(1, int(nrhs))
        self.rows = np.empty(self.nnz, np.int32)
        self.cols = np.empty(self.nnz, np.int32)
        self.vals = np.empty(self.nnz, np.float64)
        self.x_true = np.empty((self.n, self.nrhs), np.float64, order="F")
        self.b = np.empty((self.n, self.nrhs), np.float64, order="F")
        self._lib.or_synth_copy(self._s, _p32(self.rows), _p32(self.cols), _p64(self.vals), _p64(self.x_true),
                                _p64(self.b))

    def perturbed(self, seed):
        out = np.empty(self.nnz, np.float64)
        self._lib.or_synth_perturb(self._s, int(seed), _p64(out))
        return out

    def __del__(self):
        s, self._s = getattr(self, "_s", None), None
        if s and getattr(self, "_lib", None) is not None:
            self._lib.or_synth_free(s)


_ref = None


def load_reference():
    """The reference's own sources built under _ref (make -C oracle ref)."""
    global _ref
    if _ref is not None:
        return _ref
    if not os.path.exists(REF_LIB):
        raise FileNotFoundError(REF_LIB)
    lib = ctypes.CDLL(REF_LIB)
    vp = ctypes.c_void_p
    sig = {
        "ref_solver_create": (vp, []),
        "ref_solver_destroy": (None, [vp]),
        "ref_solver_set_coo": (ctypes.c_int, [vp, _i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32]),
        "ref_solver_analyze": (ctypes.c_int, [vp]),
        "ref_solver_factor": (ctypes.c_int, [vp]),
        "ref_solver_solve": (ctypes.c_int, [vp, _f64p, ctypes.c_int32]),
        "ref_solver_mode": (ctypes.c_char_p, [vp]),
        "ref_solver_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int64]),
        "btf_standin_inject": (None, [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int32, ctypes.c_int32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _ref = lib
    return lib


def inject_reference_btf(n, P=None, Q=None, R=None, nmatch=None):
    """Makes the reference build's btf_order return (P, Q, R) for order-n
    patterns (parity tests start both sides from one ordering); with P None
    the injection is cleared and the oracle's own BTF runs again."""
    lib = load_reference()
    if P is None:
        lib.btf_standin_inject(-1, None, None, None, 0, 0)
        return
    p, q, r = (np.ascontiguousarray(a, np.int32) for a in (P, Q, R))
    lib.btf_standin_inject(int(n), _p32(p), _p32(q), _p32(r), len(r) - 1, int(n if nmatch is None else nmatch))


class RefSolver:
    """blockdaglu::Solver of the reference build (set_matrix / analyze / factor /
    solve_in_place / selected_mode), for parity tests and the CPU baseline."""

    def __init__(self):
        self._lib = load_reference()
        self._h = self._lib.ref_solver_create()

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._lib.ref_solver_destroy(h)

    def set_matrix(self, rows, cols, vals, n=-1):
        r = np.ascontiguousarray(rows, np.int32)
        c = np.ascontiguousarray(cols, np.int32)
        v = np.ascontiguousarray(vals, np.float64)
        return self._lib.ref_solver_set_coo(self._h, _p32(r), _p32(c), _p64(v), len(r), int(n)) == 0

    def analyze(self):
        return self._lib.ref_solver_analyze(self._h) == 0

    def factor(self):
        return self._lib.ref_solver_factor(self._h) == 0

    def solve_in_place(self, b):
        assert b.dtype == np.float64 and b.flags.c_contiguous
        return self._lib.ref_solver_solve(self._h, _p64(b), len(b)) == 0

    def selected_mode(self):
        return self._lib.ref_solver_mode(self._h).decode()

    def last_error_message(self):
        buf = ctypes.create_string_buffer(512)
        self._lib.ref_solver_error(self._h, buf, 512)
        return buf.value.decode()


class System:
    """The reference's block route on a canonical COO under given (P, Q, merged R)."""

    def __init__(self, n, rows, cols, vals, P, Q, R, drop=None):
        self._lib = load()
        self.n = int(n)
        self._keep = [np.ascontiguousarray(a, t) for a, t in
                      ((rows, np.int32), (cols, np.int32), (vals, np.float64), (P, np.int32), (Q, np.int32), (R, np.int32))]
        r, c, v, p, q, rr = self._keep
        if drop is None:
            drop = 1e-20 if n >= 50000 else 0.0
        self._s = self._lib.or_split(self.n, len(r), _p32(r), _p32(c), _p64(v), _p32(p), _p32(q), _p32(rr), len(rr) - 1,
                                     float(drop))
        if not self._s:
            raise ValueError("permutation is not UBTF (found lower-block entries)")
        self.nblocks = len(rr) - 1

    def __del__(self):
        s, self._s = getattr(self, "_s", None), None
        if s:
            self._lib.or_free(s)

    def factor(self):
        self._factored = True
        return bool(self._lib.or_factor(self._s))

    def factor_gp(self, dense_max=64, gp_max_n=4096, diag_tol=1e-3, pivot_tol=1e-12, perturb=1e-12,
                  min_abs_diag=1e-12):
        """Factor with the reference's sparse-LU route on (or_factor_gp):
        returns (ok, reason) with reason[b] = -1 (block not tried), 0 (kept)
        or the gate's reject reason."""
        self._factored = True
        reason = np.full(self.nblocks, -1, np.int32)
        ok = self._lib.or_factor_gp(self._s, int(dense_max), int(gp_max_n), float(diag_tol), float(pivot_tol),
                                    float(perturb), float(min_abs_diag), _p32(reason))
        return bool(ok), reason

    def failed_block(self):
        return self._lib.or_failed_block(self._s)

    def levels(self):
        lev = np.zeros(self.nblocks, np.int32)
        mx = np.zeros(1, np.int32)
        self._lib.or_levels(self._s, _p32(lev), _p32(mx))
        return lev, int(mx[0])

    def offdiag(self):
        nnz = self._lib.or_offdiag_nnz(self._s)
        ptr = np.empty(self.n + 1, np.int32)
        col = np.empty(nnz, np.int32)
        val = np.empty(nnz, np.float64)
        self._lib.or_get_offdiag(self._s, _p32(ptr), _p32(col), _p64(val))
        return ptr, col, val

    def block_lu(self, b):
        piv = _i32p()
        m = ctypes.c_int32()
        ptr = self._lib.or_block_lu(self._s, int(b), ctypes.byref(piv), ctypes.byref(m))
        mm = m.value
        lu = np.ctypeslib.as_array(ptr, shape=(mm * mm,)).reshape(mm, mm).copy() if mm else np.zeros((0, 0))
        pv = np.ctypeslib.as_array(piv, shape=(mm,)).copy() if mm else np.zeros(0, np.int32)
        return lu, pv

    def solve(self, b, refine_iters=0):
        if not getattr(self, "_factored", False):
            raise RuntimeError("oracle System.solve before factor")
        x = np.ascontiguousarray(b, np.float64).copy()
        taken = self._lib.or_solve_system(self._s, _p64(x), int(refine_iters))
        if taken < 0:
            raise RuntimeError("oracle block solve failed")
        return x


# Error codes of blockdaglu::SolverError used below.
INVALID_DIMENSION, INVALID_INDEX, NON_FINITE = 2, 3, 4


def canonicalize_small(coo, dimension_hint=-1):
    """solver.cpp:642-722 for small inputs: returns (code, n, canonical list).

    Duplicate sums use math.fsum (correctly rounded); the reference sums in
    long double, which agrees on every input used by the tests."""
    if dimension_hint < -1:
        return INVALID_DIMENSION, 0, []
    max_index = -1
    for r, c, v in coo:
        if r < 0 or c < 0:
            return INVALID_INDEX, 0, []
        if not math.isfinite(v):
            return NON_FINITE, 0, []
        if dimension_hint >= 0 and (r >= dimension_hint or c >= dimension_hint):
            return INVALID_INDEX, 0, []
        max_index = max(max_index, r, c)
    n = dimension_hint if dimension_hint >= 0 else max_index + 1
    if n <= 0:
        return INVALID_DIMENSION, 0, []
    groups = {}
    for r, c, v in coo:
        groups.setdefault((r, c), []).append(v)
    out = []
    for key in sorted(groups):
        v = math.fsum(groups[key])
        if not math.isfinite(v):
            return NON_FINITE, 0, []
        if v != 0.0:
            out.append((key[0], key[1], v))
    return 0, n, out
