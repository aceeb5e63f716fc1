"""Python mirror of blockdaglu::Solver over the B200 engine's C ABI (include/bdlu.h).

The class follows the reference interface (blockdaglu/include/blockdaglu/solver.h:43-126):
set_matrix / analyze / factor / solve_in_place return bool, and last_error() /
last_error_message() explain a False.  Additions: refactor_values (value-only
refactor), multi-RHS solves, device-pointer variants, stats.

The shared library is built in-tree by block-daglu_b200/build.py.  There is no
CPU fallback: if the library or a CUDA device is missing, loading or analyze
fails with BackendUnavailable.
"""
import ctypes
import enum
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbdlu.so")
_lib = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


class SolverError(enum.IntEnum):
    """blockdaglu::SolverError (solver.h:19-31)."""
    None_ = 0
    NotPrepared = 1
    InvalidDimension = 2
    InvalidIndex = 3
    NonFiniteValue = 4
    InvalidRightHandSide = 5
    BackendUnavailable = 6
    AnalysisFailed = 7
    FactorizationFailed = 8
    SolveFailed = 9
    ExportFailed = 10


class Stats(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32), ("nblocks", ctypes.c_int32), ("nblocks_raw", ctypes.c_int32),
        ("max_block", ctypes.c_int32), ("max_level", ctypes.c_int32), ("refine_iters", ctypes.c_int32),
        ("nunits", ctypes.c_int32), ("unit_levels", ctypes.c_int32), ("max_unit", ctypes.c_int32),
        ("factor_launches", ctypes.c_int32), ("solve_launches", ctypes.c_int32),
        ("nnz", ctypes.c_int64), ("nnz_offdiag", ctypes.c_int64), ("dense_entries", ctypes.c_int64),
        ("factor_flops", ctypes.c_double), ("residual_inf", ctypes.c_double),
        ("last_factor_ms", ctypes.c_double), ("last_solve_ms", ctypes.c_double),
        ("precision", ctypes.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("p50_ms", ctypes.c_double),
        ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
        ("throughput", ctypes.c_double), ("resident_bytes", ctypes.c_int64), ("evictions", ctypes.c_int64),
        ("peak_concurrency", ctypes.c_int32), ("kernel_launches", ctypes.c_int64), ("factor_flops", ctypes.c_double),
        ("mean_stage_ms", ctypes.c_double), ("mean_factor_ms", ctypes.c_double), ("mean_solve_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def load_library(path=LIB_PATH):
    """Loads libbdlu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libbdlu.so not found at %s; run python block-daglu_b200/build.py" % path)
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "bdlu_create": (vp, []),
        "bdlu_destroy": (None, [vp]),
        "bdlu_set_coo": (ctypes.c_int, [vp, _i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32]),
        "bdlu_analyze": (ctypes.c_int, [vp]),
        "bdlu_factor": (ctypes.c_int, [vp]),
        "bdlu_refactor_values": (ctypes.c_int, [vp, _f64p, ctypes.c_int64]),
        "bdlu_refactor_values_device": (ctypes.c_int, [vp, vp, ctypes.c_int64, vp]),
        "bdlu_solve": (ctypes.c_int, [vp, _f64p, ctypes.c_int32, ctypes.c_int32]),
        "bdlu_solve_device": (ctypes.c_int, [vp, vp, ctypes.c_int32, ctypes.c_int32, vp]),
        "bdlu_refactor_solve": (ctypes.c_int, [vp, _f64p, ctypes.c_int64, _f64p, ctypes.c_int32, ctypes.c_int32]),
        "bdlu_last_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int64]),
        "bdlu_n": (ctypes.c_int32, [vp]),
        "bdlu_selected_mode": (ctypes.c_char_p, [vp]),
        "bdlu_canonical_pattern": (ctypes.c_int64, [vp, _i32p, _i32p]),
        "bdlu_export_p": (ctypes.c_int64, [vp, _i32p, _i32p, _f64p, ctypes.c_int64]),
        "bdlu_export_q": (ctypes.c_int64, [vp, _i32p, _i32p, _f64p, ctypes.c_int64]),
        "bdlu_export_l": (ctypes.c_int64, [vp, _i32p, _i32p, _f64p, ctypes.c_int64]),
        "bdlu_export_u": (ctypes.c_int64, [vp, _i32p, _i32p, _f64p, ctypes.c_int64]),
        "bdlu_export_rearranged": (ctypes.c_int64, [vp, _i32p, _i32p, _f64p, ctypes.c_int64]),
        "bdlu_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(Stats)]),
        "bdlu_set_option": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_double]),
        "bdlu_phase_times": (ctypes.c_int, [vp, _f64p, ctypes.c_int32]),
        "bdlu_btf_order": (ctypes.c_int32, [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "bdlu_merge_block_boundaries": (ctypes.c_int32, [_i32p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _i32p]),
        "bdlu_get_decomposition": (ctypes.c_int, [vp, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "bdlu_get_block_lu": (ctypes.c_int32, [vp, ctypes.c_int32, _f64p, _i32p]),
        "bdlu_matrix_signatures": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "bdlu_get_unit_routes": (ctypes.c_int32, [vp, _i32p, _i32p, _i32p, ctypes.POINTER(ctypes.c_int64),
                                                  ctypes.c_int32]),
        "bdlu_tuner_report": (ctypes.c_int64, [ctypes.c_char_p, ctypes.c_int64]),
        "bdlu_batch_create": (vp, []),
        "bdlu_batch_destroy": (None, [vp]),
        "bdlu_batch_add": (ctypes.c_int32, [vp, _i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32]),
        "bdlu_batch_analyze": (ctypes.c_int, [vp]),
        "bdlu_batch_factor": (ctypes.c_int, [vp]),
        "bdlu_batch_refactor_values": (ctypes.c_int, [vp, _f64p, ctypes.c_int64]),
        "bdlu_batch_refactor_values_device": (ctypes.c_int, [vp, vp, ctypes.c_int64, vp]),
        "bdlu_batch_solve": (ctypes.c_int, [vp, _f64p, ctypes.c_int32, ctypes.c_int32]),
        "bdlu_batch_solve_device": (ctypes.c_int, [vp, vp, ctypes.c_int32, ctypes.c_int32, vp]),
        "bdlu_batch_count": (ctypes.c_int32, [vp]),
        "bdlu_batch_row_offset": (ctypes.c_int64, [vp, ctypes.c_int32]),
        "bdlu_batch_nnz_offset": (ctypes.c_int64, [vp, ctypes.c_int32]),
        "bdlu_batch_last_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int64]),
        "bdlu_batch_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(Stats)]),
        "bdlu_batch_phase_times": (ctypes.c_int, [vp, _f64p, ctypes.c_int32]),
        "bdlu_server_create": (vp, [ctypes.c_int64, ctypes.c_int32]),
        "bdlu_server_destroy": (None, [vp]),
        "bdlu_server_add_pattern": (ctypes.c_int32, [vp, _i32p, _i32p, _f64p, ctypes.c_int64, ctypes.c_int32]),
        "bdlu_server_pattern_nnz": (ctypes.c_int64, [vp, ctypes.c_int32]),
        "bdlu_server_pattern_bytes": (ctypes.c_int64, [vp, ctypes.c_int32]),
        "bdlu_server_submit": (ctypes.c_int64, [vp, ctypes.c_int32, _f64p, ctypes.c_int64, _f64p, ctypes.c_int32,
                                                ctypes.c_int32]),
        "bdlu_server_submit_device": (ctypes.c_int64, [vp, ctypes.c_int32, vp, ctypes.c_int64, vp, ctypes.c_int32,
                                                      ctypes.c_int32]),
        "bdlu_server_wait": (ctypes.c_int, [vp, ctypes.c_int64, _f64p, _f64p]),
        "bdlu_server_drain": (ctypes.c_int, [vp]),
        "bdlu_server_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
        "bdlu_server_reset_stats": (ctypes.c_int, [vp]),
        "bdlu_server_last_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int64]),
        "bdlu_server_set_option": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_double]),
        "bdlu_synth_create": (vp, [ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
        "bdlu_synth_destroy": (None, [vp]),
        "bdlu_synth_n": (ctypes.c_int32, [vp]),
        "bdlu_synth_nnz": (ctypes.c_int64, [vp]),
        "bdlu_synth_nrhs": (ctypes.c_int32, [vp]),
        "bdlu_synth_nblocks": (ctypes.c_int32, [vp]),
        "bdlu_synth_copy": (None, [vp, _i32p, _i32p, _f64p, _f64p, _f64p]),
        "bdlu_synth_block_sizes": (None, [vp, _i32p]),
        "bdlu_synth_perturb": (None, [vp, ctypes.c_uint64, _f64p]),
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


def _coo_arrays(coo):
    """Accepts a list of (row, col, value) tuples or a (rows, cols, vals) triple of arrays."""
    if isinstance(coo, tuple) and len(coo) == 3 and hasattr(coo[0], "__len__") and not np.isscalar(coo[0]):
        r, c, v = coo
    else:
        if len(coo) == 0:
            r, c, v = [], [], []
        else:
            r, c, v = zip(*coo)
    return (np.ascontiguousarray(r, dtype=np.int32), np.ascontiguousarray(c, dtype=np.int32),
            np.ascontiguousarray(v, dtype=np.float64))


class Solver:
    """blockdaglu::Solver (solver.h:43-126) on the B200 engine."""

    def __init__(self):
        self._lib = load_library()
        self._h = self._lib.bdlu_create()
        if not self._h:
            raise MemoryError("bdlu_create failed")

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and getattr(self, "_lib", None) is not None:
            self._lib.bdlu_destroy(h)

    # -- reference API -----------------------------------------------------------
    def set_matrix(self, coo, dimension=-1):
        r, c, v = _coo_arrays(coo)
        self._keep = (r, c, v)
        return self._lib.bdlu_set_coo(self._h, _p32(r), _p32(c), _p64(v), len(r), int(dimension)) == 0

    def analyze(self):
        return self._lib.bdlu_analyze(self._h) == 0

    def factor(self):
        return self._lib.bdlu_factor(self._h) == 0

    def solve_in_place(self, b):
        """b: float64 array (n,) or (n, nrhs) in Fortran order; overwritten with x."""
        if not isinstance(b, np.ndarray) or b.dtype != np.float64:
            raise TypeError("solve_in_place expects a float64 numpy array")
        if b.ndim == 1:
            nrhs, ldb = 1, b.shape[0]
            if not b.flags.c_contiguous:
                raise ValueError("b must be contiguous")
        else:
            if not b.flags.f_contiguous:
                raise ValueError("multi-RHS b must be Fortran-ordered (column-major)")
            ldb, nrhs = b.shape
        if ldb != self.n():
            # The reference rejects any size mismatch (solver.cpp:1357-1359).
            ldb = -1
        return self._lib.bdlu_solve(self._h, _p64(b), ldb, nrhs) == 0

    def last_error(self):
        return SolverError(self._lib.bdlu_last_error(self._h, None, 0))

    def last_error_message(self):
        buf = ctypes.create_string_buffer(1024)
        self._lib.bdlu_last_error(self._h, buf, len(buf))
        return buf.value.decode()

    def get_rearranged_matrix(self):
        return self._export(self._lib.bdlu_export_rearranged)

    def getP(self):
        return self._export(self._lib.bdlu_export_p)

    def getQ(self):
        return self._export(self._lib.bdlu_export_q)

    def getL(self):
        return self._export(self._lib.bdlu_export_l)

    def getU(self):
        return self._export(self._lib.bdlu_export_u)

    def n(self):
        return self._lib.bdlu_n(self._h)

    def selected_mode(self):
        return self._lib.bdlu_selected_mode(self._h).decode()

    # -- additions ---------------------------------------------------------------
    def refactor_values(self, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        return self._lib.bdlu_refactor_values(self._h, _p64(v), len(v)) == 0

    def refactor_values_device(self, dptr, nnz, stream=0):
        return self._lib.bdlu_refactor_values_device(self._h, ctypes.c_void_p(dptr), nnz, ctypes.c_void_p(stream)) == 0

    def solve_device(self, dptr, ldb, nrhs, stream=0):
        return self._lib.bdlu_solve_device(self._h, ctypes.c_void_p(dptr), ldb, nrhs, ctypes.c_void_p(stream)) == 0

    def set_option(self, key, value):
        return self._lib.bdlu_set_option(self._h, key.encode(), float(value)) == 0

    def stats(self):
        st = Stats()
        self._lib.bdlu_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()

    PHASES = ("gather", "lu_small", "lu_large", "solve", "refine_residual")

    def phase_times(self):
        """Device ms of the last factor/solve phases (see bdlu_phase_times)."""
        out = np.zeros(5)
        self._lib.bdlu_phase_times(self._h, _p64(out), 5)
        return dict(zip(self.PHASES, out.tolist()))

    def canonical_pattern(self):
        nnz = self._lib.bdlu_canonical_pattern(self._h, None, None)
        r = np.empty(nnz, np.int32)
        c = np.empty(nnz, np.int32)
        self._lib.bdlu_canonical_pattern(self._h, _p32(r), _p32(c))
        return r, c

    def decomposition(self):
        """P, Q, merged R, off-diagonal CSR (ptr, col, canonical source) and block levels."""
        st = self.stats()
        n, nb, noff = st["n"], st["nblocks"], st["nnz_offdiag"]
        P, Q = np.empty(n, np.int32), np.empty(n, np.int32)
        R = np.empty(nb + 1, np.int32)
        optr = np.empty(n + 1, np.int32)
        ocol, osrc = np.empty(noff, np.int32), np.empty(noff, np.int32)
        lev = np.empty(nb, np.int32)
        rc = self._lib.bdlu_get_decomposition(self._h, _p32(P), _p32(Q), _p32(R), _p32(optr), _p32(ocol), _p32(osrc), _p32(lev))
        if rc != 0:
            raise RuntimeError("decomposition unavailable (analyze first)")
        return dict(P=P, Q=Q, R=R, off_ptr=optr, off_col=ocol, off_src=osrc, level=lev)

    def signatures(self):
        """(sig, sig2, value_sig) of the canonical matrix after analyze."""
        out = (ctypes.c_uint64 * 3)()
        if self._lib.bdlu_matrix_signatures(self._h, out) != 0:
            return None
        return tuple(int(v) for v in out)

    def unit_routes(self, with_nnz=False):
        """Per unit (raw BTF block): (start rows, routes, reasons[, factor
        entries]) as bdlu_get_unit_routes gives them (route 3 = sparse LU)."""
        nu = self._lib.bdlu_get_unit_routes(self._h, None, None, None, None, 0)
        if nu < 0:
            raise RuntimeError(self.last_error_message() or "unit routes unavailable")
        start, route, reason = (np.zeros(nu, np.int32) for _ in range(3))
        nnz = np.zeros(nu, np.int64)
        self._lib.bdlu_get_unit_routes(self._h, _p32(start), _p32(route), _p32(reason),
                                       nnz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), nu)
        return (start, route, reason, nnz) if with_nnz else (start, route, reason)

    def block_lu(self, b):
        """Dense LU (row-major m*m) and pivots of merged block b, as the reference's micro-kernel stores them."""
        m = self._lib.bdlu_get_block_lu(self._h, int(b), None, None)
        if m < 0:
            raise RuntimeError("block LU unavailable: %d" % m)
        lu = np.empty(m * m, np.float64)
        piv = np.empty(m, np.int32)
        self._lib.bdlu_get_block_lu(self._h, int(b), _p64(lu), _p32(piv))
        return lu.reshape(m, m), piv

    def _export(self, fn):
        cnt = fn(self._h, None, None, None, 0)
        if cnt < 0:
            return []
        r = np.empty(cnt, np.int32)
        c = np.empty(cnt, np.int32)
        v = np.empty(cnt, np.float64)
        fn(self._h, _p32(r), _p32(c), _p64(v), cnt)
        return list(zip(r.tolist(), c.tolist(), v.tolist()))


class Batch:
    """Independent systems factored and solved together (bdlu_batch_*).

    The reference handles one system per Solver; a Batch stands in for a loop
    of Solvers.  Systems are added (storage only), analysed together as one
    block-diagonal system, then factored and solved by shared launches.
    Right-hand sides stack the systems' rows (system k at row_offset(k));
    value-only refactors stack the systems' canonical values (nnz_offset(k)).
    """

    def __init__(self):
        self._lib = load_library()
        self._b = self._lib.bdlu_batch_create()
        if not self._b:
            raise MemoryError("bdlu_batch_create failed")
        self._keep = []

    def __del__(self):
        b, self._b = getattr(self, "_b", None), None
        if b and getattr(self, "_lib", None) is not None:
            self._lib.bdlu_batch_destroy(b)

    def add(self, coo, n):
        """Adds a system (COO, dimension n > 0); returns its index, or -1."""
        r, c, v = _coo_arrays(coo)
        self._keep.append((r, c, v))
        k = self._lib.bdlu_batch_add(self._b, _p32(r), _p32(c), _p64(v), len(r), int(n))
        return k if k >= 0 else -1

    def analyze(self):
        return self._lib.bdlu_batch_analyze(self._b) == 0

    def factor(self):
        return self._lib.bdlu_batch_factor(self._b) == 0

    def refactor_values(self, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        return self._lib.bdlu_batch_refactor_values(self._b, _p64(v), len(v)) == 0

    def refactor_values_device(self, dptr, nnz, stream=0):
        return self._lib.bdlu_batch_refactor_values_device(self._b, ctypes.c_void_p(dptr), nnz,
                                                            ctypes.c_void_p(stream)) == 0

    def solve_in_place(self, B):
        """B: float64 (N,) or Fortran-ordered (N, nrhs), N = row_offset(count)."""
        if not isinstance(B, np.ndarray) or B.dtype != np.float64:
            raise TypeError("solve_in_place expects a float64 numpy array")
        if B.ndim == 1:
            ldb, nrhs = B.shape[0], 1
        else:
            if not B.flags.f_contiguous:
                raise ValueError("multi-RHS B must be Fortran-ordered (column-major)")
            ldb, nrhs = B.shape
        if ldb != self.rows():
            ldb = -1
        return self._lib.bdlu_batch_solve(self._b, _p64(B), ldb, nrhs) == 0

    def solve_device(self, dptr, ldb, nrhs, stream=0):
        return self._lib.bdlu_batch_solve_device(self._b, ctypes.c_void_p(dptr), ldb, nrhs,
                                                  ctypes.c_void_p(stream)) == 0

    def count(self):
        return self._lib.bdlu_batch_count(self._b)

    def row_offset(self, k):
        return self._lib.bdlu_batch_row_offset(self._b, int(k))

    def nnz_offset(self, k):
        return self._lib.bdlu_batch_nnz_offset(self._b, int(k))

    def rows(self):
        return self.row_offset(self.count())

    def last_error(self):
        return SolverError(self._lib.bdlu_batch_last_error(self._b, None, 0))

    def last_error_message(self):
        buf = ctypes.create_string_buffer(1024)
        self._lib.bdlu_batch_last_error(self._b, buf, len(buf))
        return buf.value.decode()

    def stats(self):
        st = Stats()
        self._lib.bdlu_batch_get_stats(self._b, ctypes.byref(st))
        return st.as_dict()

    def phase_times(self):
        out = np.zeros(5)
        self._lib.bdlu_batch_phase_times(self._b, _p64(out), 5)
        return dict(zip(Solver.PHASES, out.tolist()))


class Server:
    """Refactor + solve requests over resident patterns (bdlu_server_*).

    add_pattern analyses a pattern on the host; submit queues a request (new
    values in the pattern's canonical order, right-hand sides overwritten with
    the solution) and returns its id; wait blocks for it.  Requests for
    different patterns run concurrently on the device (continuous batching
    over `slots` streams); a device-memory budget bounds the resident
    patterns.  The arrays given to submit are kept alive until wait returns.
    """

    def __init__(self, memory_budget_bytes, slots=8):
        self._lib = load_library()
        self._s = self._lib.bdlu_server_create(int(memory_budget_bytes), int(slots))
        if not self._s:
            raise ValueError("bdlu_server_create failed (budget and slots must be positive)")
        self._keep = {}

    def close(self):
        s, self._s = getattr(self, "_s", None), None
        if s and getattr(self, "_lib", None) is not None:
            self._lib.bdlu_server_destroy(s)
        self._keep = {}

    def __del__(self):
        self.close()

    def add_pattern(self, coo, n=-1):
        """Returns the pattern id, or -1 (see last_error)."""
        r, c, v = _coo_arrays(coo)
        k = self._lib.bdlu_server_add_pattern(self._s, _p32(r), _p32(c), _p64(v), len(r), int(n))
        return k if k >= 0 else -1

    def pattern_nnz(self, pattern):
        return self._lib.bdlu_server_pattern_nnz(self._s, int(pattern))

    def pattern_bytes(self, pattern):
        return self._lib.bdlu_server_pattern_bytes(self._s, int(pattern))

    def submit(self, pattern, vals, B):
        """vals: float64 (pattern_nnz,); B: float64 (n,) or Fortran (n, nrhs), overwritten.  Returns id or -1."""
        v = np.ascontiguousarray(vals, dtype=np.float64)
        if not isinstance(B, np.ndarray) or B.dtype != np.float64:
            raise TypeError("B must be a float64 numpy array")
        if B.ndim == 1:
            ldb, nrhs = B.shape[0], 1
        else:
            if not B.flags.f_contiguous:
                raise ValueError("multi-RHS B must be Fortran-ordered (column-major)")
            ldb, nrhs = B.shape
        rid = self._lib.bdlu_server_submit(self._s, int(pattern), _p64(v), len(v), _p64(B), ldb, nrhs)
        if rid < 0:
            return -1
        self._keep[rid] = (v, B)
        return rid

    def submit_device(self, pattern, d_vals, nnz, d_B, ldb, nrhs, keep=None):
        """Device-resident request: d_vals / d_B are device pointers (ints);
        X overwrites d_B.  `keep` holds the owning objects until wait.
        Returns id or -1."""
        rid = self._lib.bdlu_server_submit_device(self._s, int(pattern), int(d_vals), int(nnz), int(d_B), int(ldb),
                                                  int(nrhs))
        if rid < 0:
            return -1
        self._keep[rid] = keep
        return rid

    def wait(self, rid):
        """Returns (ok, residual, latency_ms)."""
        res = np.zeros(1)
        lat = np.zeros(1)
        st = self._lib.bdlu_server_wait(self._s, int(rid), _p64(res), _p64(lat))
        self._keep.pop(rid, None)
        return st == 0, float(res[0]), float(lat[0])

    def drain(self):
        return self._lib.bdlu_server_drain(self._s) == 0

    def stats(self):
        st = ServerStats()
        self._lib.bdlu_server_get_stats(self._s, ctypes.byref(st))
        return st.as_dict()

    def set_option(self, key, value):
        """Server-wide option for every pattern ("precision": 0, 1 or 2)."""
        return self._lib.bdlu_server_set_option(self._s, key.encode(), float(value)) == 0

    def reset_stats(self):
        self._lib.bdlu_server_reset_stats(self._s)

    def last_error(self):
        return SolverError(self._lib.bdlu_server_last_error(self._s, None, 0))

    def last_error_message(self):
        buf = ctypes.create_string_buffer(1024)
        self._lib.bdlu_server_last_error(self._s, buf, len(buf))
        return buf.value.decode()


def tuner_report():
    """The autotuner's choices on this GPU (dict; see include/bdlu.h)."""
    import json
    lib = load_library()
    need = lib.bdlu_tuner_report(None, 0)
    buf = ctypes.create_string_buffer(max(1, int(need)))
    lib.bdlu_tuner_report(buf, len(buf))
    return json.loads(buf.value.decode())


def btf_order(n, col_ptr, row_ind):
    """SuiteSparse btf_order calling convention: (nblocks, P, Q, R, nmatch)."""
    lib = load_library()
    ap = np.ascontiguousarray(col_ptr, np.int32)
    ai = np.ascontiguousarray(row_ind, np.int32)
    P, Q, R = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n + 1, np.int32)
    nm = np.zeros(1, np.int32)
    nb = lib.bdlu_btf_order(n, _p32(ap), _p32(ai), _p32(P), _p32(Q), _p32(R), _p32(nm))
    return nb, P, Q, R[: nb + 1].copy(), int(nm[0])


def merge_block_boundaries(R, n, merge_max=64):
    lib = load_library()
    r = np.ascontiguousarray(R, np.int32)
    out = np.empty(len(r), np.int32)
    k = lib.bdlu_merge_block_boundaries(_p32(r), len(r), int(n), int(merge_max), _p32(out))
    return out[:k].copy()


FAMILY_BLOCK, FAMILY_CIRCUIT, FAMILY_PRECISION = 0, 1, 3


class Synth:
    """Seeded synthetic system (canonical COO, x_true, b)."""

    def __init__(self, family, seed, n, param=0, nrhs=1):
        self._lib = load_library()
        self._s = self._lib.bdlu_synth_create(family, seed, n, param, nrhs)
        if not self._s:
            raise ValueError("unknown synthetic family %r" % family)
        self.n = self._lib.bdlu_synth_n(self._s)
        self.nnz = self._lib.bdlu_synth_nnz(self._s)
        self.nrhs = self._lib.bdlu_synth_nrhs(self._s)
        self.rows = np.empty(self.nnz, np.int32)
        self.cols = np.empty(self.nnz, np.int32)
        self.vals = np.empty(self.nnz, np.float64)
        self.x_true = np.empty((self.n, self.nrhs), np.float64, order="F")
        self.b = np.empty((self.n, self.nrhs), np.float64, order="F")
        self._lib.bdlu_synth_copy(self._s, _p32(self.rows), _p32(self.cols), _p64(self.vals), _p64(self.x_true), _p64(self.b))
        nb = self._lib.bdlu_synth_nblocks(self._s)
        self.block_sizes = np.empty(nb, np.int32)
        self._lib.bdlu_synth_block_sizes(self._s, _p32(self.block_sizes))

    def perturbed(self, seed):
        out = np.empty(self.nnz, np.float64)
        self._lib.bdlu_synth_perturb(self._s, seed, _p64(out))
        return out

    def __del__(self):
        s, self._s = getattr(self, "_s", None), None
        if s and getattr(self, "_lib", None) is not None:
            self._lib.bdlu_synth_destroy(s)


def config_seed(config, instance=0):
    """Seeds of the synthetic configurations: 20261203 + 1000*config + instance."""
    return 20261203 + 1000 * config + instance
