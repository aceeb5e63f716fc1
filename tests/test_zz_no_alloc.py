"""The no-allocation dense batch solve (bdlu_dense_batch_solve_noalloc)
against the handle-based entry point on the same systems.

That entry point serves callers that cannot allocate device memory where they
solve; its scratch lives in a static device array inside the library, so this
file runs last (pytest collects it after every other test file) and must pass
both on its own in a fresh process and after the other tests.  Tolerance: the
reference's close(), relative 1e-9 (blockdaglu/apps/tests/main.cpp:71-73).
"""
import ctypes

import numpy as np
import pytest

import blockdaglu as bd

from reference_cases import close_vec

pytestmark = pytest.mark.gpu


def noalloc_fn():
    lib = bd.load_library()
    fn = lib.bdlu_dense_batch_solve_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                   ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64]
    return fn


def random_batch(rng, batch, m, nrhs):
    A = rng.standard_normal((batch, m, m))
    A += np.eye(m)[None] * 0.5 * np.abs(A).sum(axis=2, keepdims=True)
    B = rng.standard_normal((batch, m, nrhs))
    return A, B


def handle_solution(A, B):
    """The same systems through bdlu_set_coo/analyze/factor/solve as one
    block-diagonal matrix."""
    batch, m, _ = A.shape
    nrhs = B.shape[2]
    n = batch * m
    rows, cols, vals = [], [], []
    for i in range(batch):
        r, c = np.nonzero(A[i] != 0.0)
        rows.append(r + i * m)
        cols.append(c + i * m)
        vals.append(A[i][r, c])
    s = bd.Solver()
    assert s.set_matrix((np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)), n)
    assert s.analyze(), s.last_error_message()
    assert s.factor(), s.last_error_message()
    X = np.asfortranarray(np.concatenate([B[i] for i in range(batch)], axis=0))
    assert s.solve_in_place(X), s.last_error_message()
    return np.stack([X[i * m:(i + 1) * m] for i in range(batch)])


def device_call(fn, A, B, torch, in_place=False, fill=None):
    batch, m, _ = A.shape
    nrhs = B.shape[2]
    # Column-major per matrix / per RHS block, matrices contiguous.
    dA = torch.from_numpy(np.ascontiguousarray(A.transpose(0, 2, 1))).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.transpose(0, 2, 1))).cuda()
    dX = dB if in_place else torch.empty_like(dB)
    if fill is not None and not in_place:
        dX.fill_(fill)
    msg = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(dA.data_ptr(), m, batch, dB.data_ptr(), dX.data_ptr(), nrhs, stream, msg, 256)
    return rc, msg.value.decode(), dX.cpu().numpy().transpose(0, 2, 1)


def test_noalloc_matches_handle_path_two_calls(cuda_device):
    import torch
    fn = noalloc_fn()
    rng = np.random.default_rng(2026)
    # Two calls in a row with different shapes: the shared scratch keeps the
    # first call's contents, which must not leak into the second result.
    for batch, m, nrhs, in_place in ((16, 40, 3, False), (7, 25, 2, True)):
        A, B = random_batch(rng, batch, m, nrhs)
        rc, msg, X = device_call(fn, A, B, torch, in_place)
        assert rc == bd.SolverError.None_, msg
        Xh = handle_solution(A, B)
        assert close_vec(X, Xh), (batch, m, nrhs)
        assert close_vec(X, np.linalg.solve(A, B), 1e-9)


def test_noalloc_rejects_sizes_beyond_limit(cuda_device):
    import torch
    fn = noalloc_fn()
    rng = np.random.default_rng(1)
    A, B = random_batch(rng, 1, 129, 1)
    rc, msg, _ = device_call(fn, A, B, torch)
    assert rc == bd.SolverError.InvalidDimension and "128" in msg
    A, B = random_batch(rng, 66, 127, 1)  # 66 * 127^2 = 1064514 > 1048576 factor entries
    rc, msg, _ = device_call(fn, A, B, torch)
    assert rc == bd.SolverError.InvalidDimension and "1048576" in msg


def test_noalloc_at_exact_limits(cuda_device):
    """m = 128 (128 KiB of dynamic shared memory per matrix) with
    batch * m * m exactly 1,048,576; one entry more is refused, and so is
    batch * m above 65,536 while batch * m * m stays within its limit."""
    import torch
    fn = noalloc_fn()
    rng = np.random.default_rng(128)
    A, B = random_batch(rng, 64, 128, 2)
    rc, msg, X = device_call(fn, A, B, torch)
    assert rc == bd.SolverError.None_, msg
    assert close_vec(X, np.linalg.solve(A, B), 1e-9)
    A, B = random_batch(rng, 8193, 8, 1)  # 8193 * 8 = 65544 rows; 524352 factor entries
    rc, msg, _ = device_call(fn, A, B, torch)
    assert rc == bd.SolverError.InvalidDimension and "65536" in msg


def test_noalloc_singular_matrix_reported(cuda_device):
    """A failed matrix is reported, its X block is left unwritten and the
    other matrices of the batch are still solved; a NaN pivot counts as a
    failure."""
    import torch
    fn = noalloc_fn()
    A = np.zeros((3, 4, 4))
    A[0] = np.eye(4) * 2.0
    A[1, :, 0] = 1.0  # rank 1
    A[2] = np.eye(4)
    B = np.ones((3, 4, 2))
    rc, msg, X = device_call(fn, A, B, torch, fill=-7.0)
    assert rc == bd.SolverError.FactorizationFailed and "matrix 1" in msg
    assert np.all(X[1] == -7.0)
    assert np.array_equal(X[0], B[0] / 2.0) and np.array_equal(X[2], B[2])
    rc, msg, X = device_call(fn, A, B, torch, in_place=True)
    assert rc == bd.SolverError.FactorizationFailed
    assert np.array_equal(X[1], B[1])
    A[1] = np.eye(4)
    A[1, 2, 2] = np.nan
    rc, msg, X = device_call(fn, A, B, torch, fill=-7.0)
    assert rc == bd.SolverError.FactorizationFailed and "matrix 1" in msg
    assert np.all(X[1] == -7.0)
