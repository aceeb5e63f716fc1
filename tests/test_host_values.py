"""A refactor uploads the new values without keeping a host copy; the host
copy is refreshed from the device when something reads it.  Exports,
factor() and solves must therefore see the values of the last refactor,
through both the host-buffer and the device-pointer refactor.
"""
import numpy as np
import pytest

import blockdaglu as bd

RESID_TOL = 1e-12


def _mul(g, vals, x):
    ax = np.zeros(g.n)
    np.add.at(ax, g.rows, vals * x[g.cols])
    return ax


def _resid(g, vals, x, b):
    ax = _mul(g, vals, x)
    a_inf = np.zeros(g.n)
    np.add.at(a_inf, g.rows, np.abs(vals))
    return np.max(np.abs(ax - b)) / (a_inf.max() * np.max(np.abs(x)) + np.max(np.abs(b)))


def _exported_values(s):
    return np.array([t[2] for t in s.get_rearranged_matrix()])


@pytest.mark.gpu
def test_exports_and_factor_follow_refactored_values(cuda_device, monkeypatch):
    import torch
    for k in ("BLOCKDAGLU_MODE", "USERALGO_MODE", "BLOCKDAGLU_REFINE_ITERS", "USERALGO_REFINE_ITERS"):
        monkeypatch.delenv(k, raising=False)
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 41), 3000, 6)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    assert np.array_equal(_exported_values(s), g.vals)
    # Host-buffer refactor.
    v2 = g.perturbed(7)
    assert s.refactor_values(v2), s.last_error_message()
    assert np.array_equal(_exported_values(s), v2)
    # Device-pointer refactor.
    v3 = g.perturbed(8)
    d = torch.from_numpy(v3).to("cuda")
    torch.cuda.synchronize()
    assert s.refactor_values_device(d.data_ptr(), g.nnz), s.last_error_message()
    torch.cuda.synchronize()
    assert np.array_equal(_exported_values(s), v3)
    b = _mul(g, v3, g.x_true[:, 0])
    x = b.copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert _resid(g, v3, x, b) <= RESID_TOL
    # factor() after refactors factors the refactored values.
    v4 = g.perturbed(9)
    assert s.refactor_values(v4), s.last_error_message()
    assert s.factor(), s.last_error_message()
    b = _mul(g, v4, g.x_true[:, 0])
    x = b.copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert _resid(g, v4, x, b) <= RESID_TOL
    assert np.array_equal(_exported_values(s), v4)


@pytest.mark.gpu
def test_non_finite_refactor_values_are_rejected(cuda_device, monkeypatch):
    # The values are checked while they travel to a staging buffer; a NaN or
    # an infinity anywhere (here near the end) is refused before the
    # engine's values change.
    for k in ("BLOCKDAGLU_MODE", "USERALGO_MODE", "BLOCKDAGLU_REFINE_ITERS", "USERALGO_REFINE_ITERS"):
        monkeypatch.delenv(k, raising=False)
    g = bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(1, 42), 200000)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    for bad in (np.nan, np.inf):
        v = g.perturbed(3)
        v[len(v) - 5] = bad
        assert not s.refactor_values(v)
        assert s.last_error() == bd.SolverError.NonFiniteValue
        x = g.b[:, 0].copy()
        assert s.solve_in_place(x), s.last_error_message()
        assert _resid(g, g.vals, x, g.b[:, 0]) <= RESID_TOL
    v = g.perturbed(4)
    assert s.refactor_values(v), s.last_error_message()
    b = _mul(g, v, g.x_true[:, 0])
    x = b.copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert _resid(g, v, x, b) <= RESID_TOL
