"""Mixed-precision route ("precision" = 1): tensor-core TF32 trailing updates
of the large blocks, FP64 refinement to relative residual <= 1e-12, and the
precision ladder TF32 -> 3xTF32 -> FP64 when refinement stagnates.

Every result must meet the same residual bound as the FP64 route, and agree
with the FP64 route's solution to the accuracy the conditioning allows (the
precision systems have block condition numbers near kappa from a row ramp;
the check is ||x_mixed - x_fp64||_inf <= 1e-8 ||x_fp64||_inf for kappa 1e4).
"""
import numpy as np
import pytest

import blockdaglu as bd


def _relres(g, vals, x, b):
    r = b.copy()
    np.subtract.at(r, g.rows, vals * x[g.cols])
    arow = np.zeros(g.n)
    np.add.at(arow, g.rows, np.abs(vals))
    return np.max(np.abs(r)) / (arow.max() * np.max(np.abs(x)) + np.max(np.abs(b)))


def _solver(g, mixed):
    s = bd.Solver()
    assert s.set_option("precision", 1 if mixed else 0)
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    return s


def test_precision_option_values():
    s = bd.Solver()
    assert s.set_option("precision", 0) and s.set_option("precision", 1) and s.set_option("precision", 2)
    assert not s.set_option("precision", 3)


@pytest.mark.gpu
@pytest.mark.parametrize("level,tol,agree", [(2, 1e-5, 1000), (1, 3e-2, 100)])
def test_tensor_core_update_matches_fp64_factors(cuda_device, monkeypatch, level, tol, agree):
    """The tcgen05 trailing update against the FP64 update on the same unit:
    MODE=klu makes one 1,200-row unit whose first factor runs 37 panel steps
    of tensor-core updates.  Where both factorisations chose the same pivots
    (a diagonally weighted block: nearly all of them), the factors agree to
    the accuracy of the tensor-core arithmetic: 3xTF32 (level 2) to about
    FP32 rounding, TF32 (level 1) to about TF32 rounding.  A wrong operand
    layout or descriptor would put O(1) errors into every updated entry."""
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 35), 1200, 24)
    lus = []
    for prec in (0, level):
        s = bd.Solver()
        assert s.set_option("precision", prec)
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
        assert s.stats()["max_unit"] == 1200
        lus.append(s.block_lu(0))
    (lu64, piv64), (lumx, pivmx) = lus
    same = np.flatnonzero(np.cumprod(piv64 == pivmx))  # columns before the first pivot difference
    assert len(same) > agree, len(same)
    k = len(same)
    scale = np.max(np.abs(lu64))
    assert np.max(np.abs(lu64[:k, :k] - lumx[:k, :k])) <= tol * scale


@pytest.mark.gpu
@pytest.mark.parametrize("kappa_exp", [4, 8])
def test_mixed_reaches_fp64_bound(cuda_device, kappa_exp):
    g = bd.Synth(bd.FAMILY_PRECISION, bd.config_seed(3, kappa_exp), 2, kappa_exp)
    rng = np.random.default_rng(kappa_exp)
    B = np.asfortranarray(rng.uniform(-1.0, 1.0, (g.n, 4)))
    ref = _solver(g, False)
    X64 = B.copy(order="F")
    assert ref.solve_in_place(X64), ref.last_error_message()
    mix = _solver(g, True)
    X = B.copy(order="F")
    assert mix.solve_in_place(X), mix.last_error_message()
    st = mix.stats()
    assert st["residual_inf"] <= 1e-12
    for j in range(B.shape[1]):
        assert _relres(g, g.vals, X[:, j], B[:, j]) <= 1e-12
    if kappa_exp == 4:
        assert st["precision"] in (1, 2) and st["refine_iters"] > 0, st
        assert np.max(np.abs(X - X64)) <= 1e-8 * np.max(np.abs(X64))
    # Value-only refactor keeps the level reached.
    lvl = st["precision"]
    v = g.perturbed(77)
    assert mix.refactor_values(v)
    X2 = B.copy(order="F")
    assert mix.solve_in_place(X2), mix.last_error_message()
    st2 = mix.stats()
    assert st2["precision"] == lvl or st2["precision"] in (0, 2)
    for j in range(B.shape[1]):
        assert _relres(g, v, X2[:, j], B[:, j]) <= 1e-12


@pytest.mark.gpu
def test_mixed_ladder_on_ill_conditioned_circuit(cuda_device):
    # The circuit systems are very ill-conditioned (forward error 1e-3 at an
    # FP64 residual of 1e-16): TF32 and 3xTF32 refinement stagnate and the
    # ladder must end at FP64 with the residual bound met.
    g = bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(1, 7), 20000)
    s = _solver(g, True)
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x), s.last_error_message()
    st = s.stats()
    assert st["residual_inf"] <= 1e-12
    assert _relres(g, g.vals, x, g.b[:, 0]) <= 1e-12
