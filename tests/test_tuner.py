"""The autotuner (include/bdlu.h, csrc/tuner.cpp): launch widths of the
shared-memory LU per size bucket and the refactor schedule of large units per
pattern, timed on the GPU and kept in a per-GPU JSON cache.  Every candidate
computes bit-identical results, so the parity tests (which run with tuning
on) already cover correctness; here the choices themselves are checked."""
import json
import os

import numpy as np
import pytest

import blockdaglu as bd
import oracle

pytestmark = pytest.mark.gpu


def test_tuner_picks_lu_small_widths(cuda_device, monkeypatch):
    monkeypatch.delenv("BLOCKDAGLU_MODE", raising=False)
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 50), 2000)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    rep = bd.tuner_report()
    if not rep["enabled"]:
        pytest.skip("BDLU_AUTOTUNE=0")
    widths = {e["bucket_m"]: e for e in rep["lu_small_threads"]}
    assert widths, rep
    for m, e in widths.items():
        # 1: one thread per row (units up to 96 rows); 32: one warp per unit
        # (up to 64 rows); else threads per CTA, at least one per row.
        assert (e["threads"] == 1 and m <= 96) or (e["threads"] == 32 and m <= 64) or \
            (e["threads"] in (64, 128, 256) and e["threads"] >= m)
        if "ms" in e:
            assert len(e["ms"]) == len(e["widths"]) and min(e["ms"]) > 0.0
            assert e["ms"][e["widths"].index(e["threads"])] == min(e["ms"])
    # The choice persists in the cache file.
    with open(rep["cache"]) as f:
        saved = json.load(f)
    assert {e["bucket_m"]: e["threads"] for e in saved["lu_small_threads"]} == \
        {m: e["threads"] for m, e in widths.items()}


def test_tuner_picks_refactor_schedule_per_pattern(cuda_device, monkeypatch):
    # One 2,000-row large unit: its value-only refactors run the step chain
    # and the tile task graph in turn (6 trials: a capture trial and two
    # timed trials each), then the faster stays.
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 51), 2000, 40)
    s = bd.Solver()
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    xs = []
    for k in range(6):
        v = g.perturbed(700 + (k % 2))
        assert s.refactor_values(v), s.last_error_message()
        x = g.b[:, 0].copy()
        assert s.solve_in_place(x), s.last_error_message()
        xs.append(x)
    # Same values, either schedule: bit-identical solutions.
    assert np.array_equal(xs[0], xs[2]) and np.array_equal(xs[1], xs[3]) and np.array_equal(xs[0], xs[4])
    rep = bd.tuner_report()
    if not rep["enabled"]:
        pytest.skip("BDLU_AUTOTUNE=0")
    sig = s.signatures()[0]
    entry = [e for e in rep["refactor_schedule"] if int(e["sig"], 16) == sig]
    assert len(entry) == 1, rep
    e = entry[0]
    assert e["schedule"] in (0, 1) and e["ms_chain"] > 0.0 and e["ms_graph"] > 0.0
    assert e["schedule"] == (1 if e["ms_graph"] < 0.98 * e["ms_chain"] else 0)
    assert os.path.exists(rep["cache"])


@pytest.mark.parametrize("width", [1, 32, 64, 128, 256])
def test_every_lu_width_bit_identical_to_oracle(cuda_device, monkeypatch, width):
    """Each launch width of the small-unit LU (1: one thread per row, rows in
    registers; 32: one warp per unit, rows in registers; 64 / 128 / 256
    threads per unit, unit in shared memory) gives the reference
    micro-kernel's factors and pivots bit for bit on every block of the
    2,000-row block system (units of 10-90 rows; a bucket a width cannot take
    runs the tuned width)."""
    monkeypatch.delenv("BLOCKDAGLU_MODE", raising=False)
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0), 2000)
    s = bd.Solver()
    assert s.set_option("lu_small_threads", width)
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
    d = s.decomposition()
    ref = oracle.System(g.n, g.rows, g.cols, g.vals, d["P"], d["Q"], d["R"])
    assert ref.factor()
    R = d["R"]
    for b in range(len(R) - 1):
        lu, piv = s.block_lu(b)
        lu_ref, piv_ref = ref.block_lu(b)
        assert np.array_equal(piv, piv_ref) and np.array_equal(lu, lu_ref), (width, b, R[b + 1] - R[b])
    x = g.b[:, 0].copy()
    assert s.solve_in_place(x), s.last_error_message()
    assert np.allclose(x, ref.solve(g.b[:, 0]), rtol=1e-9, atol=0.0)


@pytest.mark.parametrize("family,n", [(bd.FAMILY_BLOCK, 2000), (bd.FAMILY_CIRCUIT, 20000)])
def test_one_launch_queue_bit_identical_to_oracle(cuda_device, monkeypatch, family, n):
    """All small units in one persistent launch over a task queue (whole-CTA
    tasks for units above 32 rows, packs of eight warp tasks below) give the
    same factors as the per-bucket launches and the reference micro-kernel."""
    monkeypatch.delenv("BLOCKDAGLU_MODE", raising=False)
    g = bd.Synth(family, bd.config_seed(0 if family == bd.FAMILY_BLOCK else 1, 52), n)
    sols = []
    for mode in (1, 0):
        s = bd.Solver()
        assert s.set_option("small_launch", mode)
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
        sols.append(s)
    d = sols[0].decomposition()
    ref = oracle.System(g.n, g.rows, g.cols, g.vals, d["P"], d["Q"], d["R"])
    assert ref.factor()
    R = d["R"]
    for b in range(len(R) - 1):
        if R[b + 1] - R[b] > 169:
            continue  # large units: not on this path
        lu_q, piv_q = sols[0].block_lu(b)
        lu_b, piv_b = sols[1].block_lu(b)
        lu_ref, piv_ref = ref.block_lu(b)
        assert np.array_equal(piv_q, piv_ref) and np.array_equal(lu_q, lu_ref), b
        assert np.array_equal(piv_b, piv_ref) and np.array_equal(lu_b, lu_ref), b
    x = g.b[:, 0].copy()
    assert sols[0].solve_in_place(x), sols[0].last_error_message()
