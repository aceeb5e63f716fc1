"""Value-only refactor of large blocks as a tile task graph (one persistent
kernel, option "refactor_schedule" = 1) against the step chain (= 0).

CPU: the task list (plan.cpp build_rtasks) replayed in ticket order by an
independent checker (tests/cpp/rtask_order_test.cpp): every task finds its
input tiles at the versions the kernel waits for, so the kernel's waits only
ever point at smaller tickets; a planted misorder must be caught.
GPU: both schedules run the same per-tile arithmetic, so factors and
solutions are bit-identical (==), on several large blocks at once and on one
block factored across CTAs; residuals stay within 1e-12.
"""
import os
import subprocess

import numpy as np
import pytest

import blockdaglu as bd
from conftest import ROOT
from reference_cases import multiply

LIB = os.path.join(ROOT, "block-daglu_b200", "lib")
SRC = os.path.join(ROOT, "tests", "cpp", "rtask_order_test.cpp")
RESID_TOL = 1e-12


def test_task_order_replays_in_ticket_order(tmp_path):
    exe = str(tmp_path / "rtask_order")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "block-daglu_b200", "csrc"), "-I/usr/local/cuda/include", SRC, "-L" + LIB,
           "-lbdlu", "-Wl,-rpath," + LIB, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0 and lines[-1] == "ok", r.stdout + r.stderr
    assert any(l.startswith("planted misorder: FAIL") for l in lines), r.stdout


def _resid(g, vals, x, b):
    ax = multiply(list(zip(g.rows, g.cols, vals)), g.n, x)
    a_inf = np.zeros(g.n)
    np.add.at(a_inf, g.rows, np.abs(vals))
    return np.max(np.abs(ax - b)) / (a_inf.max() * np.max(np.abs(x)) + np.max(np.abs(b)))


def _two_schedules(g, refactors, compare_u):
    solvers = []
    for sched in (0, 1):
        s = bd.Solver()
        assert s.set_option("refactor_schedule", sched)
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
        solvers.append(s)
    for k in range(refactors):
        v = g.perturbed(500 + k)
        b = multiply(list(zip(g.rows, g.cols, v)), g.n, g.x_true[:, 0])
        xs = []
        for s in solvers:
            assert s.refactor_values(v), s.last_error_message()
            x = b.copy()
            assert s.solve_in_place(x), s.last_error_message()
            assert _resid(g, v, x, b) <= RESID_TOL
            xs.append(x)
        assert np.array_equal(xs[0], xs[1])
    if compare_u:
        assert solvers[0].getU() == solvers[1].getU()
    return solvers


@pytest.mark.gpu
def test_schedules_bit_identical_several_large_blocks(cuda_device, monkeypatch):
    for k in ("BLOCKDAGLU_MODE", "USERALGO_MODE", "BLOCKDAGLU_REFINE_ITERS", "USERALGO_REFINE_ITERS"):
        monkeypatch.delenv(k, raising=False)
    # Six blocks of 274 to 741 rows (5 to 12 tiles per side), coupled.
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 31), 3000, 6)
    assert (g.block_sizes > 169).sum() >= 4
    _two_schedules(g, 3, compare_u=True)


@pytest.mark.gpu
def test_schedules_bit_identical_one_block(cuda_device, monkeypatch):
    monkeypatch.setenv("BLOCKDAGLU_MODE", "klu")
    for k in ("BLOCKDAGLU_REFINE_ITERS", "USERALGO_REFINE_ITERS"):
        monkeypatch.delenv(k, raising=False)
    # One 2001-row block: 32 tiles per side, the last one a single row.
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 32), 2001, 40)
    _two_schedules(g, 2, compare_u=False)


def test_schedule_option_values():
    s = bd.Solver()
    assert s.set_option("refactor_schedule", 0)
    assert s.set_option("refactor_schedule", 1)
    assert not s.set_option("refactor_schedule", 2)
