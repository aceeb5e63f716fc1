"""Serving loop (bdlu_server_*): refactor + solve requests over resident
patterns with continuous batching under a device-memory budget.

A request runs exactly the host refactor + solve of bdlu_refactor_solve on
its pattern's engine, so its result may not depend on what else is being
served: the same request stream is served by one slot (each request alone on
the device) and by four slots (requests for different patterns overlapping),
and every solution must agree within the residual bound used everywhere
(relative residual <= 1e-12; the two solutions themselves agree to 1e-12
relative, they are in fact computed by the same kernels in the same order).
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


def test_server_rejects_bad_input():
    with pytest.raises(ValueError):
        bd.Server(0, 2)
    s = bd.Server(1 << 30, 2)
    assert s.add_pattern(([0, 1, 5], [0, 1, 1], [1.0, 2.0, 3.0]), 2) == -1
    assert s.last_error() == bd.SolverError.InvalidIndex
    g = bd.Synth(bd.FAMILY_BLOCK, 5, 400)
    k = s.add_pattern((g.rows, g.cols, g.vals), g.n)
    assert k == 0 and s.pattern_nnz(k) == g.nnz
    assert s.submit(k, np.ones(3), np.ones(g.n)) == -1
    assert s.last_error() == bd.SolverError.InvalidIndex
    assert s.submit(k, g.vals, np.ones(g.n - 1)) == -1
    assert s.last_error() == bd.SolverError.InvalidRightHandSide
    assert s.submit(7, g.vals, np.ones(g.n)) == -1
    s.close()


def _patterns(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(3000), np.log(20000))))
        out.append(bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(4, i), n))
    return out


def _stream(patterns, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for r in range(count):
        k = int(rng.integers(len(patterns)))
        g = patterns[k]
        nrhs = int(rng.integers(1, 5))
        vals = g.perturbed(10_000 + r)
        B = np.asfortranarray(rng.uniform(-1.0, 1.0, (g.n, nrhs)))
        reqs.append((k, vals, B))
    return reqs


def _serve(patterns, reqs, slots, budget=64 << 30):
    s = bd.Server(budget, slots)
    ids = [s.add_pattern((g.rows, g.cols, g.vals), g.n) for g in patterns]
    assert ids == list(range(len(patterns))), s.last_error_message()
    outs = [B.copy(order="F") for _, _, B in reqs]
    rids = [s.submit(k, v, X) for (k, v, _), X in zip(reqs, outs)]
    assert all(r >= 0 for r in rids), s.last_error_message()
    res = [s.wait(r) for r in rids]
    st = s.stats()
    s.close()
    return outs, res, st


@pytest.mark.gpu
def test_server_results_same_alone_and_in_mix(cuda_device):
    patterns = _patterns(4, 1)
    reqs = _stream(patterns, 24, 2)
    alone, res1, st1 = _serve(patterns, reqs, slots=1)
    mixed, res4, st4 = _serve(patterns, reqs, slots=4)
    assert st1["peak_concurrency"] == 1 and st4["peak_concurrency"] >= 2
    assert st1["completed"] == st4["completed"] == len(reqs)
    for (k, v, B), xa, xm, ra, rm in zip(reqs, alone, mixed, res1, res4):
        assert ra[0] and rm[0]
        g = patterns[k]
        for j in range(B.shape[1]):
            assert _relres(g, v, xm[:, j], B[:, j]) <= 1e-12
            assert _relres(g, v, xa[:, j], B[:, j]) <= 1e-12
        assert np.allclose(xm, xa, rtol=1e-12, atol=0.0)
    assert st4["p99_ms"] >= st4["p50_ms"] > 0.0


@pytest.mark.gpu
def test_server_budget_releases_idle_patterns(cuda_device):
    patterns = _patterns(4, 3)
    reqs = _stream(patterns, 12, 4)
    probe = bd.Server(1 << 40, 1)
    sizes = [probe.pattern_bytes(probe.add_pattern((g.rows, g.cols, g.vals), g.n)) for g in patterns]
    probe.close()
    # Room for the largest pattern and a little more, not for all four:
    # idle patterns are released and uploaded again (their next factor then
    # pivots in full) and the results stay correct.
    budget = int(max(sizes) * 1.5)
    assert budget < sum(sizes)
    outs, res, st = _serve(patterns, reqs, slots=2, budget=budget)
    assert st["completed"] == len(reqs) and st["evictions"] > 0
    for (k, v, B), X, r in zip(reqs, outs, res):
        assert r[0]
        for j in range(B.shape[1]):
            assert _relres(patterns[k], v, X[:, j], B[:, j]) <= 1e-12


@pytest.mark.gpu
def test_server_pattern_above_budget_fails(cuda_device):
    g = bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(4, 9), 20000)
    s = bd.Server(1 << 20, 2)
    k = s.add_pattern((g.rows, g.cols, g.vals), g.n)
    X = np.ones(g.n)
    rid = s.submit(k, g.vals, X)
    ok, _, _ = s.wait(rid)
    assert not ok and s.last_error() == bd.SolverError.BackendUnavailable
    s.close()


@pytest.mark.gpu
def test_server_device_resident_requests_match_host_requests(cuda_device):
    """Requests whose values and right-hand sides already live in device
    memory (bdlu_server_submit_device) run the same kernels as host-buffer
    requests: the same stream gives the same solutions, alone and mixed with
    host requests, and the mixed-precision server option keeps the bound."""
    import torch
    patterns = _patterns(3, 5)
    reqs = _stream(patterns, 12, 6)
    host, _, _ = _serve(patterns, reqs, slots=1)
    for prec in (0, 1):
        s = bd.Server(64 << 30, 4)
        assert s.set_option("precision", prec)
        for g in patterns:
            s.add_pattern((g.rows, g.cols, g.vals), g.n)
        dv = [torch.from_numpy(v).cuda() for _, v, _ in reqs]
        dB = [torch.from_numpy(np.ascontiguousarray(B.T)).cuda() for _, _, B in reqs]  # (nrhs, n): column-major
        torch.cuda.synchronize()
        rids = []
        for i, ((k, v, B), a, b) in enumerate(zip(reqs, dv, dB)):
            if i % 3 == 2:   # every third request from host buffers
                X = B.copy(order="F")
                rids.append((s.submit(k, v, X), X))
            else:
                rids.append((s.submit_device(k, a.data_ptr(), len(v), b.data_ptr(), B.shape[0], B.shape[1],
                                             keep=(a, b)), b))
        assert all(r >= 0 for r, _ in rids), s.last_error_message()
        for (k, v, B), (rid, out), xh in zip(reqs, rids, host):
            ok, resid, _ = s.wait(rid)
            assert ok and resid <= 1e-12, s.last_error_message()
            X = out if isinstance(out, np.ndarray) else out.cpu().numpy().T
            for j in range(B.shape[1]):
                assert _relres(patterns[k], v, X[:, j], B[:, j]) <= 1e-12
            if prec == 0:
                assert np.allclose(X, xh, rtol=1e-12, atol=0.0)
        s.close()


@pytest.mark.gpu
def test_server_mixed_route_on_large_units(cuda_device):
    """The server's mixed route from 3xTF32 (option "precision" 2) on a
    pattern whose units are all above the shared-memory limit (tensor-core
    trailing updates): every request meets the residual bound, the residual
    it reports is the one of the returned solution, and the solution agrees
    with a plain FP64 Solver's (the refinement bound, 1e-12 relative residual,
    leaves a forward error up to cond * 1e-12: relative 1e-6 here)."""
    g = bd.Synth(bd.FAMILY_BLOCK, bd.config_seed(0, 31), 3000, 6)
    rng = np.random.default_rng(12)
    reqs = [(0, g.perturbed(20_000 + r), np.asfortranarray(rng.uniform(-1.0, 1.0, (g.n, 1 + r % 3))))
            for r in range(6)]
    s = bd.Server(64 << 30, 2)
    assert s.set_option("precision", 2)
    assert s.add_pattern((g.rows, g.cols, g.vals), g.n) == 0, s.last_error_message()
    outs = [B.copy(order="F") for _, _, B in reqs]
    rids = [s.submit(k, v, X) for (k, v, _), X in zip(reqs, outs)]
    res = [s.wait(r) for r in rids]
    s.close()
    ref = bd.Solver()
    assert ref.set_matrix((g.rows, g.cols, g.vals), g.n) and ref.analyze() and ref.factor(), ref.last_error_message()
    assert ref.stats()["max_unit"] > 169
    for (k, v, B), X, (ok, resid, _) in zip(reqs, outs, res):
        assert ok
        host = max(_relres(g, v, X[:, j], B[:, j]) for j in range(B.shape[1]))
        assert host <= 1e-12 and 0.0 < resid <= 1e-12, (host, resid)
        assert resid == pytest.approx(host, rel=0.5), (host, resid)
        assert ref.refactor_values(v), ref.last_error_message()
        Xr = B.copy(order="F")
        assert ref.solve_in_place(Xr), ref.last_error_message()
        assert np.allclose(X, Xr, rtol=1e-6, atol=1e-6 * np.max(np.abs(Xr)))


@pytest.mark.gpu
def test_server_rejects_non_finite_inputs(cuda_device):
    """NaN or infinity in a request's values or right-hand sides fails that
    request with NonFiniteValue (the check runs while the inputs are staged);
    the pattern keeps serving."""
    g = bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(4, 11), 6000)
    s = bd.Server(8 << 30, 2)
    k = s.add_pattern((g.rows, g.cols, g.vals), g.n)
    v = g.vals.copy()
    v[7] = np.nan
    X = np.ones(g.n)
    ok, _, _ = s.wait(s.submit(k, v, X))
    assert not ok and s.last_error() == bd.SolverError.NonFiniteValue
    X = np.ones(g.n)
    X[3] = np.inf
    ok, _, _ = s.wait(s.submit(k, g.vals, X))
    assert not ok and s.last_error() == bd.SolverError.NonFiniteValue
    B = g.b[:, 0].copy()
    ok, resid, _ = s.wait(s.submit(k, g.vals, B))
    assert ok and resid <= 1e-12
    assert _relres(g, g.vals, B, g.b[:, 0]) <= 1e-12
    s.close()
