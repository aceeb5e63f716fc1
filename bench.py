"""Refactor + solve throughput of the B200 engine on the 200k-row circuit system.

Workload ("circuit-200k"): n = 200,000, ~1,000 Pareto(1.5, x_m = 10) diagonal
blocks clipped to [1, 20000] plus 1x1 blocks, 6 stored entries per row on
average, 50 bus rows/columns of 500 entries, log-uniform magnitudes in
[1e-3, 1e3], random P/Q, seed 20262203 (synthetic stand-in, no dataset).
One analyze + first factor (untimed), then steps of one value-only refactor
(values x (1 + U(-0.1, 0.1)), fresh per step) followed by one 1-RHS solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--workload circuit-200k|batch-256|serve-64|precision-200|sparse-units]

Workload "precision-200" (precision): 200 irreducible blocks of U{2000..8000}
rows with ~20 entries per row plus Pareto-sized small blocks (about 10 % of
the rows), a geometric row ramp giving block condition numbers near kappa;
instance a kappa = 1e4, instance b kappa = 1e8; 16 right-hand sides U(-1, 1).
Per instance: one full factorisation with pivoting + 16-rhs solve on the FP64
route and on the mixed route (TF32 tensor-core trailing updates, FP64
refinement to <= 1e-12, precision ladder); reports time, refinement steps,
the level used and the mixed solution's error against the FP64 one.

Workload "serve-64" (serving): 64 patterns of the circuit generator with n
log-uniform in [5,000, 300,000]; requests = value-only refactor (values
x (1 + U(-0.1, 0.1))) + solve of U{1..16} right-hand sides on a uniformly
drawn pattern; a 150 GB device budget.  Reports the served engine's
closed-loop throughput (value), an open-loop Poisson stream at --rate
requests/s for --duration seconds (p50/p99 latency, arrival to result in the
caller's buffer), and the plain FP64 path on the same requests (one request
at a time through bdlu_refactor_solve, one Solver per pattern).

Workload "batch-256" (independent systems): 256 systems of the 2,000-row
block generator's kind with n log-uniform in [1,000, 50,000] and n/50 blocks,
8 right-hand sides U(-1, 1); each step refactors all 256 systems (values
x (1 + U(-0.1, 0.1))) and solves the 8 right-hand sides of each, through one
batch (bdlu_batch_*); the metric is systems factored and solved per second.

Workload "sparse-units" (fill sweep of the sparse-LU route): per class of
extra entries per row (0.1 .. 4), 300 sparse irreducible blocks of U{200..600}
rows (a cyclic chain, the diagonal and the extra entries, magnitudes
U(0.5, 2) with random sign), coupled above the blocks, randomly permuted;
steps of one value-only refactor (values x (1 + U(-0.01, 0.01))) and one
1-rhs solve on the dense route and on the sparse-LU route (option
"sparse_lu" = 2, no fill limit), device-timed; reports the fill of the
sparse factors and the speed-up per class.  Then single blocks of 1,000,
2,000 and 4,000 rows with 0.05 .. 1 extra entries per row on the global
route (one unit in its own order, so the diagonal stays dominant and the
sparse factor is accepted): the per-block crossover of fill and size.

Prints one JSON line on rank 0.  `value` is device-timed (inputs resident in
HBM, CUDA events per step on the launching stream, L2 flushed between steps
outside the timed window); `e2e` runs the same steps through the public C ABI
call bdlu_refactor_solve with host buffers (values and b copied in, x copied
out, every step).  Under torchrun each rank runs an independent replica
(replicas only: one system is solved per GPU, no collective on the data path)
and the slowest rank's time is used.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "block-daglu_b200")]

import numpy as np  # noqa: E402

CIRCUIT_WORKLOAD = "circuit-200k"
METRIC = "refactor+solves/s"
N_ROWS = 200000
CONFIG_INDEX = 1
L2_FLUSH_BYTES = 256 << 20
BATCH_WORKLOAD = "batch-256"
BATCH_METRIC = "system factor+solves/s"
BATCH_SYSTEMS, BATCH_NRHS, BATCH_CONFIG = 256, 8, 2
SERVE_WORKLOAD = "serve-64"
WORKLOAD = SERVE_WORKLOAD  # the default: served vs plain FP64 GPU throughput and latency
SERVE_METRIC = "refactor+solves/s"
SERVE_PATTERNS, SERVE_CONFIG, SERVE_BUDGET = 64, 4, 150 << 30
REF_SERVE_MAX_BLOCK = 4000
PREC_WORKLOAD = "precision-200"
PREC_METRIC = "factor+16-rhs solves/s"
PREC_BLOCKS, PREC_CONFIG, PREC_NRHS = 200, 3, 16
SPARSE_WORKLOAD = "sparse-units"
SPARSE_EXTRAS = (0.1, 0.25, 0.5, 1.0, 2.0, 4.0)
SPARSE_BLOCKS, SPARSE_MIN_ROWS, SPARSE_MAX_ROWS, SPARSE_SEED = 300, 200, 600, 20261277
# Single sparse blocks on the global route (no BTF, so the block keeps its
# own diagonal and the sparse factor is accepted): rows x extra entries/row.
SPARSE_SINGLE = tuple((m, e) for m in (1000, 2000, 4000) for e in (0.05, 0.1, 0.25, 0.5, 1.0))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=[SERVE_WORKLOAD, CIRCUIT_WORKLOAD, BATCH_WORKLOAD, PREC_WORKLOAD, SPARSE_WORKLOAD])
    ap.add_argument("--blocks", type=int, default=PREC_BLOCKS, help="precision-200: number of large blocks")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve-64: Poisson arrival rate (requests/s)")
    ap.add_argument("--sparse-extra", type=float, nargs="*", default=None,
                    help="sparse-units: the classes to run (extra entries per row), default all")
    ap.add_argument("--sparse-single", type=int, default=None, choices=[0, 1],
                    help="sparse-units: 1 only the single-block classes, 0 only the many-block classes")
    ap.add_argument("--duration", type=float, default=2.0, help="serve-64: seconds of open-loop arrivals")
    ap.add_argument("--slots", type=int, default=16, help="serve-64: concurrent request slots")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1, 2],
                    help="serve-64: 0 FP64, 1 mixed (tensor-core updates + FP64 refinement), 2 mixed from 3xTF32")
    ap.add_argument("--refactor-schedule", type=int, default=None, choices=[0, 1],
                    help="circuit-200k: large-block refactor as a step chain (0) or one tile task graph (1); "
                         "default: the autotuner's choice")
    return ap.parse_args()


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(ms, dist, device=None):
    """Replicas: the slowest rank's time (all_reduce MAX); ms unchanged on one process."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def circuit_system():
    import blockdaglu as bd
    return bd.Synth(bd.FAMILY_CIRCUIT, bd.config_seed(CONFIG_INDEX), N_ROWS)


def step_inputs(g, k):
    """Values and b of step k: values x (1 + U(-0.1, 0.1)), b = A_k x_true."""
    v = g.perturbed(1_000_003 + k)
    b = np.zeros(g.n)
    np.add.at(b, g.rows, v * g.x_true[g.cols, 0])
    return v, b


def host_cpu():
    """(usable cores, CPU model) of this host."""
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return cores, model


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def oracle_circuit_system():
    """The circuit-200k system from the oracle's own generator (identical to the
    engine arm's; checked by tests/test_oracle_synth.py)."""
    oracle = oracle_module()
    return oracle.Synth(oracle.FAMILY_CIRCUIT, oracle.config_seed(CONFIG_INDEX), N_ROWS)


def reference_route(g, steps, warm, threads, nrhs_of=None, step_inputs_fn=None):
    """The reference's BLOCK route (its own solver.cpp / ubtf_block_solver.cpp
    built under oracle/_ref, SuiteSparse stand-ins) as a caller of its API runs
    a value change: set_matrix(new values) + analyze + factor +
    solve_in_place, on one Solver.  threads: USERALGO_THREADS (None: the
    reference's own default policy).  Returns per-phase means in seconds."""
    oracle = oracle_module()
    if threads:
        os.environ["USERALGO_THREADS"] = str(threads)
    else:
        os.environ.pop("USERALGO_THREADS", None)
    os.environ["USERALGO_MODE"] = "block"
    os.environ.pop("BLOCKDAGLU_MODE", None)
    s = oracle.RefSolver()
    rec, worst = [], 0.0
    fn = step_inputs_fn or step_inputs
    for k in range(warm + steps):
        v, b = fn(g, k)
        t0 = time.perf_counter()
        ok = s.set_matrix(g.rows, g.cols, v, g.n) and s.analyze()
        t1 = time.perf_counter()
        ok = ok and s.factor()
        t2 = time.perf_counter()
        x = np.ascontiguousarray(b, np.float64).copy()
        ok = ok and s.solve_in_place(x)
        t3 = time.perf_counter()
        if not ok:
            raise RuntimeError("reference route failed: " + s.last_error_message())
        if k >= warm:
            rec.append((t1 - t0, t2 - t1, t3 - t2))
            worst = max(worst, oracle.metrics(g.rows, g.cols, v, x, b)[0])
    os.environ.pop("USERALGO_THREADS", None)
    os.environ.pop("USERALGO_MODE", None)
    mean = [statistics.mean(r[i] for r in rec) for i in range(3)]
    return {"analyze_s": mean[0], "factor_s": mean[1], "solve_s": mean[2], "step_s": sum(mean),
            "factor_solve_s": mean[1] + mean[2], "steps": len(rec), "residual_inf_max": worst,
            "mode": s.selected_mode()}


def port_step(g):
    """The oracle's C restatement (bdlu_oracle.c), one thread: one factor + solve
    of the system under the oracle's own BTF ordering."""
    oracle = oracle_module()
    import scipy.sparse as sp
    v, b = step_inputs(g, 0)
    t0 = time.perf_counter()
    a = sp.csc_matrix((np.ones(g.nnz), (g.rows, g.cols)), shape=(g.n, g.n))
    a.sort_indices()
    nb, P, Q, R, _ = oracle.btf_order(g.n, a.indptr, a.indices)
    Q = np.where(Q < -1, -Q - 2, Q)
    R = oracle.merge_block_boundaries(R, g.n)
    ref = oracle.System(g.n, g.rows, g.cols, v, P, Q, R)
    ok = ref.factor()
    x = ref.solve(b)
    dt = time.perf_counter() - t0
    return dt, oracle.metrics(g.rows, g.cols, v, x, b)[0], ok


def cpu_baseline_reference(g):
    """cpu_baseline of the engine arm: one timed value change of the circuit-200k
    system through the reference's BLOCK route on all host cores, after one
    untimed step."""
    cores, model = host_cpu()
    r = reference_route(g, 1, 1, cores)
    return {"value": 1.0 / r["step_s"], "unit": METRIC, "cores": cores, "kind": "reference",
            "sample": "1 timed value change (set_matrix + analyze + factor + 1-RHS solve, after 1 untimed) of the "
                      "full %s system by the reference's BLOCK route built under oracle/_ref (its own solver.cpp and "
                      "ubtf_block_solver.cpp; KLU and BTF are stand-ins: SuiteSparse is unavailable on this box), "
                      "USERALGO_THREADS=%d on %s: analyze %.2f s, factor %.2f s, solve %.3f s, residual %.1e"
                      % (CIRCUIT_WORKLOAD, cores, model, r["analyze_s"], r["factor_s"], r["solve_s"], r["residual_inf_max"])}


def run_reference(args, rank, world):
    """The reference's CPU route on the circuit-200k workload (rank 0 only):
    all host cores for the line's value, the reference's default thread
    policy and the oracle's one-thread restatement beside it."""
    if rank != 0:
        return
    cores, model = host_cpu()
    g = oracle_circuit_system()
    steps = max(1, min(args.steps, 3))
    warm = 1 if args.warmup > 0 else 0
    allc = reference_route(g, steps, warm, cores)
    dflt = reference_route(g, 1, 0, None)
    port_s, port_res, port_ok = port_step(g)
    t = allc["step_s"]
    line = {"metric": METRIC, "value": 1.0 / t, "unit": METRIC, "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": CIRCUIT_WORKLOAD, "n": g.n, "nnz": int(g.nnz), "nrhs": 1},
            "impl": "reference",
            "same_steps": steps == args.steps and warm == args.warmup,
            "same_steps_reason": None if steps == args.steps else
            "each reference step takes seconds on the host: %d timed steps of --steps %d keep the run within minutes"
            % (steps, args.steps),
            "cpu_baseline": {"value": 1.0 / t, "unit": METRIC, "cores": cores, "kind": "reference",
                             "sample": "%d timed value changes (set_matrix + analyze + factor + 1-RHS solve) of the "
                                       "full system by the reference's BLOCK route built under oracle/_ref (its own "
                                       "solver.cpp and ubtf_block_solver.cpp; KLU and BTF are stand-ins: SuiteSparse "
                                       "is unavailable on this box), USERALGO_THREADS=%d on %s"
                                       % (steps, cores, model)},
            "reference_phases_s": {k: allc[k] for k in ("analyze_s", "factor_s", "solve_s")},
            "reference_factor_solve_only": {"value": 1.0 / allc["factor_solve_s"], "unit": METRIC},
            "reference_default_threads": {"value": 1.0 / dflt["step_s"], "unit": METRIC,
                                          "factor_solve_only": 1.0 / dflt["factor_solve_s"],
                                          "threads": "reference default (solver.cpp:366-390)"},
            "reference_selected_mode": allc["mode"],
            "residual_inf_max": allc["residual_inf_max"],
            "port": {"value": 1.0 / port_s, "unit": METRIC, "cores": 1, "kind": "port",
                     "sample": "the oracle's C restatement (bdlu_oracle.c, reference dense micro-kernel on every "
                               "merged block, reverse block solve) under the oracle's BTF: one factor + solve, "
                               "%.1f s, residual %.1e%s" % (port_s, port_res, "" if port_ok else ", FAILED")},
            "host": {"cores": cores, "cpu_model": model},
            "e2e": {"value": 1.0 / t, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_systems(count=BATCH_SYSTEMS, gen=None):
    """The batch workload's systems: block generator, n log-uniform in [1e3, 5e4].
    gen: the generator module (the engine package, or the oracle for the CPU
    baseline and the reference arm; both draw the same systems)."""
    if gen is None:
        import blockdaglu as gen
    rng = np.random.default_rng(gen.config_seed(BATCH_CONFIG))
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1000.0), np.log(50000.0))))
        out.append(gen.Synth(gen.FAMILY_BLOCK, gen.config_seed(BATCH_CONFIG, i), n))
    return out


def batch_step_inputs(systems, k):
    """Step k of the batch: every system's values x (1 + U(-0.1, 0.1)), and 8 rhs U(-1, 1)."""
    vals = np.concatenate([g.perturbed(2_000_003 + 7919 * k + i) for i, g in enumerate(systems)])
    rng = np.random.default_rng(3_000_017 + k)
    B = np.asfortranarray(rng.uniform(-1.0, 1.0, (sum(g.n for g in systems), BATCH_NRHS)))
    return vals, B


def batch_cpu_sample(sample=4):
    """The reference's BLOCK route (oracle/_ref, all host cores) on the first
    `sample` systems of the batch's step 0: per system set_matrix + analyze +
    factor + one solve_in_place per right-hand side (its API is single-RHS),
    after one untimed pass; scaled to systems/s."""
    oracle = oracle_module()
    cores, model = host_cpu()
    systems = batch_systems(BATCH_SYSTEMS, oracle)[:sample]
    vals, B = batch_step_inputs(systems, 0)
    os.environ["USERALGO_THREADS"] = str(cores)
    os.environ["USERALGO_MODE"] = "block"  # n < 50,000: AUTO would take the global KLU route (stand-in only)
    t_all = 0.0
    for rep in range(2):
        voff = off = 0
        t_rep = 0.0
        for g in systems:
            s = oracle.RefSolver()
            v = vals[voff:voff + g.nnz]
            t0 = time.perf_counter()
            ok = s.set_matrix(g.rows, g.cols, v, g.n) and s.analyze() and s.factor()
            for j in range(BATCH_NRHS):
                x = np.ascontiguousarray(B[off:off + g.n, j])
                ok = ok and s.solve_in_place(x)
            t_rep += time.perf_counter() - t0
            if not ok:
                raise RuntimeError("reference route failed: " + s.last_error_message())
            off += g.n
            voff += g.nnz
        t_all = t_rep
    os.environ.pop("USERALGO_THREADS", None)
    os.environ.pop("USERALGO_MODE", None)
    return {"value": sample / t_all, "unit": BATCH_METRIC, "cores": cores, "kind": "reference",
            "sample": "the first %d systems of the batch (n = %s), each through the reference's BLOCK route built "
                      "under oracle/_ref (set_matrix + analyze + factor + %d single-RHS solves, USERALGO_THREADS=%d on "
                      "%s), second of two passes: %.2f s" % (sample, [g.n for g in systems], BATCH_NRHS, cores, model,
                                                             t_all)}


def run_batch(args, rank, world):
    """batch-256: 256 independent systems per step through one bdlu_batch."""
    if args.impl == "reference":
        if rank != 0:
            return
        base = batch_cpu_sample()
        line = {"metric": BATCH_METRIC, "value": base["value"], "unit": BATCH_METRIC, "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "ms_per_step": 1000.0 * BATCH_SYSTEMS / base["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": BATCH_WORKLOAD, "systems": BATCH_SYSTEMS,
                                                "nrhs": BATCH_NRHS},
                "impl": "reference", "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": BATCH_METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch
    import blockdaglu as bd
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    systems = batch_systems()
    batch = bd.Batch()
    for g in systems:
        assert batch.add((g.rows, g.cols, g.vals), g.n) >= 0, batch.last_error_message()
    t0 = time.perf_counter()
    assert batch.analyze(), batch.last_error_message()
    analyze_s = time.perf_counter() - t0
    assert batch.factor(), batch.last_error_message()
    first = batch.stats()
    N = batch.rows()
    nnz = int(batch.nnz_offset(batch.count()))
    total = args.warmup + args.steps
    inputs = [batch_step_inputs(systems, k) for k in range(total)]
    d_vals = [torch.from_numpy(v).to(dev) for v, _ in inputs]
    d_B = [torch.from_numpy(np.ascontiguousarray(B.T)).to(dev) for _, B in inputs]  # (nrhs, N): column-major N x nrhs
    d_X = torch.empty(BATCH_NRHS, N, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sh = stream.cuda_stream

    def device_step(k):
        assert batch.refactor_values_device(d_vals[k].data_ptr(), nnz, sh), batch.last_error_message()
        assert batch.solve_device(d_X.data_ptr(), N, BATCH_NRHS, sh), batch.last_error_message()

    for k in range(args.warmup):
        d_X.copy_(d_B[k])
        device_step(k)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, phases, launches = [], [], []
    with ClockSampler(local) as clocks:
        for k in range(args.warmup, total):
            flush.fill_(float(k))
            d_X.copy_(d_B[k])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            device_step(k)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            phases.append(batch.phase_times())
            st = batch.stats()
            launches.append(st["factor_launches"] + st["solve_launches"])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # Per-system residual of the last timed step (host, FP64).
    X = d_X.cpu().numpy().T
    v_last, B_last = inputs[total - 1]
    import scipy.sparse as sp
    worst, off, voff = 0.0, 0, 0
    for g in systems:
        v = v_last[voff:voff + g.nnz]
        A = sp.csr_matrix((v, (g.rows, g.cols)), shape=(g.n, g.n))
        anorm = float(abs(A).sum(axis=1).max())
        x, b = X[off:off + g.n], B_last[off:off + g.n]
        R = b - A @ x
        rel = np.abs(R).max(axis=0) / (anorm * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
        worst = max(worst, float(rel.max()))
        off += g.n
        voff += g.nnz
    my_ms = max_over_ranks(sum(step_ms), dist, dev)
    ms_per_step = my_ms / args.steps
    value = world * BATCH_SYSTEMS * 1000.0 / ms_per_step
    # End to end through the C ABI with host buffers.
    pin_v = [torch.from_numpy(v).pin_memory() for v, _ in inputs]
    pin_B = torch.empty(BATCH_NRHS, N, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for k in range(total):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        pin_B.copy_(torch.from_numpy(np.ascontiguousarray(inputs[k][1].T)))
        t0 = time.perf_counter()
        rc = batch._lib.bdlu_batch_refactor_values(batch._b, bd._p64(pin_v[k].numpy()), nnz)
        rc = rc or batch._lib.bdlu_batch_solve(batch._b, bd._p64(pin_B.numpy()), N, BATCH_NRHS)
        dt = (time.perf_counter() - t0) * 1000.0
        assert rc == 0, batch.last_error_message()
        if k >= args.warmup:
            e2e_ms.append(dt)
    e2e = world * BATCH_SYSTEMS * 1000.0 / statistics.mean(e2e_ms)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    ph = {key: statistics.mean(p[key] for p in phases) for key in phases[0]}
    peaks = measured_peaks()
    dominant = max(("lu_small", "lu_large", "solve"), key=lambda key: ph[key])
    if dominant == "solve":
        traffic = 8 * first["dense_entries"] + 12 * first["nnz_offdiag"] + 8 * 4 * N * BATCH_NRHS
        achieved = traffic / (ph["solve"] * 1e-3) / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "kernel": "solve sweep, 8 rhs (k_solve_level levels)",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s"}
    else:
        n8 = 8192
        a = torch.randn(n8, n8, dtype=torch.float64, device=dev)
        torch.matmul(a, a)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e30
        for _ in range(3):
            e0.record()
            torch.matmul(a, a)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        dgemm = 2.0 * n8 ** 3 / (best * 1e-3) / 1e12
        achieved = first["factor_flops"] / (ph["lu_small"] + ph["lu_large"]) / 1e9
        roofline = {"bound": "tensor", "achieved": achieved, "peak": dgemm, "unit": "TFLOP/s", "frac": achieved / dgemm,
                    "traffic": None, "kernel": "dense block LU of all systems' blocks (k_lu_small), FP64",
                    "peak_source": "FP64 pipe: torch.matmul float64 8192^3 measured in this run"}
    cpu = batch_cpu_sample() if (world == 1 and not args.no_cpu_baseline) else None
    line = {
        "metric": BATCH_METRIC, "value": value, "unit": BATCH_METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "systems": BATCH_SYSTEMS, "rows": N, "nnz": nnz, "nrhs": BATCH_NRHS,
                   "nunits": first["nunits"], "max_block": first["max_unit"], "unit_levels": first["unit_levels"],
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed (256 MiB write) between timed steps, outside the step window",
                   "analyze_s": analyze_s},
        "e2e": {"value": e2e, "unit": BATCH_METRIC, "h2d_bytes_per_step": 8 * nnz + 8 * N * BATCH_NRHS,
                "d2h_bytes_per_step": 8 * N * BATCH_NRHS},
        "phases_ms": ph, "residual_inf_max": worst, "roofline": roofline, "cpu_baseline": cpu,
        "clocks": clocks.summary(), "gpu_launches": int(sum(launches)), "tuner": bd.tuner_report(),
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def serve_patterns(count=SERVE_PATTERNS, gen=None):
    """The serving workload's patterns: circuit generator, n log-uniform in
    [5e3, 3e5] (gen: engine package or oracle, same draws)."""
    if gen is None:
        import blockdaglu as gen
    rng = np.random.default_rng(gen.config_seed(SERVE_CONFIG))
    sizes = [int(np.exp(rng.uniform(np.log(5000.0), np.log(300000.0)))) for _ in range(count)]
    return [gen.Synth(gen.FAMILY_CIRCUIT, gen.config_seed(SERVE_CONFIG, i), n) for i, n in enumerate(sizes)]


def serve_reference_sample(args, budget_s):
    """The reference serving the closed-loop request stream the way its API
    allows: one Solver per pattern, each request set_matrix(new values) +
    analyze + factor + one solve_in_place per right-hand side, one request at
    a time, on all host cores (oracle/_ref).  A bounded sample: requests in
    stream order until about `budget_s` seconds of work, skipping requests
    whose pattern has a diagonal block above REF_SERVE_MAX_BLOCK rows (the
    dense KLU stand-in takes minutes on those), so the sample overstates the
    reference's throughput.  Returns the cpu_baseline dict."""
    import scipy.sparse as sp
    oracle = oracle_module()
    cores, model = host_cpu()
    patterns = serve_patterns(SERVE_PATTERNS, oracle)
    closed = serve_requests(patterns, max(args.steps, 1) * 64, 11)
    os.environ["USERALGO_THREADS"] = str(cores)
    # The BLOCK route: under AUTO the reference sends n < 50,000 to its global
    # KLU route, which the dense KLU stand-in cannot run at these sizes.
    os.environ["USERALGO_MODE"] = "block"
    solvers, done, skipped, t_total, worst = {}, 0, 0, 0.0, 0.0
    max_block = {}
    for k, v, B in closed:
        g = patterns[k]
        if k not in max_block:
            a = sp.csc_matrix((np.ones(g.nnz), (g.rows, g.cols)), shape=(g.n, g.n))
            a.sort_indices()
            _, _, _, R, _ = oracle.btf_order(g.n, a.indptr, a.indices)
            max_block[k] = int(np.max(np.diff(R)))
        if max_block[k] > REF_SERVE_MAX_BLOCK:
            skipped += 1
            continue
        s = solvers.setdefault(k, oracle.RefSolver())
        t0 = time.perf_counter()
        ok = s.set_matrix(g.rows, g.cols, v, g.n) and s.analyze() and s.factor()
        xs = []
        for j in range(B.shape[1]):
            if not ok:
                break
            x = np.ascontiguousarray(B[:, j])
            ok = s.solve_in_place(x)
            xs.append(x)
        dt = time.perf_counter() - t0
        if not ok:
            raise RuntimeError("reference route failed: " + s.last_error_message())
        t_total += dt
        done += 1
        worst = max(worst, max(oracle.metrics(g.rows, g.cols, v, x, B[:, j])[0] for j, x in enumerate(xs)))
        if t_total > budget_s and done >= 2:
            break
    os.environ.pop("USERALGO_THREADS", None)
    os.environ.pop("USERALGO_MODE", None)
    value = done / t_total
    sample = ("%d requests of the closed-loop stream in order (%d skipped: their pattern has a diagonal block above "
              "%d rows, which the dense KLU stand-in factors in minutes; the sample overstates the reference's "
              "throughput), each set_matrix + analyze + factor + single-RHS solves through the reference's BLOCK "
              "route built under oracle/_ref (own solver.cpp / ubtf_block_solver.cpp, KLU and BTF stand-ins; "
              "USERALGO_MODE=block: AUTO would send n < 50,000 to the global KLU route, which the stand-in cannot "
              "run), one Solver per pattern, one request at a time, USERALGO_THREADS=%d on %s: %.1f s, worst "
              "residual %.1e" % (done, skipped, REF_SERVE_MAX_BLOCK, cores, model, t_total, worst))
    return {"value": value, "unit": SERVE_METRIC, "cores": cores, "kind": "reference", "sample": sample,
            "requests": done, "seconds": t_total, "residual_inf_max": worst}


def run_serve_reference(args):
    """serve-64 reference arm: the sampled request stream (about a minute) and
    the circuit-200k value change, both through the reference build."""
    cores, model = host_cpu()
    base = serve_reference_sample(args, 60.0)
    circ = reference_route(oracle_circuit_system(), 1, 1, cores)
    value = base["value"]
    line = {"metric": SERVE_METRIC, "value": value, "unit": SERVE_METRIC, "n_gpus": args.gpus,
            "steps": base["requests"], "warmup": 0, "ms_per_step": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": SERVE_WORKLOAD, "patterns": SERVE_PATTERNS},
            "impl": "reference", "same_steps": False,
            "same_steps_reason": "a bounded sample of the request stream (about a minute of host work)",
            "residual_inf_max": base["residual_inf_max"],
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "circuit_200k": {"value": 1.0 / circ["step_s"], "unit": METRIC,
                             "factor_solve_only": 1.0 / circ["factor_solve_s"],
                             "phases_s": {k: circ[k] for k in ("analyze_s", "factor_s", "solve_s")},
                             "sample": "1 timed value change after 1 untimed, USERALGO_THREADS=%d" % cores},
            "host": {"cores": cores, "cpu_model": model},
            "e2e": {"value": value, "unit": SERVE_METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_requests(patterns, count, seed, nvals=3):
    """count requests: (pattern, values, B); values drawn from nvals perturbations per pattern."""
    rng = np.random.default_rng(seed)
    vals = [[g.perturbed(5_000_011 + 131 * i + j) for j in range(nvals)] for i, g in enumerate(patterns)]
    out = []
    for r in range(count):
        k = int(rng.integers(len(patterns)))
        nrhs = int(rng.integers(1, 17))
        B = np.asfortranarray(rng.uniform(-1.0, 1.0, (patterns[k].n, nrhs)))
        out.append((k, vals[k][r % nvals], B))
    return out


def serve_roofline_time(st, nnz, n, nrhs, p_flops, bw):
    """t_roof of one request: max(F / P, B / BW) with F = dense-block LU flops +
    2 * dense entries * nrhs (solve), B = values in (8 nnz) + factor write and
    read (8 + 8 per dense entry, the read once per 16 right-hand sides) +
    12 * coupling entries + 32 bytes per row and right-hand side."""
    passes = (nrhs + 15) // 16
    F = st["factor_flops"] + 2.0 * st["dense_entries"] * nrhs
    B = 8.0 * nnz + 8.0 * st["dense_entries"] * (1 + passes) + 12.0 * st["nnz_offdiag"] + 32.0 * n * nrhs
    return max(F / p_flops, B / bw)


def run_serve(args, rank, world):
    """serve-64: the served engine against the plain FP64 GPU path on one
    request stream.  `value`: closed loop with device-resident requests (values
    and right-hand sides already in HBM); `e2e`: the same stream through host
    buffers (bdlu_server_submit); open-loop Poisson arrivals for p50 / p99;
    the plain path runs the same requests one at a time, one Solver per
    pattern, through bdlu_refactor_solve with host buffers."""
    import concurrent.futures as cf
    if args.impl == "reference":
        if rank == 0:
            run_serve_reference(args)
        return
    import torch
    import blockdaglu as bd
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    cores, _ = host_cpu()
    patterns = serve_patterns()
    srv = bd.Server(SERVE_BUDGET, args.slots)
    assert srv.set_option("precision", args.precision), srv.last_error_message()
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max(1, min(8, cores))) as ex:
        ids = list(ex.map(lambda g: srv.add_pattern((g.rows, g.cols, g.vals), g.n), patterns))
    analyze_s = time.perf_counter() - t0
    assert all(i >= 0 for i in ids), srv.last_error_message()
    closed = serve_requests(patterns, max(args.steps, 1) * 64, 11)
    # Warm-up: per pattern an upload + first factor, a refactor with 1 and
    # with 16 right-hand sides (both solve graphs captured), and one
    # device-resident request.
    warm = [(k, patterns[k].vals, np.asfortranarray(np.ones((patterns[k].n, nr))))
            for nr in (1, 1, 16) for k in range(len(patterns))]
    for k, v, B in warm:
        srv.submit(ids[k], v, B)
    srv.drain()
    # Device-resident inputs: one device copy of each value set, one device
    # right-hand-side block per request (column-major, overwritten with X).
    dvals = {}
    for k, v, _ in closed:
        if id(v) not in dvals:
            dvals[id(v)] = torch.from_numpy(v).to(dev)
    dB0 = [torch.from_numpy(np.ascontiguousarray(B.T)).to(dev) for _, _, B in closed]
    wk = [(k, torch.from_numpy(patterns[k].vals).to(dev), torch.ones(1, patterns[k].n, dtype=torch.float64,
                                                                      device=dev)) for k in range(len(patterns))]
    for k, dv, db in wk:
        srv.submit_device(ids[k], dv.data_ptr(), patterns[k].nnz, db.data_ptr(), patterns[k].n, 1, keep=(dv, db))
    srv.drain()
    del wk
    # Closed loop, device-resident requests (value): all requests queued at
    # once; the time runs from the first submit to the last result, between
    # device synchronisations (the requests run on the server's worker
    # streams, which one event pair cannot bracket).
    dB = [b.clone() for b in dB0]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    srv.reset_stats()
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rids = [srv.submit_device(ids[k], dvals[id(v)].data_ptr(), len(v), b.data_ptr(), B.shape[0], B.shape[1])
                for (k, v, B), b in zip(closed, dB)]
        res = [srv.wait(r) for r in rids]
        torch.cuda.synchronize()
        dev_s = time.perf_counter() - t0
    dstats = srv.stats()
    assert all(r[0] for r in res), srv.last_error_message()
    worst = max(r[1] for r in res)
    # Check the device-resident solutions on the host (FP64 residual).
    for (k, v, B), b in zip(closed[:8], dB[:8]):
        g = patterns[k]
        X = b.cpu().numpy().T
        for j in range(B.shape[1]):
            r = B[:, j].copy()
            np.subtract.at(r, g.rows, v * X[g.cols, j])
            arow = np.zeros(g.n)
            np.add.at(arow, g.rows, np.abs(v))
            worst = max(worst, float(np.max(np.abs(r)) / (arow.max() * np.max(np.abs(X[:, j])) + np.max(np.abs(B[:, j])))))
    del dB
    dev_s_max = max_over_ranks(dev_s, dist, dev)
    value = world * len(closed) / dev_s_max
    # Closed loop, host buffers (e2e): the same requests through
    # bdlu_server_submit.
    outs = [B.copy(order="F") for _, _, B in closed]
    srv.reset_stats()
    t0 = time.perf_counter()
    rids = [srv.submit(ids[k], v, X) for (k, v, _), X in zip(closed, outs)]
    res = [srv.wait(r) for r in rids]
    host_s = time.perf_counter() - t0
    hstats = srv.stats()
    assert all(r[0] for r in res), srv.last_error_message()
    worst = max(worst, max(r[1] for r in res))
    host_s_max = max_over_ranks(host_s, dist, dev)
    e2e = world * len(closed) / host_s_max

    # Open loop: Poisson arrivals for --duration seconds at --rate, and at
    # 70 % of the closed-loop host-buffer throughput (a load it sustains).
    def open_loop(rate, seed):
        rng = np.random.default_rng(seed)
        n_open = max(1, int(rate * args.duration))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_open))
        opened = serve_requests(patterns, n_open, seed + 1)
        oouts = [B.copy(order="F") for _, _, B in opened]
        srv.reset_stats()
        t0 = time.perf_counter()
        orids = []
        for (k, v, _), X, ta in zip(opened, oouts, arrivals):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            orids.append(srv.submit(ids[k], v, X))
        ores = [srv.wait(r) for r in orids]
        secs = time.perf_counter() - t0
        st = srv.stats()
        assert all(r[0] for r in ores), srv.last_error_message()
        return {"rate": rate, "requests": n_open, "seconds": secs, "throughput": st["throughput"],
                "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
                "peak_concurrency": st["peak_concurrency"], "resident_bytes": st["resident_bytes"],
                "evictions": st["evictions"]}, max(r[1] for r in ores)

    open_spec, w1 = open_loop(args.rate, 17)
    open_fit, w2 = open_loop(0.7 * e2e / world, 23)
    worst = max(worst, w1, w2)
    # The same closed loop (host buffers) on the mixed route from 3xTF32
    # (server option "precision" 2: tensor-core trailing updates of the large
    # units, FP64 refinement to the same residual bound), after one 1-rhs and
    # one 16-rhs warm-up request per pattern at that precision.
    mixed = None
    if args.precision == 0:
        assert srv.set_option("precision", 2), srv.last_error_message()
        for k, v, B in warm[len(patterns):]:
            srv.submit(ids[k], v, np.asfortranarray(np.ones(B.shape)))
        srv.drain()
        mouts = [B.copy(order="F") for _, _, B in closed]
        srv.reset_stats()
        t0 = time.perf_counter()
        rids = [srv.submit(ids[k], v, X) for (k, v, _), X in zip(closed, mouts)]
        mres = [srv.wait(r) for r in rids]
        msecs = max_over_ranks(time.perf_counter() - t0, dist, dev)
        mst = srv.stats()
        assert all(r[0] for r in mres), srv.last_error_message()
        worst = max(worst, max(r[1] for r in mres))
        mixed = {"precision": 2, "requests": len(closed), "seconds": msecs,
                 "throughput": world * len(closed) / msecs, "p50_ms": mst["p50_ms"], "p99_ms": mst["p99_ms"],
                 "host_buffers": True, "worst_residual": max(r[1] for r in mres)}
    srv.close()
    # Plain FP64 GPU path: one request at a time, one Solver per pattern.
    sample = closed[: min(len(closed), 192)]
    solvers = {}
    for k in sorted({k for k, _, _ in closed}):
        s = bd.Solver()
        g = patterns[k]
        assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze() and s.factor(), s.last_error_message()
        X = np.ones(g.n)
        assert s.solve_in_place(X)
        X = np.asfortranarray(np.ones((g.n, 16)))
        assert s.refactor_values(g.vals) and s.solve_in_place(X), s.last_error_message()
        solvers[k] = s
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k, v, B in sample:
        X = B.copy(order="F")
        s = solvers[k]
        assert s._lib.bdlu_refactor_solve(s._h, bd._p64(v), len(v), bd._p64(X), X.shape[0], X.shape[1]) == 0, \
            s.last_error_message()
    plain_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    plain = world * len(sample) / plain_s
    # Roofline of the serving loop: sum over requests of max(F/P, B/BW), the
    # time an ideal device would need, against the wall time (value's run).
    pstats = {k: s.stats() for k, s in solvers.items()}
    del solvers
    peaks = measured_peaks()
    dgemm = measured_dgemm(dev)
    bw = peaks.get("hbm_gbs", 6650.0) * 1e9
    t_roof = sum(serve_roofline_time(pstats[k], patterns[k].nnz, patterns[k].n, B.shape[1], dgemm * 1e12, bw)
                 for k, _, B in closed)
    # The plain path on the 200k-row circuit system: device-timed steps, the
    # end-to-end call, phases and the roofline of its dominant phase.
    circ = measure_circuit(args, world, dist, dev)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = serve_reference_sample(args, 30.0) if (world == 1 and not args.no_cpu_baseline) else None
    nrhs_mean = float(np.mean([B.shape[1] for _, _, B in closed]))
    n_mean = float(np.mean([patterns[k].n for k, _, _ in closed]))
    nnz_mean = float(np.mean([patterns[k].nnz for k, _, _ in closed]))
    line = {
        "metric": SERVE_METRIC, "value": value, "unit": SERVE_METRIC, "n_gpus": world, "steps": len(closed),
        "warmup": len(warm) + len(patterns), "ms_per_step": 1000.0 * dev_s_max / len(closed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == 0 else "f64 storage, tf32 tensor-core updates, f64 refinement",
        "data": "synthetic",
        "config": {"workload": SERVE_WORKLOAD, "patterns": SERVE_PATTERNS, "slots": args.slots,
                   "precision": args.precision, "budget_bytes": SERVE_BUDGET,
                   "rows_min_max": [min(g.n for g in patterns), max(g.n for g in patterns)],
                   "requests": len(closed), "nrhs": "U{1..16}", "analyze_s": analyze_s,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (the request stream's factors and values total GBs)",
                   "value": "closed loop, device-resident requests (bdlu_server_submit_device), first submit to "
                            "last result between device synchronisations"},
        "e2e": {"value": e2e, "unit": SERVE_METRIC, "h2d_bytes_per_step": int(8 * nnz_mean + 8 * n_mean * nrhs_mean),
                "d2h_bytes_per_step": int(8 * n_mean * nrhs_mean)},
        "served_device_resident": {"requests": len(closed), "seconds": dev_s, "throughput": value,
                                   "p50_ms": dstats["p50_ms"], "p99_ms": dstats["p99_ms"],
                                   "peak_concurrency": dstats["peak_concurrency"]},
        "served_host_buffers": {"requests": len(closed), "seconds": host_s, "throughput": e2e,
                                "p50_ms": hstats["p50_ms"], "p99_ms": hstats["p99_ms"],
                                "peak_concurrency": hstats["peak_concurrency"]},
        "served_open_loop": open_spec,
        "served_open_loop_sustainable": open_fit,
        "served_mixed_3xtf32": mixed,
        "plain_fp64_path": {"requests": len(sample), "throughput": plain, "host_buffers": True},
        "ratio_served_over_plain": e2e / plain,
        "ratio_served_device_resident_over_plain": value / plain,
        "serving_roofline": {"sum_t_roof_s": t_roof, "wall_s": dev_s, "frac": t_roof / dev_s,
                             "peaks": {"fp64_tflops": dgemm, "hbm_gbs": bw / 1e9},
                             "formula": "t_roof(req) = max(F/P_fp64, B/BW) summed over the closed-loop requests"},
        "plain_circuit_200k": {"value": circ["value"], "e2e": circ["e2e"], "ms_per_step": circ["ms_per_step"],
                               "phases_ms": circ["phases_ms"], "residual_inf_max": circ["residual_inf_max"],
                               "gpu_launches": circ["gpu_launches"], "unit": METRIC},
        "residual_inf_max": worst,
        "roofline": dict(circ["roofline"], workload=CIRCUIT_WORKLOAD + " plain FP64 path (measured in this run)"),
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": int(dstats["kernel_launches"]),
        "tuner": circ["tuner"],
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_precision(args, rank, world):
    """precision-200: FP64 route vs mixed route, kappa 1e4 and 1e8."""
    import blockdaglu as bd
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "metric": PREC_METRIC, "unavailable":
                              "precision-200 needs about 45 GB of dense FP64 factors; the single-thread oracle port "
                              "would take hours (see the circuit-200k reference arm)"}), flush=True)
        return
    if world > 1 and rank != 0:
        return
    out = {}
    for label, kexp in (("a", 4), ("b", 8)):
        g = bd.Synth(bd.FAMILY_PRECISION, bd.config_seed(PREC_CONFIG, kexp), args.blocks, kexp)
        rng = np.random.default_rng(kexp)
        B = np.asfortranarray(rng.uniform(-1.0, 1.0, (g.n, PREC_NRHS)))
        res = {"n": g.n, "nnz": int(g.nnz)}
        X64 = None
        for mode in (0, 1, 2):
            s = bd.Solver()
            s.set_option("precision", mode)
            s.set_option("refactor_pivoting", 1)   # every factorisation searches pivots
            t0 = time.perf_counter()
            assert s.set_matrix((g.rows, g.cols, g.vals), g.n) and s.analyze(), s.last_error_message()
            analyze_s = time.perf_counter() - t0
            assert s.factor(), s.last_error_message()   # warm-up (upload, first launch of every kernel)
            steps = []
            for k in range(max(1, min(args.steps, 2))):
                v = g.perturbed(900 + k)
                X = B.copy(order="F")
                t0 = time.perf_counter()
                assert s.refactor_values(v), s.last_error_message()
                tf = time.perf_counter() - t0
                assert s.solve_in_place(X), s.last_error_message()
                steps.append((time.perf_counter() - t0, tf))
            st = s.stats()
            ph = s.phase_times()
            key = {0: "fp64", 1: "mixed", 2: "mixed_3xtf32"}[mode]
            res[key] = {"seconds_per_step": statistics.mean(t for t, _ in steps),
                        "factor_seconds": statistics.mean(f for _, f in steps),
                        "residual_inf": st["residual_inf"], "refine_iters": st["refine_iters"],
                        "precision_level": {0: "fp64", 1: "tf32", 2: "3xtf32"}[st["precision"]],
                        "factor_flops": st["factor_flops"], "max_block": st["max_unit"], "analyze_s": analyze_s,
                        "last_phases_ms": ph}
            if mode == 0:
                X64 = X.copy()
            else:
                res[key]["error_vs_fp64"] = float(np.max(np.abs(X - X64)) / np.max(np.abs(X64)))
            del s
        res["speedup_mixed_over_fp64"] = res["fp64"]["seconds_per_step"] / res["mixed"]["seconds_per_step"]
        res["speedup_mixed_3xtf32_over_fp64"] = res["fp64"]["seconds_per_step"] / res["mixed_3xtf32"]["seconds_per_step"]
        out[label] = res
        del g
    a = out["a"]
    best = min(("mixed", "mixed_3xtf32"), key=lambda k: a[k]["seconds_per_step"])
    value = 1.0 / a[best]["seconds_per_step"]
    line = {"metric": PREC_METRIC, "value": value, "unit": PREC_METRIC, "n_gpus": 1, "steps": max(1, min(args.steps, 2)),
            "warmup": 1, "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 storage, tf32 tensor-core updates, f64 refinement", "data": "synthetic",
            "config": {"workload": PREC_WORKLOAD, "blocks": args.blocks, "nrhs": PREC_NRHS,
                       "value_from": "instance a (kappa 1e4), the faster mixed route (TF32 start or 3xTF32 start), "
                                     "host buffers"},
            "instances": out, "roofline": None, "cpu_baseline": None, "gpu_launches": None}
    flops = a["mixed"]["factor_flops"]
    line["tensor_update_tflops"] = flops / a["mixed"]["factor_seconds"] / 1e12
    line["fp64_update_tflops"] = flops / a["fp64"]["factor_seconds"] / 1e12
    print(json.dumps(line), flush=True)


def measure_circuit(args, world, dist, dev):
    """circuit-200k on this rank: device-timed value-only refactor + 1-RHS solve
    steps (inputs resident in HBM, L2 flushed between steps), the same steps
    end to end through bdlu_refactor_solve with pinned host buffers, phase
    times and the roofline of the dominant phase.  Returns a dict."""
    import torch
    import blockdaglu as bd
    stream = torch.cuda.current_stream(dev)
    g = circuit_system()
    s = bd.Solver()
    if args.refactor_schedule is not None:
        assert s.set_option("refactor_schedule", args.refactor_schedule)
    assert s.set_matrix((g.rows, g.cols, g.vals), g.n), s.last_error_message()
    t0 = time.perf_counter()
    assert s.analyze(), s.last_error_message()
    analyze_s = time.perf_counter() - t0
    assert s.factor(), s.last_error_message()
    first = s.stats()
    nnz = int(g.nnz)
    total = args.warmup + args.steps
    inputs = [step_inputs(g, k) for k in range(total)]
    d_vals = [torch.from_numpy(v).to(dev) for v, _ in inputs]
    d_b = [torch.from_numpy(b).to(dev) for _, b in inputs]
    d_x = torch.empty(g.n, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    sh = stream.cuda_stream

    def device_step(k):
        assert s.refactor_values_device(d_vals[k].data_ptr(), nnz, sh), s.last_error_message()
        assert s.solve_device(d_x.data_ptr(), g.n, 1, sh), s.last_error_message()

    # Untimed: six host-buffer refactor + solve calls (the autotuner's trials
    # of the large-unit refactor schedule), then the device-path warm-up.
    for k in range(6):
        v, b = inputs[k % total]
        x = b.copy()
        assert s.refactor_values(v) and s.solve_in_place(x), s.last_error_message()
    for k in range(args.warmup):
        d_x.copy_(d_b[k])
        device_step(k)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, phases, resid, launches = [], [], [], []
    with ClockSampler(dev.index or 0) as clocks:
        for k in range(args.warmup, total):
            flush.fill_(float(k))
            d_x.copy_(d_b[k])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            device_step(k)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            phases.append(s.phase_times())
            st = s.stats()
            launches.append(st["factor_launches"] + st["solve_launches"])
            x = d_x.cpu().numpy()
            v, b = inputs[k]
            r = b.copy()
            np.subtract.at(r, g.rows, v * x[g.cols])
            arow = np.zeros(g.n)
            np.add.at(arow, g.rows, np.abs(v))
            resid.append(float(np.max(np.abs(r)) / (arow.max() * np.max(np.abs(x)) + np.max(np.abs(b)))))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    my_ms = max_over_ranks(sum(step_ms), dist, dev)
    ms_per_step = my_ms / args.steps
    value = world * 1000.0 / ms_per_step
    # End to end through the C ABI with pinned host buffers.
    pin_v = [torch.from_numpy(v).pin_memory() for v, _ in inputs]
    pin_b = torch.empty(g.n, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for k in range(total):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        pin_b.copy_(torch.from_numpy(inputs[k][1]))
        t0 = time.perf_counter()
        ok = s._lib.bdlu_refactor_solve(s._h, bd._p64(pin_v[k].numpy()), nnz, bd._p64(pin_b.numpy()), g.n, 1)
        dt = (time.perf_counter() - t0) * 1000.0
        assert ok == 0, s.last_error_message()
        if k >= args.warmup:
            e2e_ms.append(dt)
    e2e_ms_max = max_over_ranks(statistics.mean(e2e_ms), dist, dev)
    e2e = world * 1000.0 / e2e_ms_max
    ph = {key: statistics.mean(p[key] for p in phases) for key in phases[0]}
    dominant = max(("lu_small", "lu_large", "solve"), key=lambda key: ph[key])
    peaks = measured_peaks()
    if dominant == "solve":
        traffic = 8 * first["dense_entries"] + 12 * first["nnz_offdiag"] + 8 * 4 * g.n
        achieved = traffic / (ph["solve"] * 1e-3) / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "kernel": "solve sweep (k_solve_level / k_trsv_tiles levels)",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s"}
    else:
        dgemm = measured_dgemm(dev)
        achieved = first["factor_flops"] / (ph["lu_small"] + ph["lu_large"]) / 1e9
        roofline = {"bound": "tensor", "achieved": achieved, "peak": dgemm, "unit": "TFLOP/s",
                    "frac": achieved / dgemm, "traffic": profile_traffic("k_rgemm"),
                    "kernel": "dense block LU phases (k_lu_small; value-only refactor: k_rpanel / k_rgemm step "
                              "chain, or k_rdag tile task graph), FP64 FMA pipe",
                    "peak_source": "FP64: torch.matmul float64 8192^3 measured in this run (MEASURED_PEAKS.json "
                                   "has no FP64 figure)"}
    return {"value": value, "ms_per_step": ms_per_step, "e2e": e2e, "phases_ms": ph, "tuner": bd.tuner_report(),
            "residual_inf_max": max(resid), "roofline": roofline, "clocks": clocks.summary(),
            "gpu_launches": int(sum(launches)), "n": g.n, "nnz": nnz, "first": first, "analyze_s": analyze_s}


def measured_dgemm(dev):
    """FP64 GEMM throughput of this GPU (torch.matmul float64, 8192^3, best of 3)."""
    import torch
    n8 = 8192
    a = torch.randn(n8, n8, dtype=torch.float64, device=dev)
    torch.matmul(a, a)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(3):
        e0.record()
        torch.matmul(a, a)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a
    return 2.0 * n8 ** 3 / (best * 1e-3) / 1e12


def profile_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary profiles/traffic.json, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel, {}).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def run_circuit(args, rank, world):
    """circuit-200k: the plain FP64 path on the 200k-row circuit system."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    c = measure_circuit(args, world, dist, dev)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_reference(oracle_circuit_system())
    first = c["first"]
    line = {
        "metric": METRIC, "value": c["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": c["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": CIRCUIT_WORKLOAD, "n": c["n"], "nnz": c["nnz"], "nrhs": 1, "nblocks": first["nblocks"],
                   "nunits": first["nunits"], "max_block": first["max_unit"], "unit_levels": first["unit_levels"],
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed (256 MiB write) between timed steps, outside the step window",
                   "refactor_schedule": {None: "autotuned", 0: "step chain", 1: "task graph"}[args.refactor_schedule],
                   "analyze_s": c["analyze_s"]},
        "e2e": {"value": c["e2e"], "unit": METRIC, "h2d_bytes_per_step": 8 * c["nnz"] + 8 * c["n"],
                "d2h_bytes_per_step": 8 * c["n"]},
        "phases_ms": c["phases_ms"],
        "residual_inf_max": c["residual_inf_max"],
        "roofline": c["roofline"],
        "cpu_baseline": cpu,
        "clocks": c["clocks"],
        "gpu_launches": c["gpu_launches"],
        "tuner": c["tuner"],
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def sparse_units_system(seed, blocks, extra, lo=SPARSE_MIN_ROWS, hi=SPARSE_MAX_ROWS, single=False):
    """Upper block triangular system of `blocks` sparse irreducible blocks of
    U{lo..hi} rows: a cyclic chain, the diagonal and extra*m random entries
    per block, magnitudes U(0.5, 2) with random sign; every third row couples
    to a later block (N(0, 0.1)); random row and column permutations.
    single: one block left in its own order with its diagonal scaled by 4
    (the global route factors it as it is).  Returns the canonical COO (rows
    sorted, duplicates summed)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, blocks)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    n = int(starts[-1])
    rows, cols = [], []
    for b, m in enumerate(sizes):
        o = int(starts[b])
        i = np.arange(m)
        k = int(extra * m)
        rows += [o + i, o + i, o + rng.integers(0, m, k)]
        cols += [o + i, o + (i + 1) % m, o + rng.integers(0, m, k)]
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = rng.uniform(0.5, 2.0, len(r)) * rng.choice([-1.0, 1.0], len(r))
    cr, cc = [np.zeros(0, np.int64)], [np.zeros(0, np.int64)]
    for b, m in enumerate(sizes[:-1]):
        i = np.arange(int(starts[b]), int(starts[b + 1]), 3)
        cr.append(i)
        cc.append(rng.integers(int(starts[b + 1]), n, len(i)))
    cr, cc = np.concatenate(cr), np.concatenate(cc)
    r = np.concatenate([r, cr])
    c = np.concatenate([c, cc])
    v = np.concatenate([v, 0.1 * rng.standard_normal(len(cr))])
    if single:
        v[:n] *= 4.0  # the diagonal entries come first
        p = q = np.arange(n)
    else:
        p, q = rng.permutation(n), rng.permutation(n)
    A = sp.csr_matrix((v, (np.argsort(p)[r], np.argsort(q)[c])), shape=(n, n))
    A.sum_duplicates()
    A.eliminate_zeros()
    A = A.tocoo()
    order = np.lexsort((A.col, A.row))
    return n, A.row[order].astype(np.int32), A.col[order].astype(np.int32), A.data[order].astype(np.float64)


def run_sparse_units(args, rank, world):
    """sparse-units: refactor + solve of systems of sparse blocks on the
    sparse-LU route against the dense route, per fill class."""
    import blockdaglu as bd
    if args.impl == "reference" or (world > 1 and rank != 0):
        if rank == 0:
            print(json.dumps({"impl": "reference", "metric": METRIC, "unavailable":
                              "sparse-units is the engine's fill-threshold sweep; the reference's sparse route is "
                              "timed in its cpu_baseline"}), flush=True)
        return
    classes = []
    steps, warm = max(1, args.steps), max(1, args.warmup)
    plan = [("blocks", ci, SPARSE_BLOCKS, SPARSE_MIN_ROWS, SPARSE_MAX_ROWS, e) for ci, e in enumerate(SPARSE_EXTRAS)]
    plan += [("single", 100 + ci, 1, m, m, e) for ci, (m, e) in enumerate(SPARSE_SINGLE)]
    for kind, ci, blocks, lo, hi, extra in plan:
        if args.sparse_extra and extra not in args.sparse_extra:
            continue
        if args.sparse_single is not None and (kind == "single") != bool(args.sparse_single):
            continue
        n, r, c, v = sparse_units_system(SPARSE_SEED + ci, blocks, extra, lo, hi, single=kind == "single")
        rng = np.random.default_rng(ci)
        vals = [v * (1.0 + rng.uniform(-0.01, 0.01, len(v))) for _ in range(steps + warm)]
        b = rng.uniform(-1.0, 1.0, n)
        res = {"kind": kind, "blocks": blocks, "rows": [lo, hi], "extra_per_row": extra, "n": n, "nnz": int(len(v))}
        for label, mode in (("dense", 0), ("sparse", 2)):
            s = bd.Solver()
            s.set_option("sparse_lu", mode)
            s.set_option("sparse_fill_max", 1.0)
            s.set_option("sparse_max_n", 8192)
            # A single block on the global route: one unit in its own order.
            saved = os.environ.get("BLOCKDAGLU_MODE")
            if kind == "single":
                os.environ["BLOCKDAGLU_MODE"] = "klu"
            try:
                assert s.set_matrix((r, c, v), n) and s.analyze() and s.factor(), s.last_error_message()
            finally:
                if saved is None:
                    os.environ.pop("BLOCKDAGLU_MODE", None)
                else:
                    os.environ["BLOCKDAGLU_MODE"] = saved
            fac, sol = [], []
            for k in range(steps + warm):
                x = b.copy()
                assert s.refactor_values(vals[k]), s.last_error_message()
                st = s.stats()
                assert s.solve_in_place(x), s.last_error_message()
                st2 = s.stats()
                if k >= warm:
                    fac.append(st["last_factor_ms"])
                    sol.append(st2["last_solve_ms"])
                assert st2["residual_inf"] <= 1e-12, st2["residual_inf"]
            start, route, reason, lu_nnz = s.unit_routes(with_nnz=True)
            m = np.diff(np.append(start, n))
            sel = route == 3
            res[label] = {"factor_ms": statistics.median(fac), "solve_ms": statistics.median(sol),
                          "factor_flops": s.stats()["factor_flops"]}
            if mode:
                big = m > 64
                res[label].update({"sparse_units": int(sel.sum()), "candidate_units": int(big.sum()),
                                   "rejected_by_pivot_test": int(((reason >= 1) & (reason <= 4)).sum()),
                                   "mean_fill": float(np.mean(lu_nnz[sel] / (m[sel].astype(float) ** 2)))
                                   if sel.any() else None})
            del s
        res["sparse_over_dense"] = ((res["dense"]["factor_ms"] + res["dense"]["solve_ms"]) /
                                    (res["sparse"]["factor_ms"] + res["sparse"]["solve_ms"]))
        classes.append(res)
        print(json.dumps({"class": res}), file=sys.stderr, flush=True)
    wins = [cl["sparse"]["mean_fill"] for cl in classes if cl["sparse_over_dense"] > 1.0 and cl["sparse"]["mean_fill"]]
    first = classes[0]
    ms = first["sparse"]["factor_ms"] + first["sparse"]["solve_ms"]
    line = {"metric": METRIC, "value": 1000.0 / ms, "unit": METRIC, "n_gpus": 1, "steps": steps, "warmup": warm,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": SPARSE_WORKLOAD, "blocks": SPARSE_BLOCKS,
                       "block_rows": [SPARSE_MIN_ROWS, SPARSE_MAX_ROWS],
                       "value_from": "first class run, on the sparse-LU route, device-timed factor + 1-rhs solve"},
            "classes": classes, "largest_fill_where_sparse_wins": max(wins) if wins else None,
            "roofline": None, "cpu_baseline": None, "gpu_launches": None}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.workload == BATCH_WORKLOAD:
        run_batch(args, rank, world)
    elif args.workload == SERVE_WORKLOAD:
        run_serve(args, rank, world)
    elif args.workload == PREC_WORKLOAD:
        run_precision(args, rank, world)
    elif args.workload == SPARSE_WORKLOAD:
        run_sparse_units(args, rank, world)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_circuit(args, rank, world)


if __name__ == "__main__":
    main()
