// C ABI (include/bdlu.h): the Solver state machine of blockdaglu/src/solver.cpp
// (set_matrix :749-800, analyze :802-1182, factor :1184-1350, solve_in_place
// :1352-1539, exports :1541-1725) over the GPU engine.  No exception crosses
// the boundary; every failure maps to a status code and a message.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "analysis.h"
#include "bdlu.h"
#include "capi_internal.h"
#include "engine.h"
#include "plan.h"
#include "tuner.h"

using bdlu::Status;
using bdlu::Tuner;

namespace {
// Normwise residual above which a refactor that reused the pivot order is
// redone with partial pivoting by the host-buffer solve.
constexpr double kReuseResidualLimit = 1e-12;
}  // namespace

namespace {

int fail(bdlu_solver* h, int code, std::string msg) {
  h->last_error = code;
  h->last_message = std::move(msg);
  return code;
}

void clear_error(bdlu_solver* h) {
  h->last_error = BDLU_OK;
  h->last_message.clear();
}

int refine_iters_for(const bdlu_solver* h) {
  if (h->refine_iters >= 0) return h->refine_iters;
  if (const char* e = bdlu::getenv_compat("USERALGO_REFINE_ITERS")) {
    const int v = std::atoi(e);
    if (v >= 0) return v;
  }
  return 0;
}

int pick_mode() {
  // solver.cpp:824-841: unknown values fall back to AUTO.
  if (const char* e = bdlu::getenv_compat("USERALGO_MODE")) {
    std::string v(e);
    for (auto& c : v) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    if (v == "klu") return BDLU_MODE_KLU;
    if (v == "block") return BDLU_MODE_BLOCK;
  }
  return BDLU_MODE_AUTO;
}

// Runs validation + canonicalisation once (solver.cpp:806-819).
int ensure_validated(bdlu_solver* h) {
  if (h->validated) return BDLU_OK;
  std::string msg;
  const Status st = bdlu::canonicalize(h->in_rows.data(), h->in_cols.data(), h->in_vals.data(),
                                       static_cast<int64_t>(h->in_rows.size()), h->dimension_hint, h->coo, msg);
  if (st != Status::Ok) return fail(h, static_cast<int>(st), msg);
  h->n = h->coo.n;
  h->validated = true;
  return BDLU_OK;
}

// Whether the refactor schedule of this handle is being tuned: FP64 route,
// large units with a tile task graph, no schedule set by the caller.
bool schedule_tunable(const bdlu_solver* h) {
  return !h->schedule_user_set && !h->mixed && h->engine && Tuner::get().enabled() &&
         !h->engine->plan().large_units.empty() && h->engine->plan().rtasks > 0;
}

// Schedule of the next value-only refactor: the caller's, the tuned one, or
// the next trial (chain, graph, chain, graph, chain, graph).
int32_t schedule_for(bdlu_solver* h) {
  if (!schedule_tunable(h)) return h->refactor_schedule;
  const int t = Tuner::get().refactor_schedule(h->sig);
  if (t >= 0) return t;
  return h->sched_trials & 1;
}

// After a refactor that reused the pivot order completed: a trial's device
// time.  The first trial of each schedule captures its graph and is not
// counted; each schedule's time is the faster of its next two, and after the
// sixth trial the faster schedule is kept for the pattern.
constexpr int kScheduleTrials = 6;
void record_schedule(bdlu_solver* h, int32_t used) {
  if (!schedule_tunable(h) || !h->engine->last_factor_reused()) return;
  Tuner& tu = Tuner::get();
  if (tu.refactor_schedule(h->sig) >= 0 || (h->sched_trials & 1) != used) return;
  const float ms = h->engine->last_factor_ms();
  if (h->sched_trials >= 2) h->sched_ms[used] = h->sched_trials < 4 ? ms : std::min(h->sched_ms[used], ms);
  if (++h->sched_trials == kScheduleTrials) {
    // The chain is the default: the graph must win by more than 2 %, so
    // trial noise between two close schedules does not flip the choice.
    const int best = h->sched_ms[1] < 0.98f * h->sched_ms[0] ? 1 : 0;
    tu.set_refactor_schedule(h->sig, best, h->sched_ms[0], h->sched_ms[1]);
  }
}

int replan_without(bdlu_solver* h, const std::vector<int32_t>& units, const std::vector<int32_t>& reasons,
                   cudaStream_t stream);

// Factor from the engine's value buffer.  reuse: large blocks keep the pivot
// order of the last full factorisation (value-only refactor); a zero pivot
// met that way falls back to a factorisation with pivoting.  A sparse-LU unit
// that fails its pivot test (the reference's gate would reject it) moves to
// the dense route: the plan is rebuilt without it and the factor rerun.
int do_factor(bdlu_solver* h, cudaStream_t stream, bool reuse) {
  std::string err;
  h->engine->set_precision(h->mixed ? h->prec_level : 0);
  h->engine->set_lu_small_width(h->lu_small_threads);
  h->engine->set_blocking_sync(h->blocking_sync);
  h->engine->set_programmatic_launch(h->programmatic_launch);
  h->engine->set_small_mode(h->small_mode);
  const int32_t sched = schedule_for(h);
  h->engine->set_refactor_schedule(sched);
  h->engine->set_wait_limit(h->wait_limit);
  h->engine->set_sparse_tests(h->gp.diag_tol, h->gp.pivot_tol, h->gp.min_abs_diag);
  int replans = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const bool r = reuse && attempt == 0;
    if (!h->engine->factor_async(h->engine->values_buffer(), stream, err, r))
      return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
    const int st = h->engine->factor_status(stream, err);
    if (st == 0) {
      h->factored = true;
      h->exported = false;
      if (r) record_schedule(h, sched);
      return BDLU_OK;
    }
    if (st == 3 && replans < 2) {
      std::vector<int32_t> units, reasons;
      if (!h->engine->sparse_rejections(units, reasons, err)) return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
      if (const int e = replan_without(h, units, reasons, stream)) {
        h->factored = false;
        return e;
      }
      ++replans;
      --attempt;
      continue;
    }
    if (st == 2 && r) continue;
    h->factored = false;
    return fail(h, st < 0 ? BDLU_BACKEND_UNAVAILABLE : BDLU_FACTORIZATION_FAILED, err);
  }
  h->factored = false;
  return fail(h, BDLU_FACTORIZATION_FAILED, err);
}

// True if no entry is NaN or infinite: branch-free over the whole array (no
// early exit, so the loop vectorises).  One thread: helper threads lost to
// busy OpenMP workers of the calling process in measurements.
bool all_finite(const double* v, int64_t n);

}  // namespace

bool bdlu_copy_finite(double* dst, const double* src, int64_t n) {
  uint64_t bad = 0;
  for (int64_t k = 0; k < n; ++k) {
    uint64_t x;
    std::memcpy(&x, src + k, sizeof(x));
    bad |= static_cast<uint64_t>(((x >> 52) & 0x7ff) == 0x7ff);
    std::memcpy(dst + k, &x, sizeof(x));
  }
  return bad == 0;
}

namespace {

bool all_finite(const double* v, int64_t n) {
  uint64_t bad = 0;
  for (int64_t k = 0; k < n; ++k) {
    uint64_t x;
    std::memcpy(&x, v + k, sizeof(x));
    bad |= static_cast<uint64_t>(((x >> 52) & 0x7ff) == 0x7ff);
  }
  return bad == 0;
}

int upload_values(bdlu_solver* h, const double* vals, bool device, cudaStream_t stream) {
  const size_t bytes = static_cast<size_t>(h->engine->nnz()) * sizeof(double);
  const cudaError_t e = cudaMemcpyAsync(h->engine->values_buffer(), vals, bytes,
                                        device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return fail(h, BDLU_BACKEND_UNAVAILABLE, std::string("value upload: ") + cudaGetErrorString(e));
  return BDLU_OK;
}

// Units whose sparse LU failed its pivot test join the dense route for this
// handle (the reference rejects such a block at its gate and factors it with
// KLU): the plan is rebuilt without them, with the current values.
int replan_without(bdlu_solver* h, const std::vector<int32_t>& units, const std::vector<int32_t>& reasons,
                   cudaStream_t stream) {
  const bdlu::Plan& old = h->engine->plan();
  for (size_t i = 0; i < units.size(); ++i) {
    const int32_t s0 = old.ustart[static_cast<size_t>(units[i])];
    h->gp.rejected.push_back(s0);
    h->gp_rejected_reason.emplace_back(s0, reasons[i]);
  }
  if (const int st = bdlu_sync_host_values(h)) return st;
  try {
    const bdlu::Plan plan = bdlu::build_plan(h->coo, h->dec, bdlu::small_unit_max(), &h->gp);
    std::string err;
    if (!h->engine->upload(plan, h->dec, h->coo, err)) return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
  } catch (const std::exception& e) {
    return fail(h, BDLU_ANALYSIS_FAILED, e.what());
  }
  h->engine->set_pattern_key(h->sig);
  return upload_values(h, h->coo.val.data(), false, stream);
}

}  // namespace

int bdlu_sync_host_values(bdlu_solver* h) {
  if (!h->host_vals_stale) return BDLU_OK;
  if (!h->engine) return fail(h, BDLU_BACKEND_UNAVAILABLE, "the device holding the current values was released");
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess)
    e = cudaMemcpy(h->coo.val.data(), h->engine->values_buffer(), static_cast<size_t>(h->coo.nnz()) * sizeof(double),
                   cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(h, BDLU_BACKEND_UNAVAILABLE, std::string("value download: ") + cudaGetErrorString(e));
  h->host_vals_stale = false;
  return BDLU_OK;
}

// Analysis of an already validated canonical matrix under route `mode`
// (solver.cpp:820-1182): signatures, decomposition, device plan and upload.
int bdlu_analyze_validated(bdlu_solver* h, int mode, const bdlu::PrecomputedBtf* btf) {
  if (const int st = bdlu_sync_host_values(h)) return st;
  h->sig = bdlu::matrix_sig(h->n, h->coo);
  h->sig2 = bdlu::matrix_sig2(h->n, h->coo);
  h->value_sig = bdlu::matrix_value_sig(h->coo);
  h->mode = mode;
  // The GPU engine runs the block route under AUTO; "klu" forces the global
  // route, which here means one diagonal block with partial pivoting.  AUTO
  // still takes the reference's route decision so selected_mode() reports
  // what the reference would select (solver.cpp:846-861).
  h->global_route = (h->mode == BDLU_MODE_KLU);
  h->auto_picked_klu = (h->mode == BDLU_MODE_AUTO) && !bdlu::auto_choose_block(h->n, h->coo);
  h->decomposed = false;
  h->factored = false;
  h->exported = false;
  try {
    bdlu::AnalysisOptions opt = bdlu::analysis_options_from_env();
    opt.single_block = h->global_route;
    opt.btf = btf;
    h->dec = bdlu::build_decomposition(h->coo, opt);
    if (h->analysis_only) {
      h->engine.reset();
      h->decomposed = true;
      return BDLU_OK;
    }
    int dev_count = 0;
    const cudaError_t ce = cudaGetDeviceCount(&dev_count);
    if (ce != cudaSuccess || dev_count <= 0)
      return fail(h, BDLU_BACKEND_UNAVAILABLE,
                  std::string("no CUDA device available: ") + (ce != cudaSuccess ? cudaGetErrorString(ce) : "0 devices"));
    h->gp = bdlu::gp_config_from_env();
    if (h->sparse_lu_opt >= 0) h->gp.mode = h->sparse_lu_opt;
    if (h->sparse_fill_max > 0.0) h->gp.fill_max = h->sparse_fill_max;
    if (h->sparse_max_n > 0) h->gp.max_n = h->sparse_max_n;
    h->gp_rejected_reason.clear();
    const bdlu::Plan plan = bdlu::build_plan(h->coo, h->dec, bdlu::small_unit_max(), &h->gp);
    if (!h->engine) h->engine = std::make_unique<bdlu::Engine>();
    std::string err;
    if (!h->engine->upload(plan, h->dec, h->coo, err)) return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
    h->engine->set_pattern_key(h->sig);
    // The engine keeps its own value buffer; load the analysed values.
    if (const int st = upload_values(h, h->coo.val.data(), false, nullptr)) return st;
  } catch (const std::bad_alloc&) {
    return fail(h, BDLU_ANALYSIS_FAILED, "out of host memory during analysis");
  } catch (const std::exception& e) {
    return fail(h, BDLU_ANALYSIS_FAILED, e.what());
  }
  h->decomposed = true;
  return BDLU_OK;
}

// Host values to the engine's value buffer: they travel to a device staging
// buffer while the host checks them (the copy overlaps the check for pinned
// buffers) and move to the value buffer only if every entry is finite.  No
// host copy is kept (10 MB per million entries): coo.val is refreshed from
// the device when something reads it.
static int stage_host_values(bdlu_solver* h, const double* vals, int64_t nnz, cudaStream_t stream, bool checked) {
  std::string err;
  double* stg = h->engine->value_staging(err);
  if (!stg) return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
  const size_t bytes = static_cast<size_t>(nnz) * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(stg, vals, bytes, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return fail(h, BDLU_BACKEND_UNAVAILABLE, std::string("value upload: ") + cudaGetErrorString(e));
  if (!checked && !all_finite(vals, nnz)) {
    cudaStreamSynchronize(stream);  // the staging copy ends before the error returns
    return fail(h, BDLU_NON_FINITE_VALUE, "matrix contains NaN or infinity");
  }
  e = cudaMemcpyAsync(h->engine->values_buffer(), stg, bytes, cudaMemcpyDeviceToDevice, stream);
  if (e != cudaSuccess) return fail(h, BDLU_BACKEND_UNAVAILABLE, std::string("value upload: ") + cudaGetErrorString(e));
  h->host_vals_stale = true;
  return BDLU_OK;
}

static int refactor_checks(bdlu_solver* h, const double* vals, int64_t nnz) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (!h->decomposed) return fail(h, BDLU_NOT_PREPARED, "analyze must succeed before refactor");
  if (!h->engine) return fail(h, BDLU_BACKEND_UNAVAILABLE, "analysis was run without a device (analysis_only)");
  if (!vals || nnz != h->coo.nnz()) return fail(h, BDLU_INVALID_INDEX, "value count does not match the analysed pattern");
  return BDLU_OK;
}

int bdlu_refactor_values_on(bdlu_solver* h, const double* vals, int64_t nnz, cudaStream_t stream, bool checked) {
  if (const int st = refactor_checks(h, vals, nnz)) return st;
  if (const int st = stage_host_values(h, vals, nnz, stream, checked)) return st;
  return do_factor(h, stream, h->reuse_pivots);
}

// Device upload of an analysed handle whose engine was released (or never
// built): plan, tables and values; the next factor pivots in full.
int bdlu_device_restore(bdlu_solver* h) {
  if (!h->decomposed) return fail(h, BDLU_NOT_PREPARED, "analyze must succeed before a device upload");
  if (h->engine) return BDLU_OK;
  if (h->host_vals_stale) return fail(h, BDLU_BACKEND_UNAVAILABLE, "values were not saved before the device release");
  try {
    const bdlu::Plan plan = bdlu::build_plan(h->coo, h->dec, bdlu::small_unit_max(), &h->gp);
    h->engine = std::make_unique<bdlu::Engine>();
    std::string err;
    if (!h->engine->upload(plan, h->dec, h->coo, err)) {
      h->engine.reset();
      return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
    }
    h->engine->set_pattern_key(h->sig);
    if (const int st = upload_values(h, h->coo.val.data(), false, nullptr)) {
      h->engine.reset();
      return st;
    }
  } catch (const std::exception& e) {
    h->engine.reset();
    return fail(h, BDLU_ANALYSIS_FAILED, e.what());
  }
  h->factored = false;
  h->exported = false;
  return BDLU_OK;
}

void bdlu_device_release(bdlu_solver* h) {
  // Keep the current values on the host for the next upload.
  if (bdlu_sync_host_values(h) != BDLU_OK) h->decomposed = false;
  h->engine.reset();
  h->factored = false;
  h->exported = false;
}

bool bdlu_engine_ready(const bdlu_solver* h) { return h && h->engine != nullptr; }

int64_t bdlu_device_bytes(const bdlu_solver* h) {
  return (h && h->engine) ? static_cast<int64_t>(h->engine->device_bytes()) : 0;
}

int bdlu_solve_on(bdlu_solver* h, double* B, int32_t ldb, int32_t nrhs, cudaStream_t stream) {
  return bdlu_solve_checked_on(h, B, ldb, nrhs, stream, false);
}

int bdlu_refactor_values_device_on(bdlu_solver* h, const double* d_vals, int64_t nnz, cudaStream_t stream) {
  if (const int st = refactor_checks(h, d_vals, nnz)) return st;
  if (const int st = upload_values(h, d_vals, true, stream)) return st;
  h->host_vals_stale = true;
  return do_factor(h, stream, h->reuse_pivots);
}

int bdlu_solve_checked_on(bdlu_solver* h, double* B, int32_t ldb, int32_t nrhs, cudaStream_t stream, bool device,
                          bool checked) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (!h->factored) return fail(h, BDLU_NOT_PREPARED, "factor must succeed before solve");
  if (!B || nrhs < 1 || ldb < h->n) return fail(h, BDLU_INVALID_RHS, "right-hand side size does not match matrix dimension");
  if (!device && !checked)
    for (int32_t k = 0; k < nrhs; ++k)
      if (!all_finite(B + static_cast<size_t>(k) * ldb, h->n))
        return fail(h, BDLU_NON_FINITE_VALUE, "right-hand side contains NaN or infinity");
  std::string err;
  // The right-hand sides go to the engine's buffer.  A factor redone below
  // may re-plan the pattern (a sparse-LU unit moved to the dense route),
  // which replaces every engine buffer, so each redo stages them again from
  // B, which holds them until the solution is copied out.
  double* d_B = nullptr;
  cudaError_t e = cudaSuccess;
  auto stage = [&]() -> int {
    d_B = h->engine->rhs_buffer(nrhs, err);
    if (!d_B) return fail(h, BDLU_SOLVE_FAILED, err);
    e = cudaMemcpy2DAsync(d_B, static_cast<size_t>(h->n) * sizeof(double), B, static_cast<size_t>(ldb) * sizeof(double),
                          static_cast<size_t>(h->n) * sizeof(double), static_cast<size_t>(nrhs),
                          device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return fail(h, BDLU_SOLVE_FAILED, std::string("rhs upload: ") + cudaGetErrorString(e));
    return BDLU_OK;
  };
  if (const int st = stage()) return st;
  const int iters = refine_iters_for(h);
  auto relres = [](const bdlu::SolveResidual& q) {
    const double denom = q.a_inf * q.x_inf + q.b_inf;
    return denom > 0.0 ? q.resid_inf / denom : q.resid_inf;
  };
  bdlu::SolveResidual r{};
  // Solve from the stored right-hand sides and read the residual.
  auto solve_once = [&]() -> int {
    if (!h->engine->solve_async(d_B, h->n, nrhs, iters, stream, err)) return fail(h, BDLU_SOLVE_FAILED, err);
    if (!h->engine->last_residual(stream, r, err)) return fail(h, BDLU_SOLVE_FAILED, err);
    h->last_residual = relres(r);
    return BDLU_OK;
  };
  auto redo_factor = [&]() -> int {
    if (const int st = do_factor(h, stream, false)) return st;
    return stage();
  };
  if (const int st = solve_once()) return st;
  // A zero pivot met by a refactor queued without its own status wait
  // surfaces here; a refactor that reused the pivot order of large blocks
  // is then redone with pivoting, and one whose sparse-LU unit failed its
  // pivot test is redone with that unit on the dense route.
  int fst = h->engine->factor_status(stream, err);
  if (fst == 1 || fst < 0 || (fst == 2 && !h->engine->last_factor_reused())) {
    h->factored = false;
    return fail(h, fst < 0 ? BDLU_BACKEND_UNAVAILABLE : BDLU_FACTORIZATION_FAILED, err);
  }
  if (fst == 2 || fst == 3) {
    if (const int st = redo_factor()) return st;
    if (const int st = solve_once()) return st;
  }
  int32_t steps = 0;
  if (h->mixed) {
    // Mixed route: FP64 refinement until the residual bound; a level whose
    // refinement stagnates (less than a halving per step after two steps, or
    // kMaxRefine steps) is replaced by the next one (TF32 -> 3xTF32 -> FP64)
    // for this and later factorisations, and the system is factored again.
    constexpr int kMaxRefine = 30;
    while (true) {
      double prev = h->last_residual;
      int k = 0;
      while (!(h->last_residual <= kReuseResidualLimit) && k < kMaxRefine) {
        if (!h->engine->refine_async(d_B, h->n, nrhs, stream, err)) return fail(h, BDLU_SOLVE_FAILED, err);
        if (!h->engine->last_residual(stream, r, err)) return fail(h, BDLU_SOLVE_FAILED, err);
        h->last_residual = relres(r);
        ++k;
        if (k >= 2 && !(h->last_residual < 0.5 * prev)) break;
        prev = h->last_residual;
      }
      steps += k;
      // Every refinement step costs a solve: a level that needed more than
      // kSlowRefine steps is replaced for the next factorisation as well.
      constexpr int kSlowRefine = 4;
      if (h->last_residual <= kReuseResidualLimit && k > kSlowRefine && h->prec_level != 0)
        h->prec_level = (h->prec_level == 1) ? 2 : 0;
      if (h->last_residual <= kReuseResidualLimit || h->prec_level == 0) break;
      h->prec_level = (h->prec_level == 1) ? 2 : 0;
      if (const int st = do_factor(h, stream, h->engine->last_factor_reused())) return st;
      if (const int st = stage()) return st;
      if (const int st = solve_once()) return st;
    }
  }
  // A refactor that reused the pivot order and still misses the bound is
  // redone with pivoting.
  if (h->engine->last_factor_reused() && !(h->last_residual <= kReuseResidualLimit)) {
    if (const int st = redo_factor()) return st;
    if (const int st = solve_once()) return st;
  }
  e = cudaMemcpy2DAsync(B, static_cast<size_t>(ldb) * sizeof(double), d_B, static_cast<size_t>(h->n) * sizeof(double),
                        static_cast<size_t>(h->n) * sizeof(double), static_cast<size_t>(nrhs),
                        device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = h->engine->wait(stream);
  if (e != cudaSuccess) return fail(h, BDLU_SOLVE_FAILED, std::string("solution download: ") + cudaGetErrorString(e));
  h->last_refine = iters + steps;
  if (!std::isfinite(h->last_residual)) return fail(h, BDLU_SOLVE_FAILED, "block solve produced a non-finite solution");
  return BDLU_OK;
}

extern "C" {

bdlu_solver* bdlu_create(void) {
  try {
    return new bdlu_solver();
  } catch (...) {
    return nullptr;
  }
}

void bdlu_destroy(bdlu_solver* h) { delete h; }

int bdlu_set_coo(bdlu_solver* h, const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
                 int32_t dimension) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (dimension < -1) return fail(h, BDLU_INVALID_DIMENSION, "matrix dimension must be non-negative");
  if (nnz < 0 || (nnz > 0 && (!rows || !cols || !vals))) return fail(h, BDLU_INVALID_INDEX, "invalid COO arrays");
  try {
    h->engine.reset();
    h->host_vals_stale = false;
    h->in_rows.assign(rows, rows + nnz);
    h->in_cols.assign(cols, cols + nnz);
    h->in_vals.assign(vals, vals + nnz);
    h->coo = bdlu::CanonicalCoo{};
    h->dec = bdlu::Decomposition{};
  } catch (const std::exception& e) {
    return fail(h, BDLU_ANALYSIS_FAILED, e.what());
  }
  // Storage only (solver.cpp:771-774): validation is deferred to analyze.
  h->dimension_hint = dimension;
  h->n = dimension >= 0 ? dimension : -1;
  h->prepared = true;
  h->validated = false;
  h->decomposed = false;
  h->factored = false;
  h->exported = false;
  h->mode = BDLU_MODE_AUTO;
  h->global_route = false;
  h->auto_picked_klu = false;
  return BDLU_OK;
}

int bdlu_analyze(bdlu_solver* h) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (!h->prepared) return fail(h, BDLU_NOT_PREPARED, "set_matrix must be called before analyze");
  if (const int st = ensure_validated(h)) return st;
  return bdlu_analyze_validated(h, pick_mode(), nullptr);
}

int bdlu_factor(bdlu_solver* h) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (!h->decomposed) return fail(h, BDLU_NOT_PREPARED, "analyze must succeed before factor");
  if (!h->engine) return fail(h, BDLU_BACKEND_UNAVAILABLE, "analysis was run without a device (analysis_only)");
  // After refactors the device buffer already holds the current values.
  if (!h->host_vals_stale)
    if (const int st = upload_values(h, h->coo.val.data(), false, nullptr)) return st;
  return do_factor(h, nullptr, false);
}

int bdlu_refactor_values(bdlu_solver* h, const double* vals, int64_t nnz) {
  return bdlu_refactor_values_on(h, vals, nnz, nullptr);
}

int bdlu_refactor_values_device(bdlu_solver* h, const double* d_vals, int64_t nnz, void* stream) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (!h->decomposed) return fail(h, BDLU_NOT_PREPARED, "analyze must succeed before refactor");
  if (!h->engine) return fail(h, BDLU_BACKEND_UNAVAILABLE, "analysis was run without a device (analysis_only)");
  if (!d_vals || nnz != h->coo.nnz()) return fail(h, BDLU_INVALID_INDEX, "value count does not match the analysed pattern");
  auto s = static_cast<cudaStream_t>(stream);
  if (const int st = upload_values(h, d_vals, true, s)) return st;
  h->host_vals_stale = true;
  std::string err;
  // No status wait here, so no schedule trial: the tuned schedule if the
  // pattern has one, else the handle's.
  const int tuned = schedule_tunable(h) ? Tuner::get().refactor_schedule(h->sig) : -1;
  h->engine->set_precision(h->mixed ? h->prec_level : 0);
  h->engine->set_lu_small_width(h->lu_small_threads);
  h->engine->set_blocking_sync(h->blocking_sync);
  h->engine->set_small_mode(h->small_mode);
  h->engine->set_refactor_schedule(tuned >= 0 ? tuned : h->refactor_schedule);
  h->engine->set_wait_limit(h->wait_limit);
  if (!h->engine->factor_async(h->engine->values_buffer(), s, err, h->reuse_pivots))
    return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
  // Zero pivots, and sparse-LU units that fail their pivot test, are reported
  // by the next host-buffer solve, which factors again.
  h->factored = true;
  h->exported = false;
  return BDLU_OK;
}

int bdlu_solve(bdlu_solver* h, double* B, int32_t ldb, int32_t nrhs) { return bdlu_solve_on(h, B, ldb, nrhs, nullptr); }

int bdlu_solve_device(bdlu_solver* h, double* d_B, int32_t ldb, int32_t nrhs, void* stream) {
  if (!h) return BDLU_NOT_PREPARED;
  clear_error(h);
  if (!h->factored) return fail(h, BDLU_NOT_PREPARED, "factor must succeed before solve");
  if (!d_B || nrhs < 1 || ldb < h->n) return fail(h, BDLU_INVALID_RHS, "right-hand side size does not match matrix dimension");
  std::string err;
  const int iters = refine_iters_for(h);
  if (!h->engine->solve_async(d_B, ldb, nrhs, iters, static_cast<cudaStream_t>(stream), err))
    return fail(h, BDLU_SOLVE_FAILED, err);
  h->last_refine = iters;
  return BDLU_OK;
}

int bdlu_refactor_solve(bdlu_solver* h, const double* vals, int64_t nnz, double* B, int32_t ldb, int32_t nrhs) {
  // The factor is queued without its own status wait: the solve reads the
  // status after its first sweep and redoes a refactor whose reused pivot
  // order met a zero pivot (with pivoting), or reports a zero pivot.
  if (const int st = refactor_checks(h, vals, nnz)) return st;
  if (const int st = stage_host_values(h, vals, nnz, nullptr, false)) return st;
  std::string err;
  h->engine->set_precision(h->mixed ? h->prec_level : 0);
  h->engine->set_lu_small_width(h->lu_small_threads);
  h->engine->set_blocking_sync(h->blocking_sync);
  h->engine->set_small_mode(h->small_mode);
  const int32_t sched = schedule_for(h);
  h->engine->set_refactor_schedule(sched);
  h->engine->set_wait_limit(h->wait_limit);
  if (!h->engine->factor_async(h->engine->values_buffer(), nullptr, err, h->reuse_pivots))
    return fail(h, BDLU_BACKEND_UNAVAILABLE, err);
  h->factored = true;
  h->exported = false;
  const int st = bdlu_solve(h, B, ldb, nrhs);
  if (st == BDLU_OK) record_schedule(h, sched);
  return st;
}

int bdlu_last_error(const bdlu_solver* h, char* buf, int64_t len) {
  if (!h) return BDLU_NOT_PREPARED;
  if (buf && len > 0) {
    const size_t k = std::min<size_t>(static_cast<size_t>(len - 1), h->last_message.size());
    std::memcpy(buf, h->last_message.data(), k);
    buf[k] = '\0';
  }
  return h->last_error;
}

int32_t bdlu_n(const bdlu_solver* h) { return h ? h->n : 0; }

const char* bdlu_selected_mode(const bdlu_solver* h) {
  return (h && (h->global_route || h->auto_picked_klu)) ? "KLU" : "BLOCK";
}

int64_t bdlu_canonical_pattern(const bdlu_solver* h, int32_t* rows, int32_t* cols) {
  if (!h || !h->validated) return 0;
  const int64_t nnz = h->coo.nnz();
  if (rows) std::memcpy(rows, h->coo.row.data(), static_cast<size_t>(nnz) * sizeof(int32_t));
  if (cols) std::memcpy(cols, h->coo.col.data(), static_cast<size_t>(nnz) * sizeof(int32_t));
  return nnz;
}

int64_t bdlu_tuner_report(char* buf, int64_t len) {
  try {
    const std::string r = bdlu::Tuner::get().report();
    if (buf && len > 0) {
      const size_t k = std::min<size_t>(static_cast<size_t>(len - 1), r.size());
      std::memcpy(buf, r.data(), k);
      buf[k] = '\0';
    }
    return static_cast<int64_t>(r.size()) + 1;
  } catch (...) {
    return -1;
  }
}

int bdlu_matrix_signatures(const bdlu_solver* h, uint64_t* sigs) {
  if (!h || !sigs || !h->decomposed) return BDLU_NOT_PREPARED;
  sigs[0] = h->sig;
  sigs[1] = h->sig2;
  sigs[2] = h->value_sig;
  return BDLU_OK;
}

int bdlu_get_stats(const bdlu_solver* h, bdlu_stats* out) {
  if (!h || !out) return BDLU_NOT_PREPARED;
  std::memset(out, 0, sizeof(*out));
  out->n = h->n;
  out->nnz = h->coo.nnz();
  out->nblocks = h->dec.nblocks;
  out->nblocks_raw = h->dec.nblocks_raw;
  out->max_level = h->dec.max_level;
  for (int32_t b = 0; b < h->dec.nblocks; ++b) out->max_block = std::max(out->max_block, h->dec.R[static_cast<size_t>(b) + 1] - h->dec.R[static_cast<size_t>(b)]);
  out->nnz_offdiag = h->dec.off_ptr.empty() ? 0 : h->dec.off_ptr.back();
  out->refine_iters = h->last_refine;
  out->precision = h->engine ? h->engine->precision() : 0;
  out->residual_inf = h->last_residual;
  if (h->engine) {
    auto* e = const_cast<bdlu::Engine*>(h->engine.get());
    out->dense_entries = e->plan().dense_entries;
    out->factor_flops = e->plan().factor_flops;
    out->unit_levels = e->plan().umax_level + 1;
    out->nunits = e->plan().nunits;
    out->max_unit = e->plan().max_unit;
    out->factor_launches = e->launches_factor_;
    out->solve_launches = e->launches_solve_;
    out->last_factor_ms = e->last_factor_ms();
    out->last_solve_ms = e->last_solve_ms();
  }
  return BDLU_OK;
}

int bdlu_phase_times(bdlu_solver* h, double* ms, int32_t cap) {
  if (!h || !h->engine) return 0;
  float f[bdlu::Engine::kPhases];
  h->engine->phase_ms(f);
  for (int32_t i = 0; i < cap && i < bdlu::Engine::kPhases; ++i) ms[i] = f[i];
  return bdlu::Engine::kPhases;
}

int bdlu_set_option(bdlu_solver* h, const char* key, double value) {
  if (!h || !key) return BDLU_INVALID_DIMENSION;
  const std::string k(key);
  if (k == "refine_iters") {
    h->refine_iters = static_cast<int32_t>(value);
    return BDLU_OK;
  }
  if (k == "refactor_pivoting") {
    h->reuse_pivots = value == 0.0;
    return BDLU_OK;
  }
  if (k == "refactor_schedule") {
    if (value != 0.0 && value != 1.0) return BDLU_INVALID_DIMENSION;
    h->refactor_schedule = static_cast<int32_t>(value);
    h->schedule_user_set = true;
    if (h->engine) h->engine->set_refactor_schedule(h->refactor_schedule);
    return BDLU_OK;
  }
  if (k == "lu_small_threads") {
    // Launch width of the shared-memory LU: 0 the autotuner's choice (or the
    // default rule), 1 one thread per row with the rows in registers (units
    // up to 96 rows), 32 one warp per unit (units up to 64 rows), 64 / 128 /
    // 256 threads per unit (units up to that many rows).  All give the same
    // factors; a width a bucket cannot take falls back to the tuned one.
    if (value != 0.0 && value != 1.0 && value != 32.0 && value != 64.0 && value != 128.0 && value != 256.0)
      return BDLU_INVALID_DIMENSION;
    h->lu_small_threads = static_cast<int32_t>(value);
    return BDLU_OK;
  }
  if (k == "blocking_sync") {
    // 1: waits for the device sleep on blocking-sync events instead of
    // spinning (for processes where many threads wait at once).
    h->blocking_sync = value != 0.0;
    if (h->engine) h->engine->set_blocking_sync(h->blocking_sync);
    return BDLU_OK;
  }
  if (k == "programmatic_launch") {
    // 1 (default): from the second solve level on, each level's launch is a
    // programmatic dependent of the previous one (its factor staging and
    // launch overlap the previous level).  0: plain stream order, for
    // processes that run many solves on many streams at once.
    if (value != 0.0 && value != 1.0) return BDLU_INVALID_DIMENSION;
    h->programmatic_launch = value != 0.0;
    if (h->engine) h->engine->set_programmatic_launch(h->programmatic_launch);
    return BDLU_OK;
  }
  if (k == "small_launch") {
    // Small units: -1 the autotuner's choice, 0 one launch per size bucket,
    // 1 one persistent launch over a task queue.  Same factors either way.
    if (value != -1.0 && value != 0.0 && value != 1.0) return BDLU_INVALID_DIMENSION;
    h->small_mode = static_cast<int32_t>(value);
    return BDLU_OK;
  }
  if (k == "wait_limit") {
    // Polls a bounded wait between tiles makes before the solve (or the tile
    // graph refactor) gives up with an error status; 0 restores the default
    // (about half a second).  Shorter limits exist to exercise that error
    // path on purpose.
    if (value < 0.0 || value > 2147483647.0) return BDLU_INVALID_DIMENSION;
    h->wait_limit = static_cast<int32_t>(value);
    if (h->engine) h->engine->set_wait_limit(h->wait_limit);
    return BDLU_OK;
  }
  if (k == "sparse_lu") {
    // Sparse-LU route for diagonal blocks, from the next analyze: 0 off,
    // 1 the reference's route (USERALGO_SPARSE_LU_KERNEL=gp: every block of
    // USERALGO_DENSE_BLOCK_MAX < m <= USERALGO_GP_MAX_N rows), 2 only blocks
    // whose no-pivot fill is at most "sparse_fill_max" of m^2.
    if (value != 0.0 && value != 1.0 && value != 2.0) return BDLU_INVALID_DIMENSION;
    h->sparse_lu_opt = static_cast<int32_t>(value);
    return BDLU_OK;
  }
  if (k == "sparse_fill_max") {
    if (!(value > 0.0 && value <= 1.0)) return BDLU_INVALID_DIMENSION;
    h->sparse_fill_max = value;
    return BDLU_OK;
  }
  if (k == "sparse_max_n") {
    if (!(value >= 1.0 && value <= 2147483647.0)) return BDLU_INVALID_DIMENSION;
    h->sparse_max_n = static_cast<int32_t>(value);
    return BDLU_OK;
  }
  if (k == "analysis_only") {
    h->analysis_only = value != 0.0;
    return BDLU_OK;
  }
  if (k == "precision") {
    // 0: FP64 throughout; 1: mixed (tensor-core trailing updates of large
    // blocks, FP64 refinement, ladder TF32 -> 3xTF32 -> FP64); 2: mixed with
    // the ladder starting at 3xTF32.  Takes effect at the next factor.
    if (value != 0.0 && value != 1.0 && value != 2.0) return BDLU_INVALID_DIMENSION;
    h->mixed = value != 0.0;
    h->prec_level = value == 2.0 ? 2 : 1;
    return BDLU_OK;
  }
  return BDLU_INVALID_DIMENSION;
}

int32_t bdlu_get_unit_routes(const bdlu_solver* h, int32_t* start, int32_t* route, int32_t* reason, int64_t* lu_nnz,
                             int32_t cap) {
  if (!h || !h->decomposed || !h->engine) return -BDLU_NOT_PREPARED;
  const bdlu::Plan& p = h->engine->plan();
  for (int32_t u = 0; u < p.nunits && u < cap; ++u) {
    const int32_t s0 = p.ustart[static_cast<size_t>(u)];
    if (start) start[u] = s0;
    if (route) route[u] = p.ukind[static_cast<size_t>(u)];
    if (reason) {
      int32_t r = p.ukind[static_cast<size_t>(u)] == bdlu::kUnitSparse ? 0 : -1;
      for (const auto& e : h->gp_rejected_reason)
        if (e.first == s0) r = e.second;
      if (std::find(p.gp_symbolic_rejected.begin(), p.gp_symbolic_rejected.end(), u) != p.gp_symbolic_rejected.end())
        r = 5;
      reason[u] = r;
    }
    if (lu_nnz) {
      const int64_t m = p.ustart[static_cast<size_t>(u) + 1] - s0;
      const int32_t g = p.gp_index.empty() ? -1 : p.gp_index[static_cast<size_t>(u)];
      lu_nnz[u] = g >= 0 ? static_cast<int64_t>(p.gp_cptr[static_cast<size_t>(p.gp_col0[static_cast<size_t>(g) + 1])] -
                                                p.gp_cptr[static_cast<size_t>(p.gp_col0[static_cast<size_t>(g)])])
                         : m * m;
    }
  }
  return p.nunits;
}

int32_t bdlu_btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q, int32_t* R,
                       int32_t* nmatch) {
  try {
    return bdlu::btf_order(n, Ap, Ai, P, Q, R, nmatch);
  } catch (...) {
    return -1;
  }
}

int32_t bdlu_merge_block_boundaries(const int32_t* R, int32_t nR, int32_t n, int32_t merge_max, int32_t* Rout) {
  try {
    const std::vector<int32_t> in(R, R + nR);
    const std::vector<int32_t> out = bdlu::merge_block_boundaries(in, n, merge_max);
    if (Rout) std::memcpy(Rout, out.data(), std::min<size_t>(out.size(), static_cast<size_t>(nR)) * sizeof(int32_t));
    return static_cast<int32_t>(out.size());
  } catch (...) {
    return -1;
  }
}

int bdlu_get_decomposition(const bdlu_solver* h, int32_t* P, int32_t* Q, int32_t* R, int32_t* off_ptr, int32_t* off_col,
                           int32_t* off_src, int32_t* level) {
  if (!h || !h->decomposed) return BDLU_NOT_PREPARED;
  const auto& d = h->dec;
  auto cp = [](int32_t* dst, const std::vector<int32_t>& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int32_t));
  };
  cp(P, d.P);
  cp(Q, d.Q);
  cp(R, d.R);
  cp(off_ptr, d.off_ptr);
  cp(off_col, d.off_col);
  cp(off_src, d.off_src);
  cp(level, d.level);
  return BDLU_OK;
}

}  // extern "C"
