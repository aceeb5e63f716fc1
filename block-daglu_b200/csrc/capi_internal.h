// Internal state behind the opaque bdlu_solver handle (include/bdlu.h).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "analysis.h"
#include "bdlu.h"
#include "engine.h"
#include "gp.h"

struct bdlu_solver {
  // Stage flags (solver.h:86-90).
  bool prepared = false;
  bool validated = false;
  bool decomposed = false;
  bool factored = false;
  int32_t dimension_hint = -1;
  int32_t n = 0;
  std::vector<int32_t> in_rows, in_cols;
  std::vector<double> in_vals;
  bdlu::CanonicalCoo coo;
  uint64_t sig = 0, sig2 = 0, value_sig = 0;
  int mode = BDLU_MODE_AUTO;
  bool global_route = false;  // "KLU": one block, no BTF
  // AUTO's route decision (solver.cpp:846-861, auto_choose_block): reported
  // by selected_mode() like the reference's; the numerics stay
  // block-structured either way.
  bool auto_picked_klu = false;
  bdlu::Decomposition dec;
  std::unique_ptr<bdlu::Engine> engine;
  // Options.
  int32_t refine_iters = -1;  // -1: REFINE_ITERS env, else 0
  bool analysis_only = false; // host analysis without device upload (inspection, CPU tests)
  bool reuse_pivots = true;   // value-only refactors keep the pivot order of large blocks
  bool mixed = false;         // "precision" = 1: tensor-core updates + FP64 refinement
  int32_t prec_level = 1;     // mixed route's current level: 1 TF32, 2 3xTF32, 0 FP64 (sticky)
  int32_t refactor_schedule = 0;  // 0 step chain, 1 tile task graph (Engine::set_refactor_schedule)
  bool schedule_user_set = false; // refactor_schedule set by the caller: no autotuning
  // Autotuning of the refactor schedule (tuner.h): trial refactors run
  // chain, graph, chain, graph; the second time of each decides.
  int32_t sched_trials = 0;
  float sched_ms[2] = {0.0f, 0.0f};
  int32_t wait_limit = 0;         // polls of a bounded wait between tiles (0: default; Engine::set_wait_limit)
  int32_t lu_small_threads = 0;   // forced shared-memory LU width (0: autotuned; Engine::set_lu_small_width)
  int32_t small_mode = -1;        // small units per bucket (0) or in one queue launch (1); -1 autotuned
  bool blocking_sync = false;     // waits sleep on blocking-sync events (Engine::set_blocking_sync)
  bool programmatic_launch = true;  // Engine::set_programmatic_launch
  // Sparse-LU route (gp.h): configuration of the current analysis (the
  // environment's, overridden by the options below; -1 = not set) and, by
  // first permuted row, the reasons of units a factor's pivot test sent to
  // the dense route.
  bdlu::GpConfig gp;
  int32_t sparse_lu_opt = -1;
  double sparse_fill_max = -1.0;
  int32_t sparse_max_n = -1;
  std::vector<std::pair<int32_t, int32_t>> gp_rejected_reason;
  // Error state (solver.h:122-123).
  int last_error = BDLU_OK;
  std::string last_message;
  // The device value buffer holds newer values than coo.val (refactors
  // upload without a host copy; bdlu_sync_host_values fetches them when the
  // host copy is read).
  bool host_vals_stale = false;
  // Stats of the last solve.
  int32_t last_refine = 0;
  double last_residual = 0.0;
  // Export cache.
  bool exported = false;
  std::vector<int32_t> exP;          // row order of the exported factorisation
  std::vector<int32_t> l_r, l_c, u_r, u_c;
  std::vector<double> l_v, u_v;
};


inline int bdlu_fail(bdlu_solver* h, int code, std::string msg) {
  h->last_error = code;
  h->last_message = std::move(msg);
  return code;
}

// Analysis of h->coo (validated and canonical; h->n set) under route `mode`
// (a bdlu_mode value); btf, if not null, replaces the BTF ordering step.
// Returns a status code and sets the handle's error.
int bdlu_analyze_validated(bdlu_solver* h, int mode, const bdlu::PrecomputedBtf* btf);

// Host-buffer refactor and solve on a given stream (the C ABI's host-buffer
// calls use the legacy default stream).  Same checks, fallbacks and
// synchronisation as bdlu_refactor_values / bdlu_solve.
// `checked`: the caller has already checked the values for NaN and infinity
// (bdlu_copy_finite while staging them), so no second pass is made.
int bdlu_refactor_values_on(bdlu_solver* h, const double* vals, int64_t nnz, cudaStream_t stream,
                            bool checked = false);
int bdlu_solve_on(bdlu_solver* h, double* B, int32_t ldb, int32_t nrhs, cudaStream_t stream);

// Copies n doubles and reports whether all are finite, in one pass.
bool bdlu_copy_finite(double* dst, const double* src, int64_t n);

// The same two steps with the values and right-hand sides in device memory
// (the serving loop's device-resident requests): no host finiteness check;
// the solve still reads the residual and status and applies the fallbacks,
// and returns with B overwritten on the device and `stream` synchronised.
int bdlu_refactor_values_device_on(bdlu_solver* h, const double* d_vals, int64_t nnz, cudaStream_t stream);
int bdlu_solve_checked_on(bdlu_solver* h, double* B, int32_t ldb, int32_t nrhs, cudaStream_t stream, bool device,
                          bool checked = false);

// Brings coo.val up to date from the engine's value buffer after refactors
// that skipped the host copy (synchronises the device).  Returns a status
// code and sets the handle's error.
int bdlu_sync_host_values(bdlu_solver* h);

// Device residency of an analysed handle: release frees every device
// allocation (the host analysis stays); restore uploads again; bytes is the
// device memory held now.
void bdlu_device_release(bdlu_solver* h);
int bdlu_device_restore(bdlu_solver* h);
int64_t bdlu_device_bytes(const bdlu_solver* h);
bool bdlu_engine_ready(const bdlu_solver* h);

// Builds the export cache (P, L, U in the engine's factor order); returns a
// status code and sets the handle's error on failure.
int bdlu_build_export(bdlu_solver* h);
