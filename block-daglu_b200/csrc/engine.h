// Device engine: per-pattern device plan, numeric factor and solve on the GPU.
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "gp.h"
#include "plan.h"

namespace bdlu {

// Width code of the row-per-thread small-unit LU (one CTA of 64 or 96
// threads per unit, each thread one row in registers).
constexpr int kLuRowsWidth = 1;


// Device-side view of a plan (all pointers device memory owned by Engine).
struct DevPlan {
  int32_t n;
  int32_t nunits;
  int64_t nnz;
  const int32_t* P;
  const int32_t* Q;
  const int32_t* ustart;
  const int64_t* lu_off;
  const int64_t* dent_ptr;
  const int32_t* dent_pos;
  const int32_t* dent_src;
  const int32_t* sdiag_src;
  const int32_t* cpl_ptr;
  const int32_t* cpl_col;
  const int32_t* cpl_src;
  const int32_t* csr_ptr;
  const int32_t* csr_col;
  const int32_t* step_unit;
  const int32_t* step_trsm_pref;
  const int32_t* step_gemm_pref;
  const int32_t* rstep_unit;
  const int32_t* rstep_strip_pref;
  const int32_t* rstep_ga_pref;
  const int32_t* rstep_gb_pref;
  double* dscratch;  // refactor: factored diagonal block per active unit of a step
  double* lu;
  int32_t* piv;
  int32_t* lperm;   // final row order of each large unit (local indices)
  int32_t* liperm;  // its inverse
  double* sdiag;
  double* cpl_val;
  int32_t* status;  // [0] failure code (0 = ok), [1] failing unit
  // Polls a bounded wait between tiles makes before it gives up (solve
  // sweeps of large units, tile-graph refactor): kWaitLimitDefault, or a
  // shorter limit set through the "wait_limit" option to make waits run out
  // on purpose in tests.
  int32_t wait_limit;
};

constexpr int32_t kWaitLimitDefault = 1 << 22;  // ~0.5 s with the poll back-off

struct SolveResidual {
  double resid_inf;   // |b - Ax|_inf
  double b_inf;
  double x_inf;
  double a_inf;       // max row sum |A|
};

class Engine {
 public:
  Engine();
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Uploads the pattern: plan tables, permutations, canonical column indices.
  // Returns false and sets `err` on a CUDA error.
  bool upload(const Plan& plan, const Decomposition& dec, const CanonicalCoo& a, std::string& err);

  // Device bytes held by this engine (plan tables, LU arena, values, work).
  size_t device_bytes() const;

  // Enqueues the numeric factor of every unit from canonical-order values
  // already on the device (d_vals, nnz entries).  reuse_pivots: large units
  // keep the row order of the last full factorisation (no pivot search);
  // ignored until one full factorisation has succeeded.
  bool factor_async(const double* d_vals, cudaStream_t stream, std::string& err, bool reuse_pivots = false);
  // Waits for the factor.  Returns 0 (ok), 1 (zero pivot: the matrix is
  // singular), 2 (a reused pivot order met a zero pivot: factor again with
  // pivoting) or 3 (a sparse-LU unit failed its pivot test: re-plan it as a
  // dense unit, see sparse_rejections); -1 on a CUDA error.
  int factor_status(cudaStream_t stream, std::string& err);
  // After factor_status returned 3: the sparse units whose pivot test failed
  // (unit ids) and the reasons (gp_dev.h).
  bool sparse_rejections(std::vector<int32_t>& units, std::vector<int32_t>& reasons, std::string& err);
  bool last_factor_reused() const { return last_reuse_; }

  // Enqueues X = A^{-1} B for nrhs columns (column-major, ld ldb, in place),
  // followed by `refine_iters` FP64 refinement steps and the residual norms.
  bool solve_async(double* d_B, int32_t ldb, int32_t nrhs, int32_t refine_iters, cudaStream_t stream,
                   std::string& err);
  // One FP64 refinement step on the solution in d_B (from the last solve):
  // r = b - A x, x += A^{-1} r with the current factors; then the residual
  // norms of the new x (read by last_residual).
  bool refine_async(double* d_B, int32_t ldb, int32_t nrhs, cudaStream_t stream, std::string& err);
  // Trailing-update arithmetic of large blocks for the next factor:
  // 0 FP64, 1 TF32 tensor cores, 2 3xTF32.
  void set_precision(int32_t prec) { prec_ = prec; }
  int32_t precision() const { return prec_; }
  // Schedule of the FP64 value-only refactor of large units: 0 the step
  // chain (panel and update launches on two graph branches), 1 one
  // persistent kernel over the tile task graph (when the plan has one).
  void set_refactor_schedule(int32_t s) { schedule_ = s; }
  // Launch width of the shared-memory LU forced for this engine (32: one
  // warp per unit; kLuRowsWidth: one thread per row, rows in registers;
  // 64, 128, 256: threads per CTA; 0: the autotuner's).
  void set_lu_small_width(int32_t t) { forced_lu_width_ = t; }
  // Small units as per-bucket launches (0) or one persistent launch over a
  // task queue (1); -1: the autotuner's choice for the pattern.
  void set_small_mode(int32_t m) { forced_small_mode_ = m; }
  // Pivot test of the sparse-LU units (gp.h): diagonal preference, tiny
  // pivot and smallest pivot thresholds.
  void set_sparse_tests(double diag_tol, double pivot_tol, double min_abs_diag) {
    gp_.diag_tol = diag_tol;
    gp_.pivot_tol = pivot_tol;
    gp_.min_abs_diag = min_abs_diag;
  }
  // Pattern signature under which the autotuner keeps this engine's choices.
  void set_pattern_key(uint64_t k) { pattern_key_ = k; }
  // Bound of the waits between tiles (polls; <= 0 restores the default).
  // Captured graphs hold the old bound, so they are dropped.
  void set_wait_limit(int32_t polls) {
    const int32_t v = polls > 0 ? polls : kWaitLimitDefault;
    if (v == dp_.wait_limit) return;
    dp_.wait_limit = v;
    gp_.wait_limit = v;
    drop_graphs();
  }
  // Waits for `stream`: spinning (cudaStreamSynchronize), or, with
  // set_blocking_sync(true), sleeping on a blocking-sync event (many host
  // threads waiting at once, as the serving loop's workers do).
  cudaError_t wait(cudaStream_t stream);
  void set_blocking_sync(bool b) { blocking_sync_ = b; }
  // Solve levels launched as programmatic dependents of the previous level
  // (on by default).  Off where many streams share the GPU: a dependent's
  // CTAs hold their SM slots while they wait for the previous level, slots
  // the other streams' ready work could use.  Captured graphs are dropped.
  void set_programmatic_launch(bool on) {
    if (on == pdl_) return;
    pdl_ = on;
    drop_graphs();
  }
  // Residual norms of the last solve (synchronises the stream), worst column.
  bool last_residual(cudaStream_t stream, SolveResidual& out, std::string& err);

  double* values_buffer() { return d_vals_; }
  // Device buffer of nnz doubles for host values in flight (allocated at the
  // first call; counted by device_bytes).
  double* value_staging(std::string& err);
  // Device buffer of n * nrhs doubles for host-API right-hand sides.
  double* rhs_buffer(int32_t nrhs, std::string& err);
  int64_t nnz() const { return plan_.nnz; }
  int32_t n() const { return plan_.n; }
  const Plan& plan() const { return plan_; }
  float last_factor_ms();
  float last_solve_ms();
  // Device time of the last factor's and solve's phases, in order: value
  // gather, shared-memory LU, blocked LU of large units, first solve sweep,
  // refinement + residual.  Synchronises on the recorded events.
  static constexpr int kPhases = 5;
  void phase_ms(float out[kPhases]);

  // Copies a unit's LU (column-major m*m; a sparse unit's factor expanded,
  // with identity pivots) and pivots to the host.
  bool download_unit(int32_t u, std::vector<double>& lu, std::vector<int32_t>& piv, double& scalar,
                     std::string& err);

 private:
  void release();
  bool ensure_work(int32_t nrhs, std::string& err);
  // Shared-memory LU of one size bucket with `threads` per CTA; the width the
  // autotuner chose for a bucket (or the default rule); the tuning itself.
  void launch_lu_small(int threads, int32_t units, int32_t mb, cudaStream_t st, const double* d_vals,
                       const int32_t* list);
  int lu_small_width(int32_t mb) const;
  cudaError_t tune_lu_small(const double* d_vals, cudaStream_t stream);
  cudaError_t launch_small_buckets(const double* d_vals, cudaStream_t stream);
  cudaError_t launch_small_queue(const double* d_vals, cudaStream_t stream);
  int small_mode() const;
  cudaError_t tune_small_mode(const double* d_vals, cudaStream_t stream);
  // Page-locked words for status and residual-norm read-backs: 8 int32
  // status words, then kReadbackNorms norms.
  static constexpr size_t kReadbackNorms = 4 * 64;
  static constexpr size_t kReadbackBytes = 32 + kReadbackNorms * sizeof(unsigned long long);
  char* readback_ = nullptr;
  bool blocking_sync_ = false;
  bool pdl_ = true;
  cudaEvent_t wait_ev_ = nullptr;
  bool readback_pinned_ = true;
  int32_t forced_small_mode_ = -1;
  uint64_t pattern_key_ = 0;
  const int32_t* d_qunits_ = nullptr;  // small units, largest first
  const int32_t* d_qtasks_ = nullptr;  // (first, count) per task
  int32_t* d_qticket_ = nullptr;
  int32_t queue_tasks_ = 0;
  int queue_grid_ = 1;
  size_t queue_smem_ = 0;
  void solve_core(const double* rhs, int32_t ldr, double* xp, const int32_t* nrhs, bool wide, cudaStream_t stream);
  void refine_core(double* d_B, int32_t ldb, int32_t nrhs, cudaStream_t stream);
  int32_t prec_ = 0;
  int32_t forced_lu_width_ = 0;
  int32_t reuse_prec_ = 0;
  int32_t schedule_ = 0;
  int32_t reuse_schedule_ = 0;
  const int32_t* d_rtask_ = nullptr;  // task list of the tile-graph refactor (4 words per task)
  int32_t* d_rwords_ = nullptr;       // its ticket and tile version words

  Plan plan_;
  DevPlan dp_{};
  // Sparse-LU units (gp_dev.h): device tables, their solve lists by level,
  // and the stream their factor runs on beside the dense units.
  GpDev gp_{};
  const int32_t* lvl_sparse_ = nullptr;
  cudaStream_t gp_stream_ = nullptr;
  cudaEvent_t gp_ev_[2] = {nullptr, nullptr};
  std::vector<std::pair<void*, size_t>> allocs_;  // device allocations and their bytes
  double* d_vals_ = nullptr;
  double* d_vals_stage_ = nullptr;
  int32_t* d_status_ = nullptr;
  // Solve work space, grown to the largest nrhs seen.
  int32_t work_nrhs_ = 0;
  double* d_b0_ = nullptr;
  double* d_xp_ = nullptr;
  double* d_r_ = nullptr;
  double* d_rhs_ = nullptr;
  unsigned long long* d_norms_ = nullptr;  // 4 per rhs
  int32_t last_nrhs_ = 0;
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  // Phase boundaries: factor start, after gather, after small LU, factor end
  // (ev_[0..1] reuse), solve start, after first sweep, solve end.
  cudaEvent_t pev_[8] = {};
  bool factor_timed_ = false, solve_timed_ = false;
  const int32_t* small_list_ = nullptr;
  const int32_t* large_list_ = nullptr;
  const int32_t* lvl_scalar_ = nullptr;
  const int32_t* lvl_dense_ = nullptr;
  const int32_t* lvl_large_ = nullptr;
  const int32_t* lvl_large_tile0_ = nullptr;
  int32_t* d_sync_ = nullptr;  // tickets and ready flags of the large-unit tile solves
  int32_t sync_words_ = 0;
  int num_sms_ = 148;
  // CUDA graphs of the launch sequences that repeat unchanged: the solve
  // sweep (per nrhs and work buffers) and the refactor of large units with
  // the stored pivot order.  Captured on cap_stream_, launched on the
  // caller's stream.
  cudaStream_t cap_stream_ = nullptr;
  cudaStream_t cap_stream2_ = nullptr;  // second branch of the refactor graph
  cudaEvent_t fork_ev_[2] = {nullptr, nullptr};
  // Auxiliary streams for the small-unit factor buckets.
  static constexpr int kAux = 4;
  cudaStream_t aux_[kAux] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t aux_ev_[kAux] = {nullptr, nullptr, nullptr, nullptr};
  // Solve-sweep graphs (tile kernels 8 and 16 wide), valid for the work
  // buffers they were captured on.
  cudaGraphExec_t solve_exec_[2] = {nullptr, nullptr};
  int32_t solve_exec_launches_[2] = {0, 0};
  const double* solve_exec_b0_ = nullptr;
  int32_t* d_nrhs_ = nullptr;  // right-hand-side count read by the sweep's kernels
  cudaGraphExec_t reuse_exec_ = nullptr;
  int32_t reuse_launches_ = 0;
  void drop_graphs();
  bool have_pivots_ = false;  // a full factorisation of this pattern succeeded
  bool last_reuse_ = false;

 public:
  // Kernel launches enqueued by the last factor / solve.
  int32_t launches_factor_ = 0;
  int32_t launches_solve_ = 0;
};

// Largest unit the shared-memory LU kernel takes on this device.
int32_t small_unit_max();

}  // namespace bdlu
