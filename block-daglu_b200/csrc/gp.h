// Sparse LU route for diagonal blocks ("GP" units): the reference's opt-in
// Gilbert-Peierls route (blockdaglu/src/gp_lu.cpp:84-306, gate
// ubtf_block_solver.cpp:197-235, dispatch :1749-1773) on the device.
//
// The reference's default gate accepts a sparse factor only if it made no
// row swap and met no tiny pivot.  An accepted factor is therefore an LU
// without pivoting, whose fill pattern depends on the block's pattern alone.
// The host computes that pattern once per pattern (left-looking symbolic
// factorisation: the reach of each column through the columns of L), and the
// device runs the numeric factor over it: each column is formed by a warp in
// a shared-memory work vector from A's column and the L columns in its reach
// (ascending), the pivot test of the reference's step is applied, and the
// column is written back in compressed form.  Every entry receives the
// reference's updates in the reference's order, unfused, so accepted factors
// are bit-identical to gp_lu_factor's.  A unit whose test fails is rejected
// for the whole factorisation (the reference rejects it at the gate) and is
// factored by the dense route instead.
#pragma once

#include <cstdint>
#include <vector>

namespace bdlu {

struct Plan;

struct GpConfig {
  // 0: off (every unit dense).  1: the reference's route: every unit of
  // dense_max < m <= max_n rows (any size above dense_max with force) is
  // tried.  2: only units whose no-pivot fill is at most fill_max of m^2.
  int32_t mode = 0;
  int32_t dense_max = 64;      // USERALGO_DENSE_BLOCK_MAX
  int32_t max_n = 4096;        // USERALGO_GP_MAX_N
  bool force = false;          // USERALGO_GP_FORCE
  double fill_max = 0.01;      // mode 2 (measured: below about 1 % fill the sparse factor beats the dense one)
  double diag_tol = 1e-3;      // USERALGO_GP_DIAG_TOL (diagonal preference)
  double pivot_tol = 1e-12;    // USERALGO_GP_PIVOT_TOL (tiny pivot)
  double min_abs_diag = 1e-12; // USERALGO_GP_MIN_ABS_DIAG
  // Environment settings the device route does not implement (a gate that
  // admits swaps or tiny pivots, row scaling, dropping): the route is off.
  bool unsupported = false;
  // Units (by first permuted row) rejected by an earlier factorisation of
  // this handle: they stay on the dense route.
  std::vector<int32_t> rejected;
};

// USERALGO_SPARSE_LU_KERNEL (= gp) and the USERALGO_GP_* knobs
// (ubtf_block_solver.cpp:87-182), BLOCKDAGLU_* names first.
GpConfig gp_config_from_env();

// Largest sparse unit: the solve keeps four right-hand sides of unknowns and
// a flag per row in shared memory (6144 * 36 bytes, within 227 KB), the
// factor one work vector per warp and a flag per column.
constexpr int32_t kGpMaxRows = 6144;
// Reason a sparse factor records when a bounded wait on another column ran
// out (not a pivot-test reason).
constexpr int32_t kGpReasonSync = 9;

// Symbolic no-pivot LU of one unit from its local entries (row, col, src).
// Returns false if some column has no diagonal entry in the filled pattern
// (the reference's gate rejects such a block: a swap or a zero pivot), or if
// fill_limit >= 0 and the pattern exceeds fill_limit entries (the symbolic
// stops early).  Outputs per column: entries (rows ascending: those above
// the diagonal, the diagonal at dpos[j], then L) and A's entries.
struct GpSymbolic {
  std::vector<int32_t> cptr, row, dpos;  // dpos[j]: index of the diagonal in row[]
  std::vector<int32_t> aptr, arow, asrc;
  int64_t nnz = 0;
  double flops = 0.0;
};
bool gp_symbolic(int32_t m, const std::vector<int32_t>& er, const std::vector<int32_t>& ec,
                 const std::vector<int32_t>& esrc, int64_t fill_limit, GpSymbolic& out);

// Device pointers to the Plan's gp_* tables (plan.h) plus the factor values.
struct GpDev {
  const int32_t* units;
  const int32_t* col0;
  const int32_t* cptr;
  const int32_t* row;
  const int32_t* dpos;
  const int32_t* aptr;
  const int32_t* arow;
  const int32_t* asrc;
  const int32_t* lrp;
  const int32_t* lci;
  const int32_t* lpos;
  const int32_t* urp;
  const int32_t* uci;
  const int32_t* upos;
  double* val;      // gp_nnz factor values, column-compressed
  int32_t* gstat;   // per sparse unit: 0, or the reason its pivot test failed
  int32_t maxm;     // largest sparse unit
  int32_t wait_limit;  // polls of a bounded wait on another column or row (DevPlan::wait_limit)
  double diag_tol;
  double pivot_tol;
  double min_abs_diag;
};

// Appends unit u's symbolic to the plan's sparse-unit tables (the solve's
// row tables included).
void gp_append_unit(Plan& p, int32_t u, const GpSymbolic& s);

}  // namespace bdlu
