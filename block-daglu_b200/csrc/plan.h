// Device execution plan for one sparsity pattern.
//
// The reference factors and solves per merged block (ubtf_block_solver.cpp:
// 1427-1826 and 2220-2555).  A merged block is a run of raw BTF blocks, and
// its partial-pivoting LU is block-diagonal in those raw blocks: rows of a
// later raw block hold structural zeros in an earlier raw block's columns, so
// they are never chosen as pivots and only ever receive x - (+-0)*y updates.
// The diagonal sub-blocks of the merged LU are therefore exactly the LUs of
// the raw blocks, and the merged solve equals a solve over raw blocks.  The
// device works on raw blocks ("units"): they are smaller (less factor work)
// and their DAG is far shallower than the merged one, which the solve
// schedule needs.  The merged partition and DAG are still computed exactly
// (analysis.h) for the API and for parity.
#pragma once

#include <cstdint>
#include <vector>

#include "analysis.h"

namespace bdlu {

enum UnitKind : int32_t {
  kUnitScalar = 0,  // 1x1 raw block: the LU is the diagonal entry
  kUnitSmall = 1,   // dense LU in one CTA's shared memory
  kUnitLarge = 2,   // dense blocked LU across CTAs
  kUnitSparse = 3,  // sparse LU without pivoting over a fixed fill pattern (gp.h)
};

struct Plan {
  int32_t n = 0;
  int64_t nnz = 0;
  int32_t nunits = 0;
  int32_t small_max = 0;  // largest unit handled by the shared-memory kernel
  std::vector<int32_t> ustart;   // nunits + 1
  std::vector<int32_t> ukind;    // nunits
  std::vector<int32_t> unit_of;  // n: unit of each permuted index
  std::vector<int64_t> lu_off;   // nunits: m*m arena slot (column-major for small units,
                                 // row-major for large units), -1 for scalars
  int64_t lu_size = 0;           // doubles
  int64_t lu_large_begin = 0;    // arena range holding the large units
  int64_t lu_large_end = 0;
  // Diagonal-block entries of dense units: local column-major position and
  // canonical source index.
  std::vector<int64_t> dent_ptr;  // nunits + 1
  std::vector<int32_t> dent_pos, dent_src;
  // Scalar units: canonical source of the diagonal entry per permuted row
  // (-1 for rows of dense units, -2 for a missing diagonal).
  std::vector<int32_t> sdiag_src;
  // Coupling CSR in permuted coordinates: every stored entry outside the
  // unit diagonal blocks (all strictly upper at unit level).
  std::vector<int32_t> cpl_ptr, cpl_col, cpl_src;
  // Unit DAG levels (level 0 = no dependencies, solved first).
  std::vector<int32_t> ulevel;
  int32_t umax_level = 0;
  std::vector<int32_t> lvl_scalar_ptr, lvl_scalar;  // permuted rows of scalar units, by level
  std::vector<int32_t> lvl_dense_ptr, lvl_dense;    // small dense unit ids, by level
  std::vector<int32_t> lvl_large_ptr, lvl_large;    // large unit ids by level, largest first
  // Solve tiles (kSolveTile rows) of the large units: entry q of lvl_large
  // owns tiles lvl_large_tile0[q] .. lvl_large_tile0[q + 1] - 1 of the
  // solve's ready-flag arrays.
  std::vector<int32_t> lvl_large_tile0;  // lvl_large.size() + 1
  int32_t large_tiles = 0;
  std::vector<int32_t> small_units, large_units;  // small units by increasing size
  // Size buckets of small_units for the factor launches (shared memory per
  // CTA sized to the bucket's largest unit): small_units[small_bucket_ptr[b]
  // .. small_bucket_ptr[b+1]) have at most small_bucket_m[b] rows.
  std::vector<int32_t> small_bucket_ptr, small_bucket_m;
  std::vector<int32_t> lvl_dense_maxm;  // per level: largest small unit (0 if none)
  // Blocked LU steps for large units (panel width kPanel): per step, the
  // active large units and per-unit CTA prefix sums for the swap/TRSM and
  // GEMM-update kernels.
  int32_t nsteps = 0;
  std::vector<int32_t> step_ptr;        // nsteps + 1 into the arrays below
  std::vector<int32_t> step_unit;       // active unit ids
  std::vector<int32_t> step_trsm_pref;  // exclusive prefix of TRSM CTAs (per active unit, +1 total)
  std::vector<int32_t> step_gemm_pref;  // exclusive prefix of GEMM tiles
  std::vector<int32_t> step_trsm_total, step_gemm_total;  // per step
  std::vector<int32_t> step_max_rows;                     // per step: largest m - k0
  // Value-only refactor of large units (stored pivot order, no pivot
  // search): steps of kRPanel columns.  Per step and active unit: CTA
  // prefixes of the panel kernel (row chunks then column chunks of kRPanel,
  // at least one), of the update tiles that cover the next step's strips
  // ("a": tile row 0 and tile column 0, at least one, which places the
  // factored diagonal block) and of the remaining tiles ("b").
  int32_t rsteps = 0;
  int32_t rmax_active = 0;
  std::vector<int32_t> rstep_ptr, rstep_unit;
  std::vector<int32_t> rstep_strip_pref, rstep_ga_pref, rstep_gb_pref;  // per active unit, exclusive
  std::vector<int32_t> rstep_strip_total, rstep_ga_total, rstep_gb_total;
  // The same refactor as one tile task graph (build_rtasks): four words per
  // task and the size of the ticket + version-word array.  Empty when the
  // list would exceed kRTaskMax tasks.
  std::vector<int32_t> rtask;
  int32_t rtasks = 0;
  int32_t rt_words = 0;
  // Sparse-LU units (gp.h), indexed g = 0 .. sparse_units.size() - 1.  Their
  // columns are numbered globally: unit g's local column j is gp_col0[g] + j.
  //   gp_cptr / gp_row: entries of L + U per column (local rows ascending),
  //     gp_dpos: index of each column's diagonal entry; values in gp_val
  //     order (device): U above the diagonal, the pivot, L multipliers below.
  //   gp_aptr / gp_arow / gp_asrc: A's entries per column (local row,
  //     canonical source).
  //   Solve: strict L and strict U by rows (local column, value position),
  //     rows per global row index gp_col0[g] + i, columns ascending.
  std::vector<int32_t> sparse_units;
  std::vector<int32_t> gp_col0;
  std::vector<int32_t> gp_cptr, gp_row, gp_dpos;
  std::vector<int32_t> gp_aptr, gp_arow, gp_asrc;
  std::vector<int32_t> gp_lrp, gp_lci, gp_lpos;
  std::vector<int32_t> gp_urp, gp_uci, gp_upos;
  std::vector<int32_t> lvl_sparse_ptr, lvl_sparse;  // g by unit level
  std::vector<int32_t> gp_index;                    // per unit: g, or -1
  int64_t gp_nnz = 0;
  int32_t gp_maxm = 0;
  double gp_flops = 0.0;
  // Units the sparse route tried and kept dense: the symbolic rejected them
  // (no structural diagonal) or their fill exceeded the route's limit.
  std::vector<int32_t> gp_symbolic_rejected;  // unit ids
  // Canonical CSR (original coordinates) for the residual.
  std::vector<int32_t> csr_ptr;
  double factor_flops = 0.0;
  int64_t dense_entries = 0;
  int32_t max_unit = 0;
};

constexpr int kPanel = 32;          // panel width of the blocked LU
constexpr int kTrsmCols = 128;      // columns per CTA in the swap/TRSM kernel
constexpr int kGemmTile = 128;      // square output tile of the update kernel
constexpr int kRPanel = 64;         // panel width of the value-only refactor
constexpr int kRTileM = 128;        // update tile of the value-only refactor: rows
constexpr int kRTileN = 64;         //   and columns
constexpr int kSolveTile = 64;      // row tile of the large-unit triangular solves

constexpr int64_t kRTaskMax = int64_t{1} << 24;  // task-graph refactor: largest task list

// Task list of the value-only refactor of large units as a tile graph.
// Tiles are kRPanel x kRPanel; per unit of nt tiles per side and step k:
//   D(k)       LU without pivot search of tile (k, k), in place
//   L(i, k)    tile (i, k) <- tile (i, k) U(k, k)^{-1}, i > k
//   U(k, j)    tile (k, j) <- L(k, k)^{-1} tile (k, j), j > k
//   G(i, j, k) row tiles i and i + 1 (if it exists) of tile column j
//              -= L(i.., k) U(k, j), for the row pairs k+1, k+3, ... and
//              every j > k
// A task is four words: unit, k, (i << 16) | j, and the base of the unit's
// version words (tile (i, j) at base + i * nt + j; word 0 of the array is
// the ticket counter).  The kind follows from i, j and k (D: i = j = k,
// L: j = k < i, U: i = k < j, G: i, j > k).  Version word of a tile = steps
// applied to it: G(i, j, k) and the final D/L/U of step k leave k + 1.
// Order, per step k: D, L and U of step k (the tiles of step k + 1's panel
// first); the updates of step k - 1 that do not touch step k + 1's panel,
// soonest-needed tiles first; then step k's updates of row pair k + 1 and
// tile column k + 1 (step k + 1's panel).  Every task's inputs come from
// tasks earlier in the list.  units: unit ids, sizes: their rows.  Returns
// the task count, or -1 if a unit has more than 65535 tiles per side or the
// list would exceed max_tasks (the list is then left empty).
int64_t build_rtasks(const std::vector<int32_t>& units, const std::vector<int32_t>& sizes, int64_t max_tasks,
                     std::vector<int32_t>& tasks, int32_t& words);

struct GpConfig;
// gp: the sparse-LU route's configuration (nullptr: off).
Plan build_plan(const CanonicalCoo& a, const Decomposition& d, int32_t small_max, const GpConfig* gp = nullptr);

}  // namespace bdlu
