// Host-side integer analysis of the BlockDAGLU hot path.
//
// Everything here is integer (index) work plus value copies, done once per
// sparsity pattern on the host.  It restates the reference's own analysis so
// that permutations, block boundaries, the off-diagonal CSR and the block DAG
// come out identical to what the reference computes from the same BTF output:
//   validate_and_canonicalize_matrix   blockdaglu/src/solver.cpp:642-722
//   compute_matrix_sig / sig2 / value  blockdaglu/src/solver.cpp:96-136
//   auto_choose_block                  blockdaglu/src/solver.cpp:448-506
//   build_decomposition_btf            blockdaglu/src/ubtf_block_solver.cpp:570-938
//   merge_block_boundaries             blockdaglu/src/ubtf_block_solver.cpp:393-476
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace bdlu {

// Canonical COO: sorted by (row, col), duplicates summed, exact zeros dropped.
// Because it is row-major sorted with no duplicates it is also a CSR matrix.
struct CanonicalCoo {
  int32_t n = 0;
  std::vector<int32_t> row;
  std::vector<int32_t> col;
  std::vector<double> val;
  int64_t nnz() const { return static_cast<int64_t>(row.size()); }
};

enum class Status : int {
  Ok = 0,
  NotPrepared = 1,
  InvalidDimension = 2,
  InvalidIndex = 3,
  NonFiniteValue = 4,
  InvalidRightHandSide = 5,
  BackendUnavailable = 6,
  AnalysisFailed = 7,
  FactorizationFailed = 8,
  SolveFailed = 9,
  ExportFailed = 10,
};

// solver.cpp:642-722.  Returns Ok or the reference's error code; `msg` gets the
// reference's message text.
Status canonicalize(const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
                    int32_t dimension_hint, CanonicalCoo& out, std::string& msg);

uint64_t matrix_sig(int32_t n, const CanonicalCoo& a);       // solver.cpp:96-108
uint64_t matrix_sig2(int32_t n, const CanonicalCoo& a);      // solver.cpp:110-124
uint64_t matrix_value_sig(const CanonicalCoo& a);            // solver.cpp:126-136

// Coarse + profile-refined AUTO rule, solver.cpp:448-506 and :182-231
// (without the in-process learned override).
bool auto_choose_block(int32_t n, const CanonicalCoo& a);

// Compressed sparse column, int32 indices (sparse_formats.h:7-13).
struct Csc {
  int32_t n = 0;
  std::vector<int32_t> col_ptr;
  std::vector<int32_t> row_ind;
};

// Pattern CSC from the canonical COO; entries with |v| < drop_abs_lt are left
// out when drop_abs_lt > 0 (ubtf_block_solver.cpp:333-371, :582-589).
Csc pattern_csc(const CanonicalCoo& a, double drop_abs_lt);

// Dulmage-Mendelsohn fine decomposition with the calling convention of
// SuiteSparse btf_order: P, Q (Q flipped for unmatched columns), R, nmatch.
// Returns the number of blocks.
int32_t btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q,
                  int32_t* R, int32_t* nmatch);

// ubtf_block_solver.cpp:393-476.
std::vector<int32_t> merge_block_boundaries(const std::vector<int32_t>& R, int32_t n,
                                            int32_t merge_max);

// The UBTF split: everything ubtf_block_solver.cpp:570-909 produces, plus the
// source index of every scattered value (canonical COO position) so that a
// value-only refactor is a gather.
struct Decomposition {
  int32_t n = 0;
  int32_t nblocks_raw = 0;
  int32_t nmatch = 0;
  int32_t nblocks = 0;
  std::vector<int32_t> P, Q, invP, invQ;  // perm index -> original, and inverses
  std::vector<int32_t> R;                 // nblocks + 1 (after merging)
  std::vector<int32_t> R_raw;             // nblocks_raw + 1 (btf_order output)
  // Off-diagonal strictly-upper CSR in permuted coordinates.
  std::vector<int32_t> off_ptr;  // n + 1
  std::vector<int32_t> off_col;  // permuted column
  std::vector<int32_t> off_src;  // canonical COO index of the value
  // Per-block local COO (row, col local to the block), canonical order.
  std::vector<int64_t> diag_ptr;  // nblocks + 1
  std::vector<int32_t> diag_row, diag_col;
  std::vector<int32_t> diag_src;
  // Block DAG (ubtf_block_solver.cpp:857-909): deps to higher block ids in
  // first-appearance order, level 0 solved first.
  std::vector<int32_t> dep_ptr, dep_idx;
  std::vector<int32_t> level;
  int32_t max_level = 0;
  std::vector<int32_t> level_ptr, level_blocks;  // blocks_by_level, flattened
};

// A BTF ordering computed elsewhere (for a block-diagonal batch: the
// systems' orderings, offset and concatenated).  Q is unflipped.
struct PrecomputedBtf {
  std::vector<int32_t> P, Q, R;  // R: nblocks + 1 boundaries
  int32_t nmatch = 0;
};

struct AnalysisOptions {
  int32_t merge_max = 64;      // BLOCK_MERGE_MAX_SIZE, else DENSE_BLOCK_MAX, else 64
  bool merge = true;           // BLOCK_MERGE
  double drop_abs_lt = -1.0;   // DROP_ABS_LT (negative: auto, 1e-20 iff n >= 50000)
  bool single_block = false;   // global route: one block, identity P/Q
  const PrecomputedBtf* btf = nullptr;  // used instead of btf_order when set
};

// The drop threshold build_decomposition applies for options `opt` at size n.
double drop_threshold(const AnalysisOptions& opt, int32_t n);

// Reads the reference's environment knobs (BLOCKDAGLU_* over USERALGO_*).
AnalysisOptions analysis_options_from_env();

// Throws std::runtime_error with the reference's message on a non-UBTF result.
Decomposition build_decomposition(const CanonicalCoo& a, const AnalysisOptions& opt);

// env.h:15-25 lookup order.
const char* getenv_compat(const char* name);

}  // namespace bdlu
