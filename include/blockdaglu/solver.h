// blockdaglu::Solver on the B200 engine: a header-only C++ class over the C
// ABI in bdlu.h.
//
// Source-compatible with the reference class (blockdaglu/include/blockdaglu/
// solver.h:43-126): the same stage methods, error enum, exports, n() and
// selected_mode(), with the same conventions -- every call returns bool, a
// false return leaves last_error()/last_error_message() set, no exception
// leaves a method, set_matrix only stores (validation happens in analyze),
// solve_in_place overwrites b with x, exports return a fresh COO (empty on
// failure).  One Solver must not be used from two threads at once; distinct
// Solvers may run concurrently.
//
// Additions (no counterpart in the reference class):
//   refactor_values(values, nnz)   value-only refactor: new values in the
//                                  order of the canonical pattern (row-major,
//                                  duplicates summed, exact zeros dropped)
//   solve_in_place(B, ldb, nrhs)   column-major block of right-hand sides
//   last_stats()                   refinement steps, residual, device times
//
// Link with libbdlu.so (block-daglu_b200/lib).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "bdlu.h"
#include "blockdaglu/types.h"

namespace blockdaglu {

// Same enumerators, in the same order, as the reference (solver.h:19-31);
// the values equal the C ABI's bdlu_status codes.
enum class SolverError {
  None,
  NotPrepared,
  InvalidDimension,
  InvalidIndex,
  NonFiniteValue,
  InvalidRightHandSide,
  BackendUnavailable,
  AnalysisFailed,
  FactorizationFailed,
  SolveFailed,
  ExportFailed,
};

using ResultStats = bdlu_stats;

class Solver final {
 public:
  Solver() : h_(bdlu_create()) {
    if (!h_) {
      last_error_ = SolverError::BackendUnavailable;
      last_error_message_ = "bdlu_create failed (no CUDA device or out of memory)";
    }
  }
  ~Solver() {
    if (h_) bdlu_destroy(h_);
  }
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  bool set_matrix(CooMatrix m) { return set_matrix(std::move(m), -1); }
  bool set_matrix(CooMatrix m, int32_t dimension) {
    if (!h_) return false;
    const size_t nnz = m.size();
    std::vector<int32_t> rows(nnz), cols(nnz);
    std::vector<double> vals(nnz);
    for (size_t k = 0; k < nnz; ++k) {
      rows[k] = std::get<0>(m[k]);
      cols[k] = std::get<1>(m[k]);
      vals[k] = std::get<2>(m[k]);
    }
    return done(bdlu_set_coo(h_, rows.data(), cols.data(), vals.data(), static_cast<int64_t>(nnz), dimension));
  }
  bool analyze() { return h_ && done(bdlu_analyze(h_)); }
  bool factor() { return h_ && done(bdlu_factor(h_)); }
  bool solve_in_place(std::vector<double>& b) {
    if (!h_) return false;
    // A size mismatch is reported by the engine as InvalidRightHandSide.
    const int32_t ldb = (b.size() == static_cast<size_t>(bdlu_n(h_))) ? static_cast<int32_t>(b.size()) : -1;
    return done(bdlu_solve(h_, b.data(), ldb, 1));
  }

  bool refactor_values(const double* values, size_t nnz) {
    return h_ && done(bdlu_refactor_values(h_, values, static_cast<int64_t>(nnz)));
  }
  bool solve_in_place(double* B, int32_t ldb, int32_t nrhs) { return h_ && done(bdlu_solve(h_, B, ldb, nrhs)); }
  const ResultStats& last_stats() {
    if (h_) bdlu_get_stats(h_, &stats_);
    return stats_;
  }

  SolverError last_error() const { return last_error_; }
  const std::string& last_error_message() const { return last_error_message_; }

  CooMatrix get_rearranged_matrix() { return fetch(&bdlu_export_rearranged); }
  CooMatrix getQ() { return fetch(&bdlu_export_q); }
  CooMatrix getP() { return fetch(&bdlu_export_p); }
  CooMatrix getL() { return fetch(&bdlu_export_l); }
  CooMatrix getU() { return fetch(&bdlu_export_u); }

  int32_t n() const { return h_ ? bdlu_n(h_) : 0; }
  const char* selected_mode() const { return h_ ? bdlu_selected_mode(h_) : "KLU"; }

 private:
  using Export = int64_t (*)(bdlu_solver*, int32_t*, int32_t*, double*, int64_t);

  bool done(int status) {
    last_error_ = static_cast<SolverError>(status);
    if (status == BDLU_OK) {
      last_error_message_.clear();
      return true;
    }
    char buf[1024];
    bdlu_last_error(h_, buf, sizeof(buf));
    last_error_message_ = buf;
    return false;
  }

  CooMatrix fetch(Export fn) {
    CooMatrix out;
    if (!h_) return out;
    const int64_t count = fn(h_, nullptr, nullptr, nullptr, 0);
    if (count < 0) {
      done(static_cast<int>(-count));
      return out;
    }
    std::vector<int32_t> rows(static_cast<size_t>(count)), cols(static_cast<size_t>(count));
    std::vector<double> vals(static_cast<size_t>(count));
    const int64_t got = fn(h_, rows.data(), cols.data(), vals.data(), count);
    if (got < 0) {
      done(static_cast<int>(-got));
      return out;
    }
    done(BDLU_OK);
    out.reserve(static_cast<size_t>(got));
    for (int64_t k = 0; k < got; ++k)
      out.emplace_back(rows[static_cast<size_t>(k)], cols[static_cast<size_t>(k)], vals[static_cast<size_t>(k)]);
    return out;
  }

  bdlu_solver* h_ = nullptr;
  SolverError last_error_ = SolverError::None;
  std::string last_error_message_;
  ResultStats stats_{};
};

}  // namespace blockdaglu
