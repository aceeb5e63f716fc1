// Batches of independent systems (bdlu_batch_*, include/bdlu.h).
//
// A batch is analysed as one block-diagonal system: system k's rows and
// columns are offset by the rows of the systems before it.  Its BTF blocks
// are exactly the union of the systems' blocks (no entry couples two
// systems), so every diagonal block of every system is factored by the same
// launches (all small blocks in one k_lu_small launch, large blocks batched
// per panel step) and every DAG level of every system is solved by the same
// graph-captured level launch.  The systems' canonical patterns, concatenated
// in system order, are the canonical pattern of the block-diagonal matrix
// (row-major order keeps each system's rows together), so value-only
// refactors take the systems' values back to back.
#include <algorithm>
#include <exception>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "analysis.h"
#include "bdlu.h"
#include "capi_internal.h"

struct bdlu_batch {
  struct System {
    std::vector<int32_t> rows, cols;
    std::vector<double> vals;
    int32_t n = 0;
  };
  std::vector<System> systems;
  std::vector<int32_t> row_off;  // count + 1, after analyze
  std::vector<int64_t> nnz_off;  // count + 1, canonical entries, after analyze
  bdlu_solver* inner = nullptr;  // the block-diagonal system
  bool analyzed = false;
  int last_error = BDLU_OK;
  std::string last_message;
};

namespace {

int bfail(bdlu_batch* b, int code, std::string msg) {
  b->last_error = code;
  b->last_message = std::move(msg);
  return code;
}

int bclear(bdlu_batch* b) {
  b->last_error = BDLU_OK;
  b->last_message.clear();
  return BDLU_OK;
}

// Mirrors the inner handle's status and message into the batch.
int relay(bdlu_batch* b, int st) {
  if (st == BDLU_OK) return bclear(b);
  char buf[1024];
  bdlu_last_error(b->inner, buf, sizeof(buf));
  return bfail(b, st, buf);
}

}  // namespace

extern "C" {

bdlu_batch* bdlu_batch_create(void) {
  try {
    auto* b = new bdlu_batch();
    b->inner = bdlu_create();
    if (!b->inner) {
      delete b;
      return nullptr;
    }
    return b;
  } catch (...) {
    return nullptr;
  }
}

void bdlu_batch_destroy(bdlu_batch* b) {
  if (!b) return;
  bdlu_destroy(b->inner);
  delete b;
}

int32_t bdlu_batch_add(bdlu_batch* b, const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
                       int32_t n) {
  if (!b) return -BDLU_NOT_PREPARED;
  bclear(b);
  if (n <= 0) return -bfail(b, BDLU_INVALID_DIMENSION, "each system of a batch needs its dimension (n > 0)");
  if (nnz < 0 || (nnz > 0 && (!rows || !cols || !vals))) return -bfail(b, BDLU_INVALID_INDEX, "invalid COO arrays");
  try {
    bdlu_batch::System s;
    s.rows.assign(rows, rows + nnz);
    s.cols.assign(cols, cols + nnz);
    s.vals.assign(vals, vals + nnz);
    s.n = n;
    b->systems.push_back(std::move(s));
  } catch (const std::exception& e) {
    return -bfail(b, BDLU_ANALYSIS_FAILED, e.what());
  }
  b->analyzed = false;
  return static_cast<int32_t>(b->systems.size()) - 1;
}

int bdlu_batch_analyze(bdlu_batch* b) {
  if (!b) return BDLU_NOT_PREPARED;
  bclear(b);
  const size_t k = b->systems.size();
  if (k == 0) return bfail(b, BDLU_NOT_PREPARED, "the batch holds no system");
  b->analyzed = false;
  // Validate and canonicalise every system (parallel over host threads).
  std::vector<bdlu::CanonicalCoo> canon(k);
  std::vector<bdlu::Status> st(k, bdlu::Status::Ok);
  std::vector<std::string> msg(k);
  {
    const size_t nt = std::max<size_t>(1, std::min<size_t>(k, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t)
      pool.emplace_back([&, t] {
        for (size_t i = t; i < k; i += nt) {
          const auto& s = b->systems[i];
          try {
            st[i] = bdlu::canonicalize(s.rows.data(), s.cols.data(), s.vals.data(), static_cast<int64_t>(s.rows.size()),
                                       s.n, canon[i], msg[i]);
          } catch (const std::exception& e) {
            st[i] = bdlu::Status::AnalysisFailed;
            msg[i] = e.what();
          }
        }
      });
    for (auto& th : pool) th.join();
  }
  for (size_t i = 0; i < k; ++i)
    if (st[i] != bdlu::Status::Ok)
      return bfail(b, static_cast<int>(st[i]), "system " + std::to_string(i) + ": " + msg[i]);
  // Concatenate into the block-diagonal canonical matrix.
  bdlu_solver* h = b->inner;
  bdlu::PrecomputedBtf btf;
  try {
    b->row_off.assign(k + 1, 0);
    b->nnz_off.assign(k + 1, 0);
    for (size_t i = 0; i < k; ++i) {
      if (static_cast<int64_t>(b->row_off[i]) + canon[i].n > INT32_MAX)
        return bfail(b, BDLU_INVALID_DIMENSION, "the batch exceeds 2^31 - 1 rows");
      b->row_off[i + 1] = b->row_off[i] + canon[i].n;
      b->nnz_off[i + 1] = b->nnz_off[i] + canon[i].nnz();
    }
    bdlu::CanonicalCoo all;
    all.n = b->row_off[k];
    all.row.resize(static_cast<size_t>(b->nnz_off[k]));
    all.col.resize(all.row.size());
    all.val.resize(all.row.size());
    for (size_t i = 0; i < k; ++i) {
      const int32_t ro = b->row_off[i];
      const size_t e0 = static_cast<size_t>(b->nnz_off[i]);
      for (size_t e = 0; e < canon[i].row.size(); ++e) {
        all.row[e0 + e] = canon[i].row[e] + ro;
        all.col[e0 + e] = canon[i].col[e] + ro;
        all.val[e0 + e] = canon[i].val[e];
      }
    }
    // BTF per system, in parallel: the block-diagonal matrix's BTF blocks are
    // the systems' blocks, and a matching search over one system at a time
    // costs far less than phases over the whole batch.
    bdlu::AnalysisOptions opt = bdlu::analysis_options_from_env();
    const double drop = bdlu::drop_threshold(opt, all.n);
    std::vector<std::vector<int32_t>> P(k), Q(k), R(k);
    std::vector<int32_t> nb(k, 0), nm(k, 0);
    {
      const size_t nt = std::max<size_t>(1, std::min<size_t>(k, std::thread::hardware_concurrency()));
      std::vector<std::thread> pool;
      for (size_t t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
          for (size_t i = t; i < k; i += nt) {
            try {
              const int32_t n = canon[i].n;
              const bdlu::Csc csc = bdlu::pattern_csc(canon[i], drop);
              P[i].resize(static_cast<size_t>(n));
              Q[i].resize(static_cast<size_t>(n));
              R[i].resize(static_cast<size_t>(n) + 1);
              nb[i] = bdlu::btf_order(n, csc.col_ptr.data(), csc.row_ind.data(), P[i].data(), Q[i].data(),
                                      R[i].data(), &nm[i]);
            } catch (...) {
              nb[i] = -1;
            }
          }
        });
      for (auto& th : pool) th.join();
    }
    btf.P.reserve(static_cast<size_t>(all.n));
    btf.Q.reserve(static_cast<size_t>(all.n));
    for (size_t i = 0; i < k; ++i) {
      if (nb[i] <= 0) return bfail(b, BDLU_ANALYSIS_FAILED, "system " + std::to_string(i) + ": btf_order failed");
      const int32_t ro = b->row_off[i];
      for (int32_t v : P[i]) btf.P.push_back(v + ro);
      for (int32_t v : Q[i]) btf.Q.push_back((v < -1 ? -v - 2 : v) + ro);
      for (int32_t q = 0; q < nb[i]; ++q) btf.R.push_back(R[i][static_cast<size_t>(q)] + ro);
      btf.nmatch += nm[i];
    }
    btf.R.push_back(all.n);
    h->engine.reset();
    h->coo = std::move(all);
    h->n = h->coo.n;
    h->dimension_hint = h->n;
    h->prepared = true;
    h->validated = true;
  } catch (const std::bad_alloc&) {
    return bfail(b, BDLU_ANALYSIS_FAILED, "out of host memory while assembling the batch");
  }
  const int r = bdlu_analyze_validated(h, BDLU_MODE_BLOCK, &btf);
  if (r != BDLU_OK) return relay(b, r);
  b->analyzed = true;
  return BDLU_OK;
}

int bdlu_batch_factor(bdlu_batch* b) {
  if (!b) return BDLU_NOT_PREPARED;
  if (!b->analyzed) return bfail(b, BDLU_NOT_PREPARED, "bdlu_batch_analyze must succeed before factor");
  return relay(b, bdlu_factor(b->inner));
}

int bdlu_batch_refactor_values(bdlu_batch* b, const double* vals, int64_t nnz) {
  if (!b) return BDLU_NOT_PREPARED;
  if (!b->analyzed) return bfail(b, BDLU_NOT_PREPARED, "bdlu_batch_analyze must succeed before refactor");
  return relay(b, bdlu_refactor_values(b->inner, vals, nnz));
}

int bdlu_batch_refactor_values_device(bdlu_batch* b, const double* d_vals, int64_t nnz, void* stream) {
  if (!b) return BDLU_NOT_PREPARED;
  if (!b->analyzed) return bfail(b, BDLU_NOT_PREPARED, "bdlu_batch_analyze must succeed before refactor");
  return relay(b, bdlu_refactor_values_device(b->inner, d_vals, nnz, stream));
}

int bdlu_batch_solve(bdlu_batch* b, double* B, int32_t ldb, int32_t nrhs) {
  if (!b) return BDLU_NOT_PREPARED;
  if (!b->analyzed) return bfail(b, BDLU_NOT_PREPARED, "bdlu_batch_analyze must succeed before solve");
  return relay(b, bdlu_solve(b->inner, B, ldb, nrhs));
}

int bdlu_batch_solve_device(bdlu_batch* b, double* d_B, int32_t ldb, int32_t nrhs, void* stream) {
  if (!b) return BDLU_NOT_PREPARED;
  if (!b->analyzed) return bfail(b, BDLU_NOT_PREPARED, "bdlu_batch_analyze must succeed before solve");
  return relay(b, bdlu_solve_device(b->inner, d_B, ldb, nrhs, stream));
}

int32_t bdlu_batch_count(const bdlu_batch* b) { return b ? static_cast<int32_t>(b->systems.size()) : 0; }

int64_t bdlu_batch_row_offset(const bdlu_batch* b, int32_t k) {
  if (!b || !b->analyzed || k < 0 || k > static_cast<int32_t>(b->systems.size())) return -1;
  return b->row_off[static_cast<size_t>(k)];
}

int64_t bdlu_batch_nnz_offset(const bdlu_batch* b, int32_t k) {
  if (!b || !b->analyzed || k < 0 || k > static_cast<int32_t>(b->systems.size())) return -1;
  return b->nnz_off[static_cast<size_t>(k)];
}

int bdlu_batch_last_error(const bdlu_batch* b, char* buf, int64_t len) {
  if (!b) return BDLU_NOT_PREPARED;
  if (buf && len > 0) {
    const size_t m = std::min<size_t>(static_cast<size_t>(len - 1), b->last_message.size());
    std::copy(b->last_message.begin(), b->last_message.begin() + static_cast<std::ptrdiff_t>(m), buf);
    buf[m] = '\0';
  }
  return b->last_error;
}

int bdlu_batch_get_stats(const bdlu_batch* b, bdlu_stats* out) {
  if (!b || !out) return BDLU_NOT_PREPARED;
  return bdlu_get_stats(b->inner, out);
}

int bdlu_batch_phase_times(bdlu_batch* b, double* ms, int32_t cap) {
  if (!b) return BDLU_NOT_PREPARED;
  return bdlu_phase_times(b->inner, ms, cap);
}

}  // extern "C"
