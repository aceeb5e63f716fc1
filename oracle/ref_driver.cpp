// C entry points into the reference's own code (compiled from its sources
// where they lie, by oracle/Makefile, into oracle/_ref/libbdlu_ref.so).
// Test infrastructure only: tests and bench.py's reference arm call these to
// run the reference's Solver, decomposition, block factor and block solve.
//
// blockdaglu/src/solver.cpp is compiled as part of this translation unit
// (included unmodified) so that its file-local helpers -- the pattern and
// value signatures and the canonicalisation -- can be called for parity
// checks; the library contains it once.
#include "solver.cpp"

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <tuple>
#include <vector>

#include "blockdaglu/solver.h"
#include "gp_lu.h"
#include "ubtf_block_solver.h"

using blockdaglu::CooMatrix;
using blockdaglu::Solver;

extern "C" {

void* ref_solver_create() { return new Solver(); }
void ref_solver_destroy(void* h) { delete static_cast<Solver*>(h); }

int ref_solver_set_coo(void* h, const int32_t* r, const int32_t* c, const double* v, int64_t nnz, int32_t dim) {
  CooMatrix m;
  m.reserve(static_cast<size_t>(nnz));
  for (int64_t k = 0; k < nnz; ++k) m.emplace_back(r[k], c[k], v[k]);
  return static_cast<Solver*>(h)->set_matrix(std::move(m), dim) ? 0 : static_cast<int>(static_cast<Solver*>(h)->last_error());
}

static int status_of(Solver* s, bool ok) { return ok ? 0 : static_cast<int>(s->last_error()); }

int ref_solver_analyze(void* h) { auto* s = static_cast<Solver*>(h); return status_of(s, s->analyze()); }
int ref_solver_factor(void* h) { auto* s = static_cast<Solver*>(h); return status_of(s, s->factor()); }

int ref_solver_solve(void* h, double* b, int32_t n) {
  auto* s = static_cast<Solver*>(h);
  std::vector<double> x(b, b + n);
  const bool ok = s->solve_in_place(x);
  if (ok) std::memcpy(b, x.data(), sizeof(double) * x.size());
  return status_of(s, ok);
}

const char* ref_solver_mode(void* h) { return static_cast<Solver*>(h)->selected_mode(); }

// validate_and_canonicalize_matrix, then compute_matrix_sig / sig2 /
// value_sig (solver.cpp:96-136, :642-722) on the canonical COO.  Returns 0,
// or the SolverError code of a rejected input.
int ref_matrix_sigs(const int32_t* r, const int32_t* c, const double* v, int64_t nnz, int32_t dim, int32_t* n_out,
                    uint64_t* sigs) {
  CooMatrix m;
  m.reserve(static_cast<size_t>(nnz));
  for (int64_t k = 0; k < nnz; ++k) m.emplace_back(r[k], c[k], v[k]);
  int32_t n = 0;
  blockdaglu::SolverError err = blockdaglu::SolverError::None;
  std::string msg;
  if (!blockdaglu::validate_and_canonicalize_matrix(m, dim, n, err, msg)) return static_cast<int>(err);
  if (n_out) *n_out = n;
  sigs[0] = blockdaglu::compute_matrix_sig(n, m);
  sigs[1] = blockdaglu::compute_matrix_sig2(n, m);
  sigs[2] = blockdaglu::compute_matrix_value_sig(m);
  return 0;
}

int ref_solver_error(void* h, char* buf, int64_t len) {
  auto* s = static_cast<Solver*>(h);
  if (buf && len > 0) {
    std::strncpy(buf, s->last_error_message().c_str(), static_cast<size_t>(len - 1));
    buf[len - 1] = 0;
  }
  return static_cast<int>(s->last_error());
}

// Exports: kind 0 rearranged, 1 P, 2 Q, 3 L, 4 U.  Returns count.
int64_t ref_solver_export(void* h, int kind, int32_t* r, int32_t* c, double* v, int64_t cap) {
  auto* s = static_cast<Solver*>(h);
  CooMatrix m = kind == 0 ? s->get_rearranged_matrix() : kind == 1 ? s->getP() : kind == 2 ? s->getQ()
              : kind == 3 ? s->getL() : s->getU();
  for (int64_t k = 0; k < cap && k < static_cast<int64_t>(m.size()); ++k) {
    r[k] = std::get<0>(m[static_cast<size_t>(k)]);
    c[k] = std::get<1>(m[static_cast<size_t>(k)]);
    v[k] = std::get<2>(m[static_cast<size_t>(k)]);
  }
  return static_cast<int64_t>(m.size());
}

// The reference's decomposition, factor and reverse block solve on a
// canonical COO (build_decomposition_btf, factor_blocks_parallel, solve_ubtf).
struct RefRun {
  UbftfDecomposition dec;
  UbftfFactors fac;
  bool factored = false;
};

void* ref_decompose(const int32_t* r, const int32_t* c, const double* v, int64_t nnz, int32_t n) {
  std::vector<std::tuple<int, int, double>> coo;
  coo.reserve(static_cast<size_t>(nnz));
  for (int64_t k = 0; k < nnz; ++k) coo.emplace_back(r[k], c[k], v[k]);
  auto* run = new RefRun();
  try {
    run->dec = build_decomposition_btf(coo, n, 16, 1024);
  } catch (...) {
    delete run;
    return nullptr;
  }
  return run;
}

void ref_run_free(void* p) {
  auto* run = static_cast<RefRun*>(p);
  if (run && run->factored) free_factors(run->fac);
  delete run;
}

int32_t ref_nblocks(void* p) { return static_cast<RefRun*>(p)->dec.nblocks; }
int32_t ref_max_level(void* p) { return static_cast<RefRun*>(p)->dec.max_level; }
int32_t ref_offdiag_nnz(void* p) { return static_cast<RefRun*>(p)->dec.Aperm_csr.nnz; }

void ref_get_decomposition(void* p, int32_t* P, int32_t* Q, int32_t* R, int32_t* off_ptr, int32_t* off_col,
                           double* off_val, int32_t* level) {
  const auto& d = static_cast<RefRun*>(p)->dec;
  if (P) std::memcpy(P, d.P.data(), sizeof(int32_t) * d.P.size());
  if (Q) std::memcpy(Q, d.Q.data(), sizeof(int32_t) * d.Q.size());
  if (R) std::memcpy(R, d.R.data(), sizeof(int32_t) * d.R.size());
  if (off_ptr) std::memcpy(off_ptr, d.Aperm_csr.row_ptr.data(), sizeof(int32_t) * d.Aperm_csr.row_ptr.size());
  if (off_col) std::memcpy(off_col, d.Aperm_csr.col_ind.data(), sizeof(int32_t) * d.Aperm_csr.col_ind.size());
  if (off_val) std::memcpy(off_val, d.Aperm_csr.values.data(), sizeof(double) * d.Aperm_csr.values.size());
  if (level && !d.block_level.empty()) std::memcpy(level, d.block_level.data(), sizeof(int32_t) * d.block_level.size());
}

int ref_factor(void* p, int32_t threads) {
  auto* run = static_cast<RefRun*>(p);
  run->fac = factor_blocks_parallel(run->dec, static_cast<size_t>(threads > 0 ? threads : 1));
  run->factored = true;
  int bad = 0;
  for (const auto& b : run->fac.blocks) bad += b.ok ? 0 : 1;
  return bad;
}

// Dense factor of block b (empty when the block went to the KLU stand-in).
int32_t ref_block_lu(void* p, int32_t b, double* lu, int32_t* piv) {
  const auto& bf = static_cast<RefRun*>(p)->fac.blocks[static_cast<size_t>(b)];
  if (bf.dense_lu.empty()) return 0;
  if (lu) std::memcpy(lu, bf.dense_lu.data(), sizeof(double) * bf.dense_lu.size());
  if (piv) std::memcpy(piv, bf.piv.data(), sizeof(int32_t) * bf.piv.size());
  return bf.size;
}

int ref_block_solve(void* p, double* b, int32_t n, int32_t threads) {
  auto* run = static_cast<RefRun*>(p);
  std::vector<double> x(b, b + n);
  if (!solve_ubtf(run->dec, run->fac, x, static_cast<size_t>(threads > 0 ? threads : 1))) return 1;
  std::memcpy(b, x.data(), sizeof(double) * static_cast<size_t>(n));
  return 0;
}

// gp_lu_factor (gp_lu.cpp:84-240) on an m x m CSC with the given options.
// lu: row-major m*m (L multipliers strictly below the diagonal from L_rows,
// U on and above from U_rows and Udiag), perm: GpLuFactor::perm, row_scale
// (1.0 when scaling is off); stats: ok, row swaps, tiny pivots, zero pivots.
int ref_gp_lu(int32_t m, const int32_t* col_ptr, const int32_t* row_ind, const double* val, int32_t scale,
              double diag_tol, double pivot_tol, double perturb, double drop_tol, double* lu, int32_t* perm,
              double* row_scale, int32_t* stats) {
  CscMatrixI32 a;
  a.n = m;
  a.nnz = col_ptr[m];
  a.col_ptr.assign(col_ptr, col_ptr + m + 1);
  a.row_ind.assign(row_ind, row_ind + col_ptr[m]);
  a.values.assign(val, val + col_ptr[m]);
  GpLuOptions opt;
  opt.scale = scale;
  opt.diag_prefer_tol = diag_tol;
  opt.pivot_tol = pivot_tol;
  opt.perturb = perturb;
  opt.drop_tol = drop_tol;
  GpLuFactor f;
  const bool ok = gp_lu_factor(a, f, opt);
  stats[0] = ok ? 1 : 0;
  stats[1] = f.row_swap_count;
  stats[2] = f.tiny_pivot_count;
  stats[3] = f.zero_pivot_count;
  if (!ok) return 0;
  std::memset(lu, 0, sizeof(double) * static_cast<size_t>(m) * m);
  for (int32_t i = 0; i < m; ++i) {
    for (const auto& e : f.L_rows[static_cast<size_t>(i)]) lu[static_cast<size_t>(i) * m + e.first] = e.second;
    for (const auto& e : f.U_rows[static_cast<size_t>(i)])
      if (e.first > i) lu[static_cast<size_t>(i) * m + e.first] = e.second;
    lu[static_cast<size_t>(i) * m + i] = f.Udiag[static_cast<size_t>(i)];
    perm[i] = f.perm[static_cast<size_t>(i)];
    row_scale[i] = f.row_scale.empty() ? 1.0 : f.row_scale[static_cast<size_t>(i)];
  }
  return 1;
}

// gp_lu_solve_inplace_strided (gp_lu.cpp:242-306) after gp_lu_factor with the
// default options: b (m) is replaced by x.  Returns 1 on success.
int ref_gp_solve(int32_t m, const int32_t* col_ptr, const int32_t* row_ind, const double* val, double* b) {
  CscMatrixI32 a;
  a.n = m;
  a.nnz = col_ptr[m];
  a.col_ptr.assign(col_ptr, col_ptr + m + 1);
  a.row_ind.assign(row_ind, row_ind + col_ptr[m]);
  a.values.assign(val, val + col_ptr[m]);
  GpLuFactor f;
  if (!gp_lu_factor(a, f, GpLuOptions{})) return 0;
  return gp_lu_solve_inplace_strided(f, b, m, 1) ? 1 : 0;
}

// Route of block b after ref_factor: 0 dense micro-kernel, 1 sparse LU (GP)
// accepted, 2 KLU stand-in; *reason = BlockFactor::gp_reject_reason.
int32_t ref_block_route(void* p, int32_t b, int32_t* reason) {
  const auto& bf = static_cast<RefRun*>(p)->fac.blocks[static_cast<size_t>(b)];
  if (reason) *reason = bf.gp_reject_reason;
  if (!bf.dense_lu.empty()) return 0;
  return bf.gp ? 1 : 2;
}

// Factors of a block the sparse-LU route kept, as in ref_gp_lu.  Returns m,
// or 0 when the block has none.
int32_t ref_block_gp(void* p, int32_t b, double* lu, int32_t* perm) {
  const auto& bf = static_cast<RefRun*>(p)->fac.blocks[static_cast<size_t>(b)];
  if (!bf.gp) return 0;
  const GpLuFactor& f = *bf.gp;
  const int32_t m = f.n;
  std::memset(lu, 0, sizeof(double) * static_cast<size_t>(m) * m);
  for (int32_t i = 0; i < m; ++i) {
    for (const auto& e : f.L_rows[static_cast<size_t>(i)]) lu[static_cast<size_t>(i) * m + e.first] = e.second;
    for (const auto& e : f.U_rows[static_cast<size_t>(i)])
      if (e.first > i) lu[static_cast<size_t>(i) * m + e.first] = e.second;
    lu[static_cast<size_t>(i) * m + i] = f.Udiag[static_cast<size_t>(i)];
    perm[i] = f.perm[static_cast<size_t>(i)];
  }
  return m;
}

}  // extern "C"
