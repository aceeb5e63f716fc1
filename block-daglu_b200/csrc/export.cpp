// Lazy P/Q/L/U export and the merged-block LU view.
//
// The reference exports an independent global KLU factorisation with btf = 0
// (solver.cpp:1598-1663) such that A[pinv, qinv] = L*U (:1665-1691).  Here
// the export is built from the engine's own device factors: with the UBTF
// permutation (P, Q) and the per-unit pivot orders applied to the rows,
//   A[rows, Q] = L * U,  L = blockdiag(L_u) (unit diagonal),
//   U = blockdiag(U_u) + [L_u^{-1} P_u A_uv] (v > u),
// which satisfies the same identity (apps/tests/main.cpp:170-195).  Row scaling
// is 1.  This file is built with -ffp-contract=off so host arithmetic is not
// fused.  The coupling part costs O(m^2) per coupled column of a dense unit, so
// exports are meant for small and medium systems, as in the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "bdlu.h"
#include "capi_internal.h"
#include "plan.h"

namespace {

// Row order of a unit after its LAPACK-style sequential swaps.
std::vector<int32_t> pivot_order(const std::vector<int32_t>& piv, int32_t m) {
  std::vector<int32_t> ord(static_cast<size_t>(m));
  for (int32_t i = 0; i < m; ++i) ord[static_cast<size_t>(i)] = i;
  for (int32_t k = 0; k < m; ++k) std::swap(ord[static_cast<size_t>(k)], ord[static_cast<size_t>(piv[static_cast<size_t>(k)])]);
  return ord;
}

int ensure_factored(bdlu_solver* h) {
  if (h->factored) return BDLU_OK;
  if (!h->prepared) return bdlu_fail(h, BDLU_NOT_PREPARED, "set_matrix must be called before exporting factors");
  if (!h->decomposed) {
    if (const int st = bdlu_analyze(h)) return st;
  }
  return bdlu_factor(h);
}

}  // namespace

int bdlu_build_export(bdlu_solver* h) {
  if (h->exported) return BDLU_OK;
  if (const int st = ensure_factored(h)) return st;
  if (const int st = bdlu_sync_host_values(h)) return st;
  bdlu::Engine& eng = *h->engine;
  const bdlu::Plan& p = eng.plan();
  const auto& d = h->dec;
  const int32_t n = h->n;
  std::vector<int32_t> rows(static_cast<size_t>(n));  // new row -> original row
  h->l_r.clear(); h->l_c.clear(); h->l_v.clear();
  h->u_r.clear(); h->u_c.clear(); h->u_v.clear();
  std::string err;
  std::vector<double> lu;
  std::vector<int32_t> piv;
  for (int32_t u = 0; u < p.nunits; ++u) {
    const int32_t s = p.ustart[static_cast<size_t>(u)];
    const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - s;
    double scalar = 0.0;
    if (!eng.download_unit(u, lu, piv, scalar, err)) return bdlu_fail(h, BDLU_EXPORT_FAILED, err);
    const std::vector<int32_t> ord = (m == 1) ? std::vector<int32_t>{0} : pivot_order(piv, m);
    for (int32_t i = 0; i < m; ++i) rows[static_cast<size_t>(s + i)] = d.P[static_cast<size_t>(s + ord[static_cast<size_t>(i)])];
    // Diagonal block: L (unit) and U from the column-major LU.
    for (int32_t j = 0; j < m; ++j) {
      for (int32_t i = 0; i < m; ++i) {
        const double v = (m == 1) ? scalar : lu[static_cast<size_t>(j) * m + i];
        if (i > j) {
          if (v != 0.0) {
            h->l_r.push_back(s + i); h->l_c.push_back(s + j); h->l_v.push_back(v);
          }
        } else if (v != 0.0 || i == j) {
          h->u_r.push_back(s + i); h->u_c.push_back(s + j); h->u_v.push_back(v);
        }
      }
      h->l_r.push_back(s + j); h->l_c.push_back(s + j); h->l_v.push_back(1.0);
    }
    // Coupling rows of the unit: y = L_u^{-1} (rows in pivot order), per column.
    std::map<int32_t, std::vector<double>> cols;  // permuted column -> dense column over the unit
    for (int32_t i = 0; i < m; ++i) {
      const int32_t r = s + ord[static_cast<size_t>(i)];
      for (int32_t q = p.cpl_ptr[static_cast<size_t>(r)]; q < p.cpl_ptr[static_cast<size_t>(r) + 1]; ++q) {
        auto& col = cols[p.cpl_col[static_cast<size_t>(q)]];
        if (col.empty()) col.assign(static_cast<size_t>(m), 0.0);
        col[static_cast<size_t>(i)] = h->coo.val[static_cast<size_t>(p.cpl_src[static_cast<size_t>(q)])];
      }
    }
    for (auto& kv : cols) {
      std::vector<double>& y = kv.second;
      if (m > 1) {
        for (int32_t k = 0; k < m; ++k) {
          const double yk = y[static_cast<size_t>(k)];
          if (yk == 0.0) continue;
          for (int32_t i = k + 1; i < m; ++i) y[static_cast<size_t>(i)] -= lu[static_cast<size_t>(k) * m + i] * yk;
        }
      }
      for (int32_t i = 0; i < m; ++i) {
        if (y[static_cast<size_t>(i)] != 0.0) {
          h->u_r.push_back(s + i); h->u_c.push_back(kv.first); h->u_v.push_back(y[static_cast<size_t>(i)]);
        }
      }
    }
  }
  h->exP = rows;
  h->exported = true;
  return BDLU_OK;
}

extern "C" {

int64_t bdlu_export_p(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap) {
  if (!h) return -BDLU_NOT_PREPARED;
  if (const int st = bdlu_build_export(h)) return -st;
  const int32_t n = h->n;
  if (cap > 0)
    for (int32_t i = 0; i < n && i < cap; ++i) {
      if (rows) rows[i] = i;
      if (cols) cols[i] = h->exP[static_cast<size_t>(i)];
      if (vals) vals[i] = 1.0;
    }
  return n;
}

int64_t bdlu_export_q(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap) {
  if (!h) return -BDLU_NOT_PREPARED;
  if (const int st = bdlu_build_export(h)) return -st;
  const int32_t n = h->n;
  if (cap > 0)
    for (int32_t i = 0; i < n && i < cap; ++i) {
      if (rows) rows[i] = h->dec.Q[static_cast<size_t>(i)];
      if (cols) cols[i] = i;
      if (vals) vals[i] = 1.0;
    }
  return n;
}

static int64_t copy_coo(const std::vector<int32_t>& r, const std::vector<int32_t>& c, const std::vector<double>& v,
                        int32_t* rows, int32_t* cols, double* vals, int64_t cap) {
  const int64_t cnt = static_cast<int64_t>(r.size());
  const int64_t k = std::min<int64_t>(cnt, std::max<int64_t>(cap, 0));
  if (k > 0) {
    if (rows) std::memcpy(rows, r.data(), static_cast<size_t>(k) * sizeof(int32_t));
    if (cols) std::memcpy(cols, c.data(), static_cast<size_t>(k) * sizeof(int32_t));
    if (vals) std::memcpy(vals, v.data(), static_cast<size_t>(k) * sizeof(double));
  }
  return cnt;
}

int64_t bdlu_export_l(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap) {
  if (!h) return -BDLU_NOT_PREPARED;
  if (const int st = bdlu_build_export(h)) return -st;
  return copy_coo(h->l_r, h->l_c, h->l_v, rows, cols, vals, cap);
}

int64_t bdlu_export_u(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap) {
  if (!h) return -BDLU_NOT_PREPARED;
  if (const int st = bdlu_build_export(h)) return -st;
  return copy_coo(h->u_r, h->u_c, h->u_v, rows, cols, vals, cap);
}

int64_t bdlu_export_rearranged(bdlu_solver* h, int32_t* rows, int32_t* cols, double* vals, int64_t cap) {
  // A[pinv, qinv] in canonical entry order (solver.cpp:1665-1691), Rs = 1.
  if (!h) return -BDLU_NOT_PREPARED;
  if (const int st = bdlu_build_export(h)) return -st;
  const int64_t cnt = h->coo.nnz();
  if (cap > 0) {
    std::vector<int32_t> pinv(static_cast<size_t>(h->n));
    for (int32_t i = 0; i < h->n; ++i) pinv[static_cast<size_t>(h->exP[static_cast<size_t>(i)])] = i;
    for (int64_t k = 0; k < cnt && k < cap; ++k) {
      if (rows) rows[k] = pinv[static_cast<size_t>(h->coo.row[static_cast<size_t>(k)])];
      if (cols) cols[k] = h->dec.invQ[static_cast<size_t>(h->coo.col[static_cast<size_t>(k)])];
      if (vals) vals[k] = h->coo.val[static_cast<size_t>(k)];
    }
  }
  return cnt;
}

int32_t bdlu_get_block_lu(bdlu_solver* h, int32_t b, double* lu_rowmajor, int32_t* piv_out) {
  // The reference's dense micro-kernel factor of merged block b
  // (ubtf_block_solver.cpp:1450-1498), assembled from the unit factors: unit
  // LUs on the diagonal, the unit's L^{-1} P applied to the coupling columns
  // inside the block in the micro-kernel's own operation order (per element:
  // k ascending, multiply then subtract, no fused multiply-add), zeros in L
  // below other units.
  if (!h) return -BDLU_NOT_PREPARED;
  if (!h->factored) return -BDLU_NOT_PREPARED;
  if (const int st = bdlu_sync_host_values(h)) return -st;
  const auto& d = h->dec;
  if (b < 0 || b >= d.nblocks) return -BDLU_INVALID_INDEX;
  bdlu::Engine& eng = *h->engine;
  const bdlu::Plan& p = eng.plan();
  const int32_t b0 = d.R[static_cast<size_t>(b)], b1 = d.R[static_cast<size_t>(b) + 1];
  const int32_t M = b1 - b0;
  if (!lu_rowmajor && !piv_out) return M;
  std::vector<double> A(static_cast<size_t>(M) * M, 0.0);
  std::vector<int32_t> P(static_cast<size_t>(M), 0);
  std::string err;
  std::vector<double> lu;
  std::vector<int32_t> piv;
  // Local (row, col) -> value of the merged block's entries.
  for (int64_t q = d.diag_ptr[static_cast<size_t>(b)]; q < d.diag_ptr[static_cast<size_t>(b) + 1]; ++q)
    A[static_cast<size_t>(d.diag_row[static_cast<size_t>(q)]) * M + d.diag_col[static_cast<size_t>(q)]] =
        h->coo.val[static_cast<size_t>(d.diag_src[static_cast<size_t>(q)])];
  for (int32_t u = p.unit_of[static_cast<size_t>(b0)]; u < p.nunits && p.ustart[static_cast<size_t>(u)] < b1; ++u) {
    const int32_t s = p.ustart[static_cast<size_t>(u)] - b0;
    const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
    double scalar = 0.0;
    if (!eng.download_unit(u, lu, piv, scalar, err)) {
      bdlu_fail(h, BDLU_EXPORT_FAILED, err);
      return -BDLU_EXPORT_FAILED;
    }
    // Row swaps over the whole merged row (columns right of the unit move too).
    for (int32_t k = 0; k < m; ++k) {
      const int32_t pk = (m == 1) ? 0 : piv[static_cast<size_t>(k)];
      P[static_cast<size_t>(s + k)] = s + pk;
      if (pk != k)
        for (int32_t j = 0; j < M; ++j) std::swap(A[static_cast<size_t>(s + k) * M + j], A[static_cast<size_t>(s + pk) * M + j]);
    }
    for (int32_t i = 0; i < m; ++i)
      for (int32_t j = 0; j < m; ++j)
        A[static_cast<size_t>(s + i) * M + s + j] = (m == 1) ? scalar : lu[static_cast<size_t>(j) * m + i];
    // Coupling columns right of the unit: forward substitution with L_u.
    for (int32_t k = 0; k < m; ++k) {
      for (int32_t i = k + 1; i < m; ++i) {
        const double l = lu[static_cast<size_t>(k) * m + i];
        for (int32_t j = s + m; j < M; ++j) {
          A[static_cast<size_t>(s + i) * M + j] = A[static_cast<size_t>(s + i) * M + j] - l * A[static_cast<size_t>(s + k) * M + j];
        }
      }
    }
  }
  if (lu_rowmajor) std::memcpy(lu_rowmajor, A.data(), A.size() * sizeof(double));
  if (piv_out) std::memcpy(piv_out, P.data(), P.size() * sizeof(int32_t));
  return M;
}

}  // extern "C"
