/*
 * Oracle for the BlockDAGLU hot path: a plain-C CPU restatement of the
 * reference's numeric route, used only by tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg as the checker.  Nothing in the engine links or
 * calls it.
 *
 * Parity pinning: the reference's own tests pin the 3x3 golden solution
 * (blockdaglu/apps/tests/main.cpp:85-91, 111-128), the all-ones solutions of
 * cache_matrix (main.cpp:130-168, 197-204) and the P*A*Q = L*U identity
 * (main.cpp:170-195); tests/test_oracle.py checks this oracle against all of
 * them, and tests/test_oracle_ref.py checks it against the reference sources
 * compiled here (oracle/_ref, see oracle/Makefile).  KLU-factored blocks
 * (size > DENSE_BLOCK_MAX) have no reference arithmetic available here
 * (SuiteSparse is absent); the oracle factors every block with the dense
 * micro-kernel instead.
 *
 * Functions and the reference lines they restate:
 *   or_merge_block_boundaries  ubtf_block_solver.cpp:393-476
 *   or_split                   ubtf_block_solver.cpp:714-853 (offdiag CSR + block COO)
 *   or_levels                  ubtf_block_solver.cpp:857-909
 *   or_dense_lu                ubtf_block_solver.cpp:1450-1498 (= :2102-2135)
 *   or_dense_solve             ubtf_block_solver.cpp:2064-2100
 *   or_block_solve             ubtf_block_solver.cpp:2220-2414, 2548-2552 (reverse schedule)
 *   or_solve_system            solver.cpp:1352-1539 (first solve + refinement loop :1496-1536)
 *   or_metrics                 apps/benchmark/main.cpp:42-80 and the inf-norm residual
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_MIN(a, b) ((a) < (b) ? (a) : (b))
#define OR_MAX(a, b) ((a) > (b) ? (a) : (b))

/* ubtf_block_solver.cpp:393-476.  R has nR entries; writes the merged
 * boundaries to out (capacity nR) and returns their count. */
int32_t or_merge_block_boundaries(const int32_t* R, int32_t nR, int32_t n, int32_t merge_max, int32_t* out) {
  int32_t cnt = 0, nb, small_max, acc = 0, run_start = 0, run_end = 0, b;
  if (nR < 2 || nR - 1 <= 1) {
    out[0] = 0;
    out[1] = n;
    return 2;
  }
  nb = nR - 1;
  if (merge_max <= 0) merge_max = 64;
  small_max = OR_MAX(1, OR_MIN(merge_max, 32));
  out[cnt++] = 0;
#define OR_PUSH(v) do { if (out[cnt - 1] != (v)) out[cnt++] = (v); } while (0)
  for (b = 0; b < nb; ++b) {
    const int32_t s = R[b], e = R[b + 1], sz = e - s;
    if (sz <= small_max) {
      if (acc == 0) { run_start = s; run_end = e; acc = sz; continue; }
      if (acc + sz <= merge_max) { acc += sz; run_end = e; continue; }
      OR_PUSH(run_start); OR_PUSH(run_end);
      run_start = s; run_end = e; acc = sz;
      continue;
    }
    if (acc > 0) { OR_PUSH(run_start); OR_PUSH(run_end); acc = 0; }
    OR_PUSH(s); OR_PUSH(e);
  }
  if (acc > 0) { OR_PUSH(run_start); OR_PUSH(run_end); }
  OR_PUSH(n);
#undef OR_PUSH
  return cnt;
}

/* Dense micro-kernel, row-major m*m, in place (ubtf_block_solver.cpp:1450-1498):
 * pivot = first strict maximum of |a(i,k)| scanning i = k..m-1; fail on a zero
 * maximum; full-row swap; a(i,k) /= a(k,k); a(i,j) -= l(i,k) * a(k,j).
 * Returns 1 on success, 0 on a zero pivot. */
int or_dense_lu(double* a, int32_t* piv, int32_t m) {
  int32_t k, i, j;
  for (k = 0; k < m; ++k) {
    int32_t p = k;
    double best = fabs(a[(size_t)k * m + k]);
    for (i = k + 1; i < m; ++i) {
      const double v = fabs(a[(size_t)i * m + k]);
      if (v > best) { best = v; p = i; }
    }
    if (best == 0.0) return 0;
    piv[k] = p;
    if (p != k) {
      for (j = 0; j < m; ++j) {
        const double t = a[(size_t)k * m + j];
        a[(size_t)k * m + j] = a[(size_t)p * m + j];
        a[(size_t)p * m + j] = t;
      }
    }
    {
      const double akk = a[(size_t)k * m + k];
      for (i = k + 1; i < m; ++i) {
        double lik;
        a[(size_t)i * m + k] /= akk;
        lik = a[(size_t)i * m + k];
        for (j = k + 1; j < m; ++j) a[(size_t)i * m + j] -= lik * a[(size_t)k * m + j];
      }
    }
  }
  return 1;
}

/* ubtf_block_solver.cpp:2064-2100: row swaps, unit-L forward, U backward. */
int or_dense_solve(const double* lu, const int32_t* piv, int32_t m, double* rhs) {
  int32_t k, i, j;
  for (k = 0; k < m; ++k) {
    const int32_t p = piv[k];
    if (p != k) { const double t = rhs[k]; rhs[k] = rhs[p]; rhs[p] = t; }
  }
  for (i = 0; i < m; ++i) {
    double sum = rhs[i];
    for (j = 0; j < i; ++j) sum -= lu[(size_t)i * m + j] * rhs[j];
    rhs[i] = sum;
  }
  for (i = m - 1; i >= 0; --i) {
    double sum = rhs[i];
    double d;
    for (j = i + 1; j < m; ++j) sum -= lu[(size_t)i * m + j] * rhs[j];
    d = lu[(size_t)i * m + i];
    if (d == 0.0) return 0;
    rhs[i] = sum / d;
  }
  return 1;
}

/* A factored UBTF system (opaque to callers). */
typedef struct or_system {
  int32_t n, nblocks;
  int32_t *P, *Q, *invP, *invQ, *R, *block_of;
  int32_t *off_ptr, *off_col; double* off_val;   /* strictly upper CSR, permuted coordinates */
  int64_t *diag_ptr; int32_t *diag_r, *diag_c; double* diag_v;  /* per-block local COO */
  int64_t* lu_off; double* lu; int32_t* piv;      /* per-block row-major LU */
  int32_t failed_block;
  /* Canonical CSR for the residual. */
  int64_t nnz; int32_t *row, *col; double* val;
} or_system;

void or_free(or_system* s) {
  if (!s) return;
  free(s->P); free(s->Q); free(s->invP); free(s->invQ); free(s->R); free(s->block_of);
  free(s->off_ptr); free(s->off_col); free(s->off_val);
  free(s->diag_ptr); free(s->diag_r); free(s->diag_c); free(s->diag_v);
  free(s->lu_off); free(s->lu); free(s->piv);
  free(s->row); free(s->col); free(s->val);
  free(s);
}

/* UBTF split (ubtf_block_solver.cpp:714-853) of a canonical COO under (P, Q,
 * R).  Entries with |v| < drop are skipped.  Returns NULL when a lower-block
 * entry exists (the reference throws "permutation is not UBTF"). */
or_system* or_split(int32_t n, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
                    const int32_t* P, const int32_t* Q, const int32_t* R, int32_t nblocks, double drop) {
  or_system* s = (or_system*)calloc(1, sizeof(or_system));
  int32_t *rcnt, b, i;
  int64_t *dcnt, k, *dnext;
  int32_t* onext;
  s->n = n;
  s->nblocks = nblocks;
  s->failed_block = -1;
  s->P = (int32_t*)malloc(sizeof(int32_t) * n);
  s->Q = (int32_t*)malloc(sizeof(int32_t) * n);
  s->invP = (int32_t*)malloc(sizeof(int32_t) * n);
  s->invQ = (int32_t*)malloc(sizeof(int32_t) * n);
  s->R = (int32_t*)malloc(sizeof(int32_t) * (nblocks + 1));
  s->block_of = (int32_t*)malloc(sizeof(int32_t) * n);
  memcpy(s->P, P, sizeof(int32_t) * n);
  memcpy(s->Q, Q, sizeof(int32_t) * n);
  memcpy(s->R, R, sizeof(int32_t) * (nblocks + 1));
  for (i = 0; i < n; ++i) { s->invP[P[i]] = i; s->invQ[Q[i]] = i; }
  for (b = 0; b < nblocks; ++b)
    for (i = R[b]; i < R[b + 1]; ++i) s->block_of[i] = b;
  rcnt = (int32_t*)calloc(n, sizeof(int32_t));
  dcnt = (int64_t*)calloc(nblocks, sizeof(int64_t));
  for (k = 0; k < nnz; ++k) {
    int32_t rp, cp, br, bc;
    if (drop > 0.0 && fabs(val[k]) < drop) continue;
    rp = s->invP[row[k]]; cp = s->invQ[col[k]];
    br = s->block_of[rp]; bc = s->block_of[cp];
    if (bc < br) { free(rcnt); free(dcnt); or_free(s); return NULL; }
    if (bc == br) dcnt[br]++;
    else rcnt[rp]++;
  }
  s->off_ptr = (int32_t*)malloc(sizeof(int32_t) * (n + 1));
  s->off_ptr[0] = 0;
  for (i = 0; i < n; ++i) s->off_ptr[i + 1] = s->off_ptr[i] + rcnt[i];
  s->diag_ptr = (int64_t*)malloc(sizeof(int64_t) * (nblocks + 1));
  s->diag_ptr[0] = 0;
  for (b = 0; b < nblocks; ++b) s->diag_ptr[b + 1] = s->diag_ptr[b] + dcnt[b];
  s->off_col = (int32_t*)malloc(sizeof(int32_t) * (s->off_ptr[n] + 1));
  s->off_val = (double*)malloc(sizeof(double) * (s->off_ptr[n] + 1));
  s->diag_r = (int32_t*)malloc(sizeof(int32_t) * (s->diag_ptr[nblocks] + 1));
  s->diag_c = (int32_t*)malloc(sizeof(int32_t) * (s->diag_ptr[nblocks] + 1));
  s->diag_v = (double*)malloc(sizeof(double) * (s->diag_ptr[nblocks] + 1));
  onext = (int32_t*)malloc(sizeof(int32_t) * n);
  dnext = (int64_t*)malloc(sizeof(int64_t) * nblocks);
  memcpy(onext, s->off_ptr, sizeof(int32_t) * n);
  memcpy(dnext, s->diag_ptr, sizeof(int64_t) * nblocks);
  for (k = 0; k < nnz; ++k) {
    int32_t rp, cp, br, bc;
    if (drop > 0.0 && fabs(val[k]) < drop) continue;
    rp = s->invP[row[k]]; cp = s->invQ[col[k]];
    br = s->block_of[rp]; bc = s->block_of[cp];
    if (bc == br) {
      const int64_t q = dnext[br]++;
      s->diag_r[q] = rp - R[br]; s->diag_c[q] = cp - R[br]; s->diag_v[q] = val[k];
    } else {
      const int32_t q = onext[rp]++;
      s->off_col[q] = cp; s->off_val[q] = val[k];
    }
  }
  free(rcnt); free(dcnt); free(onext); free(dnext);
  s->nnz = nnz;
  s->row = (int32_t*)malloc(sizeof(int32_t) * (nnz + 1));
  s->col = (int32_t*)malloc(sizeof(int32_t) * (nnz + 1));
  s->val = (double*)malloc(sizeof(double) * (nnz + 1));
  memcpy(s->row, row, sizeof(int32_t) * nnz);
  memcpy(s->col, col, sizeof(int32_t) * nnz);
  memcpy(s->val, val, sizeof(double) * nnz);
  return s;
}

/* ubtf_block_solver.cpp:857-909: deps in first-appearance order, levels. */
void or_levels(const or_system* s, int32_t* level, int32_t* max_level) {
  int32_t b, r, p, mx = 0;
  int32_t* seen = (int32_t*)malloc(sizeof(int32_t) * s->nblocks);
  int32_t* deps = (int32_t*)malloc(sizeof(int32_t) * (s->off_ptr[s->n] + 1));
  int64_t* dptr = (int64_t*)malloc(sizeof(int64_t) * (s->nblocks + 1));
  int64_t nd = 0;
  for (b = 0; b < s->nblocks; ++b) seen[b] = -1;
  for (b = 0; b < s->nblocks; ++b) {
    const int32_t st = s->R[b], en = s->R[b + 1];
    dptr[b] = nd;
    for (r = st; r < en; ++r)
      for (p = s->off_ptr[r]; p < s->off_ptr[r + 1]; ++p) {
        const int32_t c = s->off_col[p];
        if (c >= en) {
          const int32_t bc = s->block_of[c];
          if (bc > b && seen[bc] != b) { seen[bc] = b; deps[nd++] = bc; }
        }
      }
  }
  dptr[s->nblocks] = nd;
  for (b = s->nblocks - 1; b >= 0; --b) {
    int32_t lev = 0;
    int64_t q;
    for (q = dptr[b]; q < dptr[b + 1]; ++q) lev = OR_MAX(lev, level[deps[q]] + 1);
    level[b] = lev;
    mx = OR_MAX(mx, lev);
  }
  *max_level = mx;
  free(seen); free(deps); free(dptr);
}

/* Factors every block with the dense micro-kernel (factor_one_block's dense
 * branch, ubtf_block_solver.cpp:1450-1498).  Returns 1, or 0 with
 * failed_block set. */
int or_factor(or_system* s) {
  int32_t b;
  int64_t total = 0;
  s->lu_off = (int64_t*)malloc(sizeof(int64_t) * (s->nblocks + 1));
  for (b = 0; b < s->nblocks; ++b) {
    const int64_t m = s->R[b + 1] - s->R[b];
    s->lu_off[b] = total;
    total += m * m;
  }
  s->lu_off[s->nblocks] = total;
  s->lu = (double*)calloc((size_t)(total + 1), sizeof(double));
  s->piv = (int32_t*)calloc((size_t)s->n + 1, sizeof(int32_t));
  for (b = 0; b < s->nblocks; ++b) {
    const int32_t m = s->R[b + 1] - s->R[b];
    double* a = s->lu + s->lu_off[b];
    int64_t q;
    for (q = s->diag_ptr[b]; q < s->diag_ptr[b + 1]; ++q) a[(size_t)s->diag_r[q] * m + s->diag_c[q]] += s->diag_v[q];
    if (!or_dense_lu(a, s->piv + s->R[b], m)) { s->failed_block = b; return 0; }
  }
  return 1;
}

/* or_gp_lu / or_gp_gate (gp_oracle.c). */
typedef struct or_gp_stats { int32_t ok, row_swaps, tiny_pivots, zero_pivots; double min_abs_diag; } or_gp_stats;
int or_gp_lu(int32_t m, const int32_t* col_ptr, const int32_t* row_ind, const double* val, int32_t scale,
             double diag_prefer_tol, double pivot_tol, double perturb, double drop_tol, double* lu, int32_t* piv,
             double* row_scale, or_gp_stats* st);
int or_gp_gate(const or_gp_stats* st, int32_t m, int32_t require_no_swaps, int32_t swap_max_n, int32_t swap_max,
               int32_t require_no_tiny, double min_abs_diag);

/* Factors every block as factor_one_block does with the sparse-LU route on
 * (USERALGO_SPARSE_LU_KERNEL=gp, ubtf_block_solver.cpp:1439-1498 and
 * :1749-1773) under the default gate: blocks of at most dense_max rows by the
 * dense micro-kernel; blocks of up to gp_max_n rows by or_gp_lu (no scaling,
 * no dropping), kept when the gate accepts it (no row swaps, no tiny pivots,
 * smallest |pivot| >= min_abs_diag); every other block by the dense
 * partial-pivoting micro-kernel, the stand-in for the reference's KLU.
 * Accepted factors are stored like dense ones (row-major LU, LAPACK-style
 * pivots), so the block solve is or_dense_solve: a row-oriented sweep in
 * ascending column order, the order of gp_lu_solve_inplace_strided
 * (gp_lu.cpp:242-306).  reason[b] = -1 (not tried) or the gate's reason.
 * Returns 1, or 0 with failed_block set. */
int or_factor_gp(or_system* s, int32_t dense_max, int32_t gp_max_n, double diag_tol, double pivot_tol,
                 double perturb, double min_abs_diag, int32_t* reason) {
  int32_t b;
  int64_t total = 0;
  s->lu_off = (int64_t*)malloc(sizeof(int64_t) * (s->nblocks + 1));
  for (b = 0; b < s->nblocks; ++b) {
    const int64_t m = s->R[b + 1] - s->R[b];
    s->lu_off[b] = total;
    total += m * m;
  }
  s->lu_off[s->nblocks] = total;
  s->lu = (double*)calloc((size_t)(total + 1), sizeof(double));
  s->piv = (int32_t*)calloc((size_t)s->n + 1, sizeof(int32_t));
  for (b = 0; b < s->nblocks; ++b) {
    const int32_t m = s->R[b + 1] - s->R[b];
    double* a = s->lu + s->lu_off[b];
    int64_t q;
    reason[b] = -1;
    if (m > dense_max && m <= gp_max_n) {
      /* Block CSC (coo_to_csc_i32) and the sparse LU with its gate. */
      int32_t* cp = (int32_t*)calloc((size_t)m + 1, sizeof(int32_t));
      const int64_t cnt = s->diag_ptr[b + 1] - s->diag_ptr[b];
      int32_t* ri = (int32_t*)malloc(sizeof(int32_t) * (size_t)(cnt + 1));
      double* rv = (double*)malloc(sizeof(double) * (size_t)(cnt + 1));
      double* rs = (double*)malloc(sizeof(double) * (size_t)m);
      int32_t* nx = (int32_t*)malloc(sizeof(int32_t) * (size_t)m);
      or_gp_stats st;
      int32_t c;
      for (q = s->diag_ptr[b]; q < s->diag_ptr[b + 1]; ++q) cp[s->diag_c[q] + 1]++;
      for (c = 0; c < m; ++c) cp[c + 1] += cp[c];
      memcpy(nx, cp, sizeof(int32_t) * (size_t)m);
      for (q = s->diag_ptr[b]; q < s->diag_ptr[b + 1]; ++q) {
        const int32_t k = nx[s->diag_c[q]]++;
        ri[k] = s->diag_r[q];
        rv[k] = s->diag_v[q];
      }
      or_gp_lu(m, cp, ri, rv, 0, diag_tol, pivot_tol, perturb, 0.0, a, s->piv + s->R[b], rs, &st);
      reason[b] = or_gp_gate(&st, m, 1, 256, 0, 1, min_abs_diag);
      free(cp); free(ri); free(rv); free(rs); free(nx);
      if (reason[b] == 0) continue;
      memset(a, 0, sizeof(double) * (size_t)m * (size_t)m);
    }
    for (q = s->diag_ptr[b]; q < s->diag_ptr[b + 1]; ++q) a[(size_t)s->diag_r[q] * m + s->diag_c[q]] += s->diag_v[q];
    if (!or_dense_lu(a, s->piv + s->R[b], m)) { s->failed_block = b; return 0; }
  }
  return 1;
}

const double* or_block_lu(const or_system* s, int32_t b, const int32_t** piv, int32_t* m) {
  *m = s->R[b + 1] - s->R[b];
  *piv = s->piv + s->R[b];
  return s->lu + s->lu_off[b];
}

/* solve_ubtf, reverse schedule (ubtf_block_solver.cpp:2220-2414, 2548-2552). */
int or_block_solve(const or_system* s, double* b) {
  if (!s->lu) return 0; /* not factored (or_factor first) */
  const int32_t n = s->n;
  double* bperm = (double*)malloc(sizeof(double) * n);
  double* xperm = (double*)calloc(n, sizeof(double));
  double* rhs = (double*)malloc(sizeof(double) * (n + 1));
  int32_t i, bid, ok = 1;
  for (i = 0; i < n; ++i) bperm[i] = b[s->P[i]];
  for (bid = s->nblocks - 1; bid >= 0 && ok; --bid) {
    const int32_t st = s->R[bid], m = s->R[bid + 1] - st;
    int32_t r, p;
    for (r = st; r < st + m; ++r) {
      double v = bperm[r];
      for (p = s->off_ptr[r]; p < s->off_ptr[r + 1]; ++p) v -= s->off_val[p] * xperm[s->off_col[p]];
      rhs[r - st] = v;
    }
    ok = or_dense_solve(s->lu + s->lu_off[bid], s->piv + st, m, rhs);
    for (i = 0; i < m; ++i) xperm[st + i] = rhs[i];
  }
  if (ok)
    for (i = 0; i < n; ++i) b[s->Q[i]] = xperm[i];
  free(bperm); free(xperm); free(rhs);
  return ok;
}

static double or_norm2(const double* v, int32_t n) {
  double s = 0.0;
  int32_t i;
  for (i = 0; i < n; ++i) s += v[i] * v[i];
  return sqrt(s);
}

/* Solver::solve_in_place: first solve, then up to max_iters refinement steps
 * r = b0 - A x over the canonical COO, stop at |r|_2/|b0|_2 < 1e-12
 * (solver.cpp:1496-1536).  Returns the number of refinement solves taken, or
 * -1 on failure. */
int or_solve_system(const or_system* s, double* b, int max_iters) {
  const int32_t n = s->n;
  double *b0 = NULL, *r = NULL, bnorm;
  int it, taken = 0;
  if (max_iters > 0) {
    b0 = (double*)malloc(sizeof(double) * n);
    memcpy(b0, b, sizeof(double) * n);
  }
  if (!or_block_solve(s, b)) { free(b0); return -1; }
  if (max_iters <= 0) return 0;
  bnorm = or_norm2(b0, n);
  if (bnorm == 0.0) { free(b0); return 0; }
  r = (double*)malloc(sizeof(double) * n);
  for (it = 0; it < max_iters; ++it) {
    int64_t k;
    int32_t i;
    memcpy(r, b0, sizeof(double) * n);
    for (k = 0; k < s->nnz; ++k) r[s->row[k]] -= s->val[k] * b[s->col[k]];
    if (or_norm2(r, n) / bnorm < 1e-12) break;
    if (!or_block_solve(s, r)) { taken = -1; break; }
    for (i = 0; i < n; ++i) b[i] += r[i];
    ++taken;
  }
  free(b0); free(r);
  return taken;
}

/* out[0] = |Ax-b|_inf / (|A|_inf |x|_inf + |b|_inf)
 * out[1] = |b - Ax|_2 / |b|_2          (apps/benchmark/main.cpp:55-80)
 * out[2] = |x - x_true|_2 / |x_true|_2 (apps/benchmark/main.cpp:42-53; 0 if x_true NULL) */
void or_metrics(int32_t n, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
                const double* x, const double* b, const double* x_true, double* out) {
  double* ax = (double*)calloc(n, sizeof(double));
  double* arow = (double*)calloc(n, sizeof(double));
  double rinf = 0, binf = 0, xinf = 0, ainf = 0, r2 = 0, b2 = 0, e2 = 0, t2 = 0;
  int64_t k;
  int32_t i;
  for (k = 0; k < nnz; ++k) {
    ax[row[k]] += val[k] * x[col[k]];
    arow[row[k]] += fabs(val[k]);
  }
  for (i = 0; i < n; ++i) {
    const double r = b[i] - ax[i];
    rinf = OR_MAX(rinf, fabs(r));
    binf = OR_MAX(binf, fabs(b[i]));
    xinf = OR_MAX(xinf, fabs(x[i]));
    ainf = OR_MAX(ainf, arow[i]);
    r2 += r * r;
    b2 += b[i] * b[i];
    if (x_true) {
      const double e = x[i] - x_true[i];
      e2 += e * e;
      t2 += x_true[i] * x_true[i];
    }
  }
  out[0] = (ainf * xinf + binf) > 0 ? rinf / (ainf * xinf + binf) : rinf;
  out[1] = b2 > 0 ? sqrt(r2) / sqrt(b2) : sqrt(r2);
  out[2] = (x_true && t2 > 0) ? sqrt(e2) / sqrt(t2) : 0.0;
  free(ax); free(arow);
}

int32_t or_failed_block(const or_system* s) { return s->failed_block; }
int32_t or_nblocks(const or_system* s) { return s->nblocks; }
int32_t or_offdiag_nnz(const or_system* s) { return s->off_ptr[s->n]; }
void or_get_offdiag(const or_system* s, int32_t* ptr, int32_t* col, double* val) {
  if (ptr) memcpy(ptr, s->off_ptr, sizeof(int32_t) * (s->n + 1));
  if (col) memcpy(col, s->off_col, sizeof(int32_t) * s->off_ptr[s->n]);
  if (val) memcpy(val, s->off_val, sizeof(double) * s->off_ptr[s->n]);
}
