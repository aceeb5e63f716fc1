/* Oracle (test infrastructure only): C restatement of the reference's
 * row-wise sparse LU ("Gilbert-Peierls" route) and of its acceptance gate.
 *
 *   or_gp_lu    follows gp_lu_factor      (blockdaglu/src/gp_lu.cpp:84-240)
 *   or_gp_gate  follows gp_gate_eval      (blockdaglu/src/ubtf_block_solver.cpp:197-235)
 *
 * The active matrix is held densely with a structural-presence flag per
 * entry, which reproduces the reference's sorted (col, val) rows exactly:
 * an entry exists where the reference's row holds it, a fill entry is
 * created as (-l) * u, an existing one becomes v - l * u, and column k is
 * dropped from every row it is eliminated from.  Built with
 * -ffp-contract=off so no multiply-add is fused, as in the reference's x86-64
 * build.  Only tests and the bench's CPU legs call this file. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Outputs of or_gp_lu. */
typedef struct or_gp_stats {
  int32_t ok;             /* gp_lu_factor's return value */
  int32_t row_swaps;      /* GpLuFactor::row_swap_count */
  int32_t tiny_pivots;    /* tiny_pivot_count */
  int32_t zero_pivots;    /* zero_pivot_count */
  double min_abs_diag;    /* gp_min_abs_diag_of (ubtf_block_solver.cpp:190-195) */
} or_gp_stats;

/* Sparse LU of the m x m CSC matrix (col_ptr, row_ind, val), options as
 * GpLuOptions (gp_lu.h:43-49): scale 0/1/2, diag_prefer_tol, pivot_tol,
 * perturb, drop_tol.  Outputs: lu (row-major m*m: L multipliers strictly
 * below the diagonal, U on and above, zeros where the reference stores no
 * entry), piv (LAPACK style: at step k rows k and piv[k] were swapped),
 * row_scale (m, 1.0 when scaling is off), stats.  Returns stats->ok. */
int or_gp_lu(int32_t m, const int32_t* col_ptr, const int32_t* row_ind, const double* val, int32_t scale,
             double diag_prefer_tol, double pivot_tol, double perturb, double drop_tol, double* lu, int32_t* piv,
             double* row_scale, or_gp_stats* st) {
  const size_t mm = (size_t)m * (size_t)m;
  unsigned char* pres = NULL;
  int32_t i, j, k, c;
  int64_t p;
  const double ptol = pivot_tol > 0.0 ? pivot_tol : 0.0;
  const double pert = perturb > 0.0 ? perturb : 0.0;
  memset(st, 0, sizeof(*st));
  if (m <= 0 || scale < 0 || scale > 2 || diag_prefer_tol < 0.0) return 0;
  memset(lu, 0, sizeof(double) * mm);
  for (i = 0; i < m; ++i) { piv[i] = i; row_scale[i] = 1.0; }
  /* Row scaling in original row order (gp_lu.cpp:104-119). */
  if (scale != 0) {
    double* acc = (double*)calloc((size_t)m, sizeof(double));
    for (p = 0; p < col_ptr[m]; ++p) {
      const int32_t r = row_ind[p];
      const double a = fabs(val[p]);
      if (r < 0 || r >= m) continue;
      if (scale == 1) acc[r] += a;
      else if (a > acc[r]) acc[r] = a;
    }
    for (i = 0; i < m; ++i) row_scale[i] = acc[i] > 0.0 ? 1.0 / acc[i] : 1.0;
    free(acc);
  }
  /* Active rows (gp_lu.cpp:121-146): duplicates summed, optional initial drop. */
  pres = (unsigned char*)calloc(mm, 1);
  for (c = 0; c < m; ++c)
    for (p = col_ptr[c]; p < col_ptr[c + 1]; ++p) {
      const int32_t r = row_ind[p];
      double v = val[p];
      if (r < 0 || r >= m) continue;
      if (scale != 0) v *= row_scale[r];
      if (pres[(size_t)r * m + c]) lu[(size_t)r * m + c] += v;
      else { lu[(size_t)r * m + c] = v; pres[(size_t)r * m + c] = 1; }
    }
  if (drop_tol > 0.0)
    for (p = 0; p < (int64_t)mm; ++p)
      if (pres[p] && !(fabs(lu[p]) > drop_tol)) { pres[p] = 0; lu[p] = 0.0; }

  for (k = 0; k < m; ++k) {
    int32_t pv = -1, has_diag = 0;
    double best = 0.0, diagabs = 0.0, diag;
    /* Pivot search over rows k..m-1 holding column k (gp_lu.cpp:164-181). */
    for (i = k; i < m; ++i) {
      double a;
      if (!pres[(size_t)i * m + k]) continue;
      a = fabs(lu[(size_t)i * m + k]);
      if (a > best) { best = a; pv = i; }
      if (i == k) { has_diag = 1; diagabs = a; }
    }
    if (pv < 0) { st->zero_pivots++; goto fail; }
    /* Diagonal preference (gp_lu.cpp:188-190). */
    if (has_diag && best > 0.0 && diagabs >= diag_prefer_tol * best) pv = k;
    if (pv != k) {
      /* The active row and its L multipliers move together (gp_lu.cpp:192-197). */
      for (j = 0; j < m; ++j) {
        const double t = lu[(size_t)k * m + j];
        const unsigned char f = pres[(size_t)k * m + j];
        lu[(size_t)k * m + j] = lu[(size_t)pv * m + j];
        lu[(size_t)pv * m + j] = t;
        pres[(size_t)k * m + j] = pres[(size_t)pv * m + j];
        pres[(size_t)pv * m + j] = f;
      }
      piv[k] = pv;
      st->row_swaps++;
    }
    if (!pres[(size_t)k * m + k]) { st->zero_pivots++; goto fail; }
    diag = lu[(size_t)k * m + k];
    /* Tiny pivots are perturbed away from zero (gp_lu.cpp:205-212). */
    if (ptol > 0.0 && fabs(diag) < ptol) {
      const double d = pert != 0.0 ? pert : ptol;
      st->tiny_pivots++;
      if (diag == 0.0) diag = d;
      else diag += diag > 0.0 ? d : -d;
      lu[(size_t)k * m + k] = diag;
    }
    if (diag == 0.0) { st->zero_pivots++; goto fail; }
    /* Eliminate rows below (gp_lu.cpp:222-231 and saxpy_inplace :35-77). */
    for (i = k + 1; i < m; ++i) {
      double l;
      if (!pres[(size_t)i * m + k]) continue;
      l = lu[(size_t)i * m + k] / diag;
      /* Column k leaves the active row; the multiplier is kept if nonzero. */
      pres[(size_t)i * m + k] = 0;
      lu[(size_t)i * m + k] = l != 0.0 ? l : 0.0;
      for (c = k + 1; c < m; ++c) {
        const size_t ic = (size_t)i * m + c;
        double v;
        if (!pres[(size_t)k * m + c]) continue;
        v = pres[ic] ? lu[ic] - l * lu[(size_t)k * m + c] : (-l) * lu[(size_t)k * m + c];
        if (drop_tol > 0.0 && fabs(v) <= drop_tol) { pres[ic] = 0; lu[ic] = 0.0; continue; }
        pres[ic] = 1;
        lu[ic] = v;
      }
      /* Existing entries the pivot row does not hold can still be dropped
       * by drop_tol (saxpy_inplace rewrites the whole row). */
      if (drop_tol > 0.0)
        for (c = k + 1; c < m; ++c) {
          const size_t ic = (size_t)i * m + c;
          if (pres[ic] && !pres[(size_t)k * m + c] && fabs(lu[ic]) <= drop_tol) { pres[ic] = 0; lu[ic] = 0.0; }
        }
    }
  }
  free(pres);
  {
    double mn = INFINITY;
    for (k = 0; k < m; ++k) mn = fmin(mn, fabs(lu[(size_t)k * m + k]));
    st->min_abs_diag = isfinite(mn) ? mn : 0.0;
  }
  st->ok = 1;
  return 1;
fail:
  free(pres);
  return 0;
}

/* The gate (ubtf_block_solver.cpp:197-235).  Returns the reject reason:
 * 0 accepted, 1 factor failed, 2 row swaps, 3 tiny pivots, 4 smallest
 * |pivot| below min_abs_diag. */
int or_gp_gate(const or_gp_stats* st, int32_t m, int32_t require_no_swaps, int32_t swap_max_n, int32_t swap_max,
               int32_t require_no_tiny, double min_abs_diag) {
  if (!st->ok) return 1;
  if (require_no_swaps && st->row_swaps != 0) {
    const int allowed = swap_max_n > 0 && swap_max > 0 && m > 0 && m <= swap_max_n && st->row_swaps <= swap_max;
    if (!allowed) return 2;
  }
  if (require_no_tiny && st->tiny_pivots != 0) return 3;
  if (min_abs_diag > 0.0 && !(st->min_abs_diag >= min_abs_diag)) return 4;
  return 0;
}
