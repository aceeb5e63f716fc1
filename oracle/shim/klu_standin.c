/*
 * Stand-in implementation of the KLU calls the reference makes, for building
 * the reference's own sources as an oracle here (SuiteSparse absent).  It is a
 * dense threshold-partial-pivoting LU on the CSC input: the diagonal is kept
 * when |a_kk| >= tol * max_i |a_ik| (KLU's documented tol rule, default
 * 0.001), otherwise the first maximal row is taken; optional row scaling by
 * row sums (scale 1) or row maxima (scale 2); no fill-reducing ordering and
 * no inner BTF (one block).  rcond is min|u_kk| / max|u_kk| as KLU reports it.
 * Matrices larger than 16384 are refused with KLU_TOO_LARGE.  Test
 * infrastructure only.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "suitesparse/klu.h"

#define STANDIN_MAX_N 16384

int klu_defaults(klu_common* c) {
  if (!c) return 0;
  memset(c, 0, sizeof(*c));
  c->tol = 0.001;
  c->btf = 1;
  c->ordering = 0;
  c->scale = 2;
  c->halt_if_singular = 1;
  c->status = KLU_OK;
  c->rcond = 0.0;
  return 1;
}

static klu_symbolic* make_symbolic(int32_t n) {
  klu_symbolic* s = (klu_symbolic*)calloc(1, sizeof(klu_symbolic));
  int32_t i;
  if (!s) return NULL;
  s->n = n;
  s->nblocks = 1;
  s->P = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  s->Q = (int32_t*)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
  s->R = (int32_t*)malloc(sizeof(int32_t) * 2);
  for (i = 0; i < n; ++i) s->P[i] = s->Q[i] = i;
  s->R[0] = 0;
  s->R[1] = n;
  return s;
}

klu_symbolic* klu_analyze(int32_t n, int32_t* Ap, int32_t* Ai, klu_common* c) {
  (void)Ap;
  (void)Ai;
  if (n <= 0) {
    if (c) c->status = KLU_INVALID;
    return NULL;
  }
  if (c) c->status = KLU_OK;
  return make_symbolic(n);
}

klu_symbolic* klu_analyze_given(int32_t n, int32_t* Ap, int32_t* Ai, int32_t* P, int32_t* Q, klu_common* c) {
  (void)P;
  (void)Q;
  return klu_analyze(n, Ap, Ai, c);
}

klu_numeric* klu_factor(int32_t* Ap, int32_t* Ai, double* Ax, klu_symbolic* sym, klu_common* c) {
  const int32_t n = sym ? sym->n : 0;
  klu_numeric* num;
  double *a, *rs, umin = INFINITY, umax = 0.0;
  int32_t j, k, i, *perm, *where;
  const double tol = (c && c->tol >= 0.0 && c->tol <= 1.0) ? c->tol : 0.001;
  const int scale = c ? c->scale : 0;
  if (n <= 0) {
    if (c) c->status = KLU_INVALID;
    return NULL;
  }
  if (n > STANDIN_MAX_N) {
    if (c) c->status = KLU_TOO_LARGE;
    return NULL;
  }
  a = (double*)calloc((size_t)n * n, sizeof(double));
  rs = (double*)malloc(sizeof(double) * n);
  perm = (int32_t*)malloc(sizeof(int32_t) * n);
  where = (int32_t*)malloc(sizeof(int32_t) * n);
  if (!a || !rs || !perm || !where) {
    free(a); free(rs); free(perm); free(where);
    if (c) c->status = KLU_OUT_OF_MEMORY;
    return NULL;
  }
  for (i = 0; i < n; ++i) rs[i] = (scale == 1 || scale == 2) ? 0.0 : 1.0;
  for (j = 0; j < n; ++j)
    for (k = Ap[j]; k < Ap[j + 1]; ++k) {
      a[(size_t)j * n + Ai[k]] += Ax[k];
      if (scale == 1) rs[Ai[k]] += fabs(Ax[k]);
      else if (scale == 2 && fabs(Ax[k]) > rs[Ai[k]]) rs[Ai[k]] = fabs(Ax[k]);
    }
  for (i = 0; i < n; ++i)
    if (rs[i] == 0.0) rs[i] = 1.0;
  if (scale == 1 || scale == 2)
    for (j = 0; j < n; ++j)
      for (i = 0; i < n; ++i) a[(size_t)j * n + i] /= rs[i];
  for (i = 0; i < n; ++i) perm[i] = i;
  for (k = 0; k < n; ++k) {
    double* ck = a + (size_t)k * n;
    int32_t p = k;
    double best = fabs(ck[k]);
    for (i = k + 1; i < n; ++i)
      if (fabs(ck[i]) > best) { best = fabs(ck[i]); p = i; }
    if (best == 0.0) {
      free(a); free(rs); free(perm); free(where);
      if (c) { c->status = KLU_SINGULAR; c->numerical_rank = k; }
      return NULL;
    }
    if (fabs(ck[k]) >= tol * best) p = k;
    if (p != k) {
      int32_t t = perm[k];
      perm[k] = perm[p];
      perm[p] = t;
      for (j = 0; j < n; ++j) {
        const double v = a[(size_t)j * n + k];
        a[(size_t)j * n + k] = a[(size_t)j * n + p];
        a[(size_t)j * n + p] = v;
      }
    }
    {
      const double d = ck[k];
      for (i = k + 1; i < n; ++i) ck[i] /= d;
      for (j = k + 1; j < n; ++j) {
        double* cj = a + (size_t)j * n;
        const double u = cj[k];
        if (u == 0.0) continue;
        for (i = k + 1; i < n; ++i) cj[i] -= ck[i] * u;
      }
      if (fabs(d) < umin) umin = fabs(d);
      if (fabs(d) > umax) umax = fabs(d);
    }
  }
  num = (klu_numeric*)calloc(1, sizeof(klu_numeric));
  num->n = n;
  num->lu = a;
  num->perm = perm;
  num->rs = rs;
  num->nzoff = 0;
  num->lnz = n;
  num->unz = 0;
  for (j = 0; j < n; ++j)
    for (i = 0; i < n; ++i) {
      const double v = a[(size_t)j * n + i];
      if (i > j && v != 0.0) num->lnz++;
      if (i <= j && (v != 0.0 || i == j)) num->unz++;
    }
  free(where);
  if (c) {
    c->status = KLU_OK;
    c->numerical_rank = n;
    c->rcond = umax > 0.0 ? umin / umax : 0.0;
  }
  return num;
}

int klu_solve(klu_symbolic* sym, klu_numeric* num, int32_t ldim, int32_t nrhs, double* B, klu_common* c) {
  const int32_t n = num ? num->n : 0;
  double* y;
  int32_t r, i, j;
  (void)sym;
  if (!num || !B || ldim < n || nrhs < 0) {
    if (c) c->status = KLU_INVALID;
    return 0;
  }
  y = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (r = 0; r < nrhs; ++r) {
    double* b = B + (size_t)r * ldim;
    for (i = 0; i < n; ++i) y[i] = b[num->perm[i]] / num->rs[num->perm[i]];
    for (j = 0; j < n; ++j) {
      const double yj = y[j];
      const double* cj = num->lu + (size_t)j * n;
      if (yj != 0.0)
        for (i = j + 1; i < n; ++i) y[i] -= cj[i] * yj;
    }
    for (j = n - 1; j >= 0; --j) {
      const double* cj = num->lu + (size_t)j * n;
      const double yj = y[j] / cj[j];
      y[j] = yj;
      if (yj != 0.0)
        for (i = 0; i < j; ++i) y[i] -= cj[i] * yj;
    }
    memcpy(b, y, sizeof(double) * n);
  }
  free(y);
  if (c) c->status = KLU_OK;
  return 1;
}

int klu_extract(klu_numeric* num, klu_symbolic* sym, int32_t* Lp, int32_t* Li, double* Lx, int32_t* Up, int32_t* Ui,
                double* Ux, int32_t* Fp, int32_t* Fi, double* Fx, int32_t* P, int32_t* Q, double* Rs, int32_t* R,
                klu_common* c) {
  const int32_t n = num ? num->n : 0;
  int32_t i, j, lp = 0, up = 0;
  (void)sym;
  (void)Fi;
  (void)Fx;
  if (!num) return 0;
  for (j = 0; j < n; ++j) {
    if (Lp) Lp[j] = lp;
    if (Up) Up[j] = up;
    for (i = 0; i < n; ++i) {
      const double v = num->lu[(size_t)j * n + i];
      if (i == j) {
        if (Li) Li[lp] = j;
        if (Lx) Lx[lp] = 1.0;
        ++lp;
      }
      if (i > j && v != 0.0) {
        if (Li) Li[lp] = i;
        if (Lx) Lx[lp] = v;
        ++lp;
      }
      if (i <= j && (v != 0.0 || i == j)) {
        if (Ui) Ui[up] = i;
        if (Ux) Ux[up] = v;
        ++up;
      }
    }
  }
  if (Lp) Lp[n] = lp;
  if (Up) Up[n] = up;
  if (Fp)
    for (j = 0; j <= n; ++j) Fp[j] = 0;
  for (i = 0; i < n; ++i) {
    if (P) P[i] = num->perm[i];
    if (Q) Q[i] = i;
    /* The reference divides row new_row of A[pinv, qinv] by Rs[new_row]
     * (solver.cpp:1684-1687), so scale factors are returned in factor order. */
    if (Rs) Rs[i] = num->rs[num->perm[i]];
  }
  if (R) {
    R[0] = 0;
    R[1] = n;
  }
  if (c) c->status = KLU_OK;
  return 1;
}

int klu_free_symbolic(klu_symbolic** s, klu_common* c) {
  (void)c;
  if (s && *s) {
    free((*s)->P);
    free((*s)->Q);
    free((*s)->R);
    free(*s);
    *s = NULL;
  }
  return 1;
}

int klu_free_numeric(klu_numeric** nm, klu_common* c) {
  (void)c;
  if (nm && *nm) {
    free((*nm)->lu);
    free((*nm)->perm);
    free((*nm)->rs);
    free(*nm);
    *nm = NULL;
  }
  return 1;
}
