/*
 * Seeded synthetic systems for the oracle side (test infrastructure): the
 * CPU baseline and the reference arm of the benchmark build their inputs
 * here, so they load no engine code.  A plain-C restatement of the
 * workload generator the engine's benchmark uses (same seeds, same draws in
 * the same order, same arithmetic); tests/test_oracle_synth.py checks that
 * both produce the identical matrix, x_true, b and perturbed values.
 *
 * Families (synthetic stand-ins for the reference's private benchmark set):
 *  * block   (family 0): m ~ U{10..90} rescaled by largest remainder to sum n;
 *            per row a cycle entry i -> (i+1) mod m and 4 random intra-block
 *            draws, N(0,1); one coupling entry into a strictly later block,
 *            N(0, 0.1^2); a_ii = 0.5 sum_j!=i |a_ij| + N(0, 0.1^2).
 *  * circuit (family 1): Pareto(alpha 1.5, x_m 10) block sizes clipped to
 *            [1, 20000] for at most 90% of the rows, 1x1 blocks for the rest,
 *            shuffled; Pareto rows: cycle + 3 intra draws + 1 coupling entry,
 *            1x1 rows 5 coupling entries; 50 bus rows (first 10% of blocks)
 *            and 50 bus columns (last 10%) with 500 coupling entries each;
 *            off-diagonal values log-uniform in [1e-3, 1e3] with random sign;
 *            diagonal as above.
 * Then random row and column permutations, canonical (row, col) order,
 * x_true ~ U(-1, 1), b = A x_true.
 * RNG: xoshiro256** seeded through splitmix64; uniforms from the top 53
 * bits; normals by Box-Muller.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t s[4];
} or_rng;

static void rng_seed(or_rng* r, uint64_t seed) {
  uint64_t z = seed;
  int k;
  for (k = 0; k < 4; ++k) {
    uint64_t x;
    z += 0x9e3779b97f4a7c15ull;
    x = z;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    r->s[k] = x ^ (x >> 31);
  }
}

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(or_rng* r) {
  const uint64_t out = rotl64(r->s[1] * 5, 7) * 9;
  const uint64_t t = r->s[1] << 17;
  r->s[2] ^= r->s[0];
  r->s[3] ^= r->s[1];
  r->s[1] ^= r->s[2];
  r->s[0] ^= r->s[3];
  r->s[2] ^= t;
  r->s[3] = rotl64(r->s[3], 45);
  return out;
}

static double rng_uniform(or_rng* r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }
static double rng_uniform_pos(or_rng* r) { return ((double)(rng_next(r) >> 11) + 1.0) * 0x1.0p-53; }
static int64_t rng_below(or_rng* r, int64_t k) { return (int64_t)(rng_uniform(r) * (double)k); }
static double rng_normal(or_rng* r) {
  const double u1 = rng_uniform_pos(r), u2 = rng_uniform(r);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
static double loguniform_signed(or_rng* r) {
  const double mag = pow(10.0, -3.0 + 6.0 * rng_uniform(r));
  return (rng_next(r) >> 63) ? -mag : mag;
}

typedef struct {
  int32_t* col;
  double* val;
  int32_t len, cap;
} or_row;

static int row_push(or_row* r, int32_t c, double v) {
  if (r->len == r->cap) {
    const int32_t cap = r->cap ? 2 * r->cap : 8;
    int32_t* nc = (int32_t*)realloc(r->col, sizeof(int32_t) * (size_t)cap);
    double* nv;
    if (!nc) return 0;
    r->col = nc;
    nv = (double*)realloc(r->val, sizeof(double) * (size_t)cap);
    if (!nv) return 0;
    r->val = nv;
    r->cap = cap;
  }
  r->col[r->len] = c;
  r->val[r->len] = v;
  ++r->len;
  return 1;
}

/* Stable sort of a row by column (insertion sort; rows are short), then the
 * first entry of each run of equal columns is kept. */
static void dedupe_row(or_row* r) {
  int32_t i, w = 0;
  for (i = 1; i < r->len; ++i) {
    const int32_t c = r->col[i];
    const double v = r->val[i];
    int32_t k = i - 1;
    while (k >= 0 && r->col[k] > c) {
      r->col[k + 1] = r->col[k];
      r->val[k + 1] = r->val[k];
      --k;
    }
    r->col[k + 1] = c;
    r->val[k + 1] = v;
  }
  for (i = 0; i < r->len; ++i) {
    if (w > 0 && r->col[w - 1] == r->col[i]) continue;
    r->col[w] = r->col[i];
    r->val[w] = r->val[i];
    ++w;
  }
  r->len = w;
}

typedef struct {
  int32_t n, nrhs;
  int64_t nnz;
  int32_t *row, *col;
  double *val, *x_true, *b;
} or_synth;

typedef struct {
  int32_t c;
  double v;
} or_entry;

static int cmp_entry(const void* a, const void* b) {
  const int32_t x = ((const or_entry*)a)->c, y = ((const or_entry*)b)->c;
  return (x > y) - (x < y);
}

/* Diagonal rule, permutations, canonical order, x_true and b. */
static int finish(or_synth* s, or_row* rows, or_rng* rng) {
  const int32_t n = s->n;
  int32_t i, k, *pr, *pc, *inv_pr;
  int64_t nnz = 0, p;
  or_entry* tmp;
  int32_t maxlen = 0;
  for (i = 0; i < n; ++i) {
    or_row* r = &rows[i];
    double sum = 0.0, noise, d;
    int32_t t;
    dedupe_row(r);
    for (t = 0; t < r->len; ++t) sum += fabs(r->val[t]);
    noise = 0.1 * rng_normal(rng);
    d = 0.5 * sum + noise;
    if (d == 0.0) d = 1.0;
    if (!row_push(r, i, d)) return 0;
    nnz += r->len;
    if (r->len > maxlen) maxlen = r->len;
  }
  pr = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  pc = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  inv_pr = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  tmp = (or_entry*)malloc(sizeof(or_entry) * (size_t)(maxlen > 0 ? maxlen : 1));
  s->row = (int32_t*)malloc(sizeof(int32_t) * (size_t)nnz);
  s->col = (int32_t*)malloc(sizeof(int32_t) * (size_t)nnz);
  s->val = (double*)malloc(sizeof(double) * (size_t)nnz);
  s->x_true = (double*)malloc(sizeof(double) * (size_t)n * (size_t)s->nrhs);
  s->b = (double*)calloc((size_t)n * (size_t)s->nrhs, sizeof(double));
  if (!pr || !pc || !inv_pr || !tmp || !s->row || !s->col || !s->val || !s->x_true || !s->b) {
    free(pr);
    free(pc);
    free(inv_pr);
    free(tmp);
    return 0;
  }
  for (i = 0; i < n; ++i) pr[i] = pc[i] = i;
  for (i = n - 1; i > 0; --i) {
    const int64_t j = rng_below(rng, i + 1);
    const int32_t t = pr[i];
    pr[i] = pr[j];
    pr[j] = t;
  }
  for (i = n - 1; i > 0; --i) {
    const int64_t j = rng_below(rng, i + 1);
    const int32_t t = pc[i];
    pc[i] = pc[j];
    pc[j] = t;
  }
  for (i = 0; i < n; ++i) inv_pr[pr[i]] = i;
  p = 0;
  for (i = 0; i < n; ++i) {
    const or_row* r = &rows[inv_pr[i]];
    int32_t t;
    for (t = 0; t < r->len; ++t) {
      tmp[t].c = pc[r->col[t]];
      tmp[t].v = r->val[t];
    }
    qsort(tmp, (size_t)r->len, sizeof(or_entry), cmp_entry); /* columns are distinct */
    for (t = 0; t < r->len; ++t) {
      s->row[p] = i;
      s->col[p] = tmp[t].c;
      s->val[p] = tmp[t].v;
      ++p;
    }
  }
  s->nnz = nnz;
  for (p = 0; p < (int64_t)n * s->nrhs; ++p) s->x_true[p] = 2.0 * rng_uniform(rng) - 1.0;
  for (k = 0; k < s->nrhs; ++k) {
    const double* x = s->x_true + (size_t)k * (size_t)n;
    double* bb = s->b + (size_t)k * (size_t)n;
    for (p = 0; p < nnz; ++p) bb[s->row[p]] += s->val[p] * x[s->col[p]];
  }
  free(pr);
  free(pc);
  free(inv_pr);
  free(tmp);
  return 1;
}

typedef struct {
  double f;
  int32_t i;
} or_frac;

static int cmp_frac_desc(const void* a, const void* b) {
  const or_frac *x = (const or_frac*)a, *y = (const or_frac*)b;
  if (x->f != y->f) return x->f > y->f ? -1 : 1;
  return (x->i > y->i) - (x->i < y->i); /* stable: original order on ties */
}

/* nb sizes ~ U{lo..hi} rescaled to sum n by largest remainder. */
static int32_t* rescaled_uniform_sizes(or_rng* rng, int32_t n, int32_t* nb_io, int32_t lo, int32_t hi) {
  int32_t nb = *nb_io, i;
  double tot = 0.0, *raw;
  int32_t* sz;
  or_frac* frac;
  int64_t used = 0, rem;
  size_t k;
  if (nb > n) nb = n;
  if (nb < 1) nb = 1;
  raw = (double*)malloc(sizeof(double) * (size_t)nb);
  sz = (int32_t*)malloc(sizeof(int32_t) * (size_t)nb);
  frac = (or_frac*)malloc(sizeof(or_frac) * (size_t)nb);
  for (i = 0; i < nb; ++i) {
    raw[i] = (double)(lo + rng_below(rng, hi - lo + 1));
    tot += raw[i];
  }
  for (i = 0; i < nb; ++i) {
    const double t = raw[i] * (double)n / tot;
    int32_t f = (int32_t)floor(t);
    if (f < 1) f = 1;
    sz[i] = f;
    used += f;
    frac[i].f = t - floor(t);
    frac[i].i = i;
  }
  qsort(frac, (size_t)nb, sizeof(or_frac), cmp_frac_desc);
  rem = n - used;
  for (k = 0; rem > 0; k = (k + 1) % (size_t)nb, --rem) sz[frac[k].i]++;
  for (k = (size_t)nb; rem < 0 && k-- > 0;) {
    while (rem < 0 && sz[k] > 1) {
      sz[k]--;
      rem++;
    }
  }
  free(raw);
  free(frac);
  *nb_io = nb;
  return sz;
}

static int gen_block_family(or_synth* s, or_rng* rng, int32_t n, int32_t nb) {
  int32_t *sz = rescaled_uniform_sizes(rng, n, &nb, 10, 90), *off, b, i, t;
  or_row* rows;
  int ok = 1;
  s->n = n;
  off = (int32_t*)calloc((size_t)nb + 1, sizeof(int32_t));
  rows = (or_row*)calloc((size_t)(n > 0 ? n : 0), sizeof(or_row));
  for (b = 0; b < nb; ++b) off[b + 1] = off[b] + sz[b];
  for (b = 0; b < nb && ok; ++b) {
    const int32_t m = sz[b], o = off[b];
    for (i = 0; i < m && ok; ++i) {
      or_row* r = &rows[o + i];
      if (m > 1) ok &= row_push(r, o + (i + 1) % m, rng_normal(rng));
      for (t = 0; t < 4 && m > 1; ++t) {
        const int32_t c = (int32_t)rng_below(rng, m);
        const double v = rng_normal(rng);
        if (c != i) ok &= row_push(r, o + c, v);
      }
      if (b + 1 < nb) {
        const int32_t lo = off[b + 1];
        const int32_t c = lo + (int32_t)rng_below(rng, n - lo);
        ok &= row_push(r, c, 0.1 * rng_normal(rng));
      }
    }
  }
  if (ok) ok = finish(s, rows, rng);
  for (i = 0; i < n; ++i) {
    free(rows[i].col);
    free(rows[i].val);
  }
  free(rows);
  free(off);
  free(sz);
  return ok;
}

/* Pareto(alpha = 1.5, x_m = 10) sizes clipped to [1, clip], at most `budget`
 * rows in total; returns the count. */
static int32_t pareto_sizes(or_rng* rng, int32_t count, int32_t clip, int64_t budget, int32_t* out) {
  int64_t used = 0;
  int32_t k, got = 0;
  for (k = 0; k < count; ++k) {
    const double x = 10.0 / pow(rng_uniform_pos(rng), 1.0 / 1.5);
    const double f = floor(x);
    int32_t m = (int32_t)(f < (double)clip ? f : (double)clip);
    if (m < 1) m = 1;
    if (used + m > budget) break;
    out[got++] = m;
    used += m;
  }
  return got;
}

static int couple(or_row* r, or_rng* rng, const int32_t* off, int32_t b, int32_t nb, int32_t n) {
  int32_t lo, c;
  if (b + 1 >= nb) return 1;
  lo = off[b + 1];
  c = lo + (int32_t)rng_below(rng, n - lo);
  return row_push(r, c, loguniform_signed(rng));
}

static int gen_circuit_family(or_synth* s, or_rng* rng, int32_t n, int32_t npareto, int32_t nbus) {
  int32_t *sizes = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + npareto + 1)), *off;
  int32_t npar = pareto_sizes(rng, npareto, 20000, (int64_t)n * 9 / 10, sizes), nb, b, i, t, k;
  int64_t used = 0, q;
  or_row* rows;
  int ok = 1;
  size_t early, late0;
  s->n = n;
  for (k = 0; k < npar; ++k) used += sizes[k];
  nb = npar;
  for (q = used; q < n; ++q) sizes[nb++] = 1;
  for (k = nb - 1; k > 0; --k) {
    const int64_t j = rng_below(rng, (int64_t)k + 1);
    const int32_t tt = sizes[k];
    sizes[k] = sizes[j];
    sizes[j] = tt;
  }
  off = (int32_t*)calloc((size_t)(nb > 0 ? nb : 0) + 1, sizeof(int32_t));
  rows = (or_row*)calloc((size_t)(n > 0 ? n : 0), sizeof(or_row));
  for (b = 0; b < nb; ++b) off[b + 1] = off[b] + sizes[b];
  for (b = 0; b < nb && ok; ++b) {
    const int32_t m = sizes[b], o = off[b];
    for (i = 0; i < m && ok; ++i) {
      or_row* r = &rows[o + i];
      if (m > 1) {
        ok &= row_push(r, o + (i + 1) % m, loguniform_signed(rng));
        for (t = 0; t < 3; ++t) {
          const int32_t c = (int32_t)rng_below(rng, m);
          const double v = loguniform_signed(rng);
          if (c != i) ok &= row_push(r, o + c, v);
        }
        ok &= couple(r, rng, off, b, nb, n);
      } else {
        for (t = 0; t < 5; ++t) ok &= couple(r, rng, off, b, nb, n);
      }
    }
  }
  early = (size_t)(nb / 10 > 1 ? nb / 10 : 1);
  late0 = (size_t)nb - (size_t)(nb / 10 > 1 ? nb / 10 : 1);
  for (k = 0; k < nbus && ok; ++k) {
    const int32_t bb = (int32_t)rng_below(rng, (int64_t)early);
    const int32_t r = off[bb] + (int32_t)rng_below(rng, sizes[bb]);
    const int32_t lo = off[bb + 1];
    if (lo >= n) continue;
    for (t = 0; t < 500; ++t) {
      const int32_t c = lo + (int32_t)rng_below(rng, n - lo);
      ok &= row_push(&rows[r], c, loguniform_signed(rng));
    }
  }
  for (k = 0; k < nbus && ok; ++k) {
    const int32_t bb = (int32_t)late0 + (int32_t)rng_below(rng, (int64_t)((size_t)nb - late0));
    const int32_t c = off[bb] + (int32_t)rng_below(rng, sizes[bb]);
    const int32_t hi = off[bb];
    if (hi <= 0) continue;
    for (t = 0; t < 500; ++t) {
      const int32_t r = (int32_t)rng_below(rng, hi);
      ok &= row_push(&rows[r], c, loguniform_signed(rng));
    }
  }
  if (ok) ok = finish(s, rows, rng);
  for (i = 0; i < n; ++i) {
    free(rows[i].col);
    free(rows[i].val);
  }
  free(rows);
  free(off);
  free(sizes);
  return ok;
}

void or_synth_free(or_synth* s) {
  if (!s) return;
  free(s->row);
  free(s->col);
  free(s->val);
  free(s->x_true);
  free(s->b);
  free(s);
}

/* family 0 (block): n rows, param blocks (0: n/50); family 1 (circuit): n
 * rows, param Pareto blocks (0: 1000 n / 200000).  NULL for other families. */
or_synth* or_synth_create(int32_t family, uint64_t seed, int32_t n, int32_t param, int32_t nrhs) {
  or_synth* s = (or_synth*)calloc(1, sizeof(or_synth));
  or_rng rng;
  int ok = 0;
  if (!s) return NULL;
  s->nrhs = nrhs > 0 ? nrhs : 1;
  rng_seed(&rng, seed);
  if (family == 0) {
    ok = gen_block_family(s, &rng, n, param > 0 ? param : (n / 50 > 1 ? n / 50 : 1));
  } else if (family == 1) {
    const int64_t np = 1000LL * n / 200000;
    ok = gen_circuit_family(s, &rng, n, param > 0 ? param : (np > 1 ? (int32_t)np : 1), 50);
  }
  if (!ok) {
    or_synth_free(s);
    return NULL;
  }
  return s;
}

int32_t or_synth_n(const or_synth* s) { return s ? s->n : 0; }
int64_t or_synth_nnz(const or_synth* s) { return s ? s->nnz : 0; }

void or_synth_copy(const or_synth* s, int32_t* rows, int32_t* cols, double* vals, double* x_true, double* b) {
  if (!s) return;
  if (rows) memcpy(rows, s->row, sizeof(int32_t) * (size_t)s->nnz);
  if (cols) memcpy(cols, s->col, sizeof(int32_t) * (size_t)s->nnz);
  if (vals) memcpy(vals, s->val, sizeof(double) * (size_t)s->nnz);
  if (x_true) memcpy(x_true, s->x_true, sizeof(double) * (size_t)s->n * (size_t)s->nrhs);
  if (b) memcpy(b, s->b, sizeof(double) * (size_t)s->n * (size_t)s->nrhs);
}

/* values x (1 + U(-0.1, 0.1)), one draw per stored entry. */
void or_synth_perturb(const or_synth* s, uint64_t seed, double* out) {
  or_rng rng;
  int64_t k;
  if (!s || !out) return;
  rng_seed(&rng, seed);
  for (k = 0; k < s->nnz; ++k) out[k] = s->val[k] * (1.0 + 0.2 * rng_uniform(&rng) - 0.1);
}
