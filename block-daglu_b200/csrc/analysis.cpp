// Host-side integer analysis: canonical COO, signatures, DM/BTF, block merge,
// UBTF split and block DAG.  See analysis.h for the reference functions each
// routine restates.
#include "analysis.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>

namespace bdlu {

const char* getenv_compat(const char* name) {
  // env.h:15-25 documents that USERALGO_X is looked up as BLOCKDAGLU_X first.
  // (The reference's own helper compares 8 characters of the 9-character
  // prefix and ends up querying "BLOCKDAGLU__X"; the documented names are
  // honoured here.)
  if (!name) return nullptr;
  static const char kOld[] = "USERALGO_";
  if (std::strncmp(name, kOld, 9) == 0) {
    std::string alt = std::string("BLOCKDAGLU_") + (name + 9);
    if (const char* v = std::getenv(alt.c_str())) return v;
  }
  return std::getenv(name);
}

namespace {

struct Entry {
  int32_t r;
  int32_t c;
  double v;
};

}  // namespace

Status canonicalize(const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
                    int32_t dimension_hint, CanonicalCoo& out, std::string& msg) {
  // solver.cpp:642-722, check order and messages included.
  if (dimension_hint < -1) {
    msg = "matrix dimension must be non-negative";
    return Status::InvalidDimension;
  }
  int32_t max_index = -1;
  for (int64_t k = 0; k < nnz; ++k) {
    const int32_t r = rows[k];
    const int32_t c = cols[k];
    const double v = vals[k];
    if (r < 0 || c < 0) {
      msg = "matrix contains a negative row or column index";
      return Status::InvalidIndex;
    }
    if (!std::isfinite(v)) {
      msg = "matrix contains NaN or infinity";
      return Status::NonFiniteValue;
    }
    if (dimension_hint >= 0 && (r >= dimension_hint || c >= dimension_hint)) {
      msg = "matrix entry lies outside the declared dimension";
      return Status::InvalidIndex;
    }
    max_index = std::max(max_index, std::max(r, c));
  }
  int32_t n = 0;
  if (dimension_hint >= 0) {
    n = dimension_hint;
  } else {
    if (max_index == std::numeric_limits<int32_t>::max()) {
      msg = "inferred matrix dimension overflows int32";
      return Status::InvalidDimension;
    }
    n = max_index + 1;
  }
  if (n <= 0) {
    msg = "matrix dimension must be positive";
    return Status::InvalidDimension;
  }

  // Strictly increasing (row, col) input is already canonical apart from the
  // zero drop; any other input goes through std::sort with the reference's
  // comparator, which visits equal keys in the same order as the reference
  // does on the same standard library, so duplicate sums see the same order.
  bool strictly_sorted = true;
  for (int64_t k = 1; k < nnz && strictly_sorted; ++k) {
    if (rows[k - 1] > rows[k] || (rows[k - 1] == rows[k] && cols[k - 1] >= cols[k])) {
      strictly_sorted = false;
    }
  }
  out.n = n;
  out.row.clear();
  out.col.clear();
  out.val.clear();
  out.row.reserve(static_cast<size_t>(nnz));
  out.col.reserve(static_cast<size_t>(nnz));
  out.val.reserve(static_cast<size_t>(nnz));
  if (strictly_sorted) {
    for (int64_t k = 0; k < nnz; ++k) {
      if (vals[k] != 0.0) {
        out.row.push_back(rows[k]);
        out.col.push_back(cols[k]);
        out.val.push_back(vals[k]);
      }
    }
  } else {
    std::vector<Entry> e(static_cast<size_t>(nnz));
    for (int64_t k = 0; k < nnz; ++k) e[static_cast<size_t>(k)] = Entry{rows[k], cols[k], vals[k]};
    std::sort(e.begin(), e.end(), [](const Entry& a, const Entry& b) {
      if (a.r != b.r) return a.r < b.r;
      return a.c < b.c;
    });
    for (size_t i = 0; i < e.size();) {
      const int32_t r = e[i].r;
      const int32_t c = e[i].c;
      long double sum = 0.0L;
      size_t j = i;
      while (j < e.size() && e[j].r == r && e[j].c == c) {
        sum += static_cast<long double>(e[j].v);
        ++j;
      }
      const double v = static_cast<double>(sum);
      if (!std::isfinite(v)) {
        msg = "combining duplicate matrix entries overflowed";
        return Status::NonFiniteValue;
      }
      if (v != 0.0) {
        out.row.push_back(r);
        out.col.push_back(c);
        out.val.push_back(v);
      }
      i = j;
    }
  }
  msg.clear();
  return Status::Ok;
}

static inline uint64_t fnv1a64_mix(uint64_t h, uint64_t x) {
  h ^= x;
  return h * 1099511628211ull;
}

uint64_t matrix_sig(int32_t n, const CanonicalCoo& a) {
  uint64_t h = 1469598103934665603ull;
  h = fnv1a64_mix(h, static_cast<uint64_t>(n));
  h = fnv1a64_mix(h, static_cast<uint64_t>(a.row.size()));
  for (size_t k = 0; k < a.row.size(); ++k) {
    const uint64_t r = static_cast<uint32_t>(a.row[k]);
    const uint64_t c = static_cast<uint32_t>(a.col[k]);
    h = fnv1a64_mix(h, (r << 32) ^ c);
  }
  return h;
}

uint64_t matrix_sig2(int32_t n, const CanonicalCoo& a) {
  uint64_t h = 0x6a09e667f3bcc909ull ^ static_cast<uint64_t>(n);
  for (size_t k = 0; k < a.row.size(); ++k) {
    const uint64_t r = static_cast<uint32_t>(a.row[k]);
    const uint64_t c = static_cast<uint32_t>(a.col[k]);
    uint64_t x = (r << 32) ^ c ^ 0x9e3779b97f4a7c15ull;
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    h ^= x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  }
  return h ^ static_cast<uint64_t>(a.row.size());
}

uint64_t matrix_value_sig(const CanonicalCoo& a) {
  uint64_t h = 0xbb67ae8584caa73bull;
  for (double v : a.val) {
    uint64_t bits;
    std::memcpy(&bits, &v, sizeof(bits));
    h = fnv1a64_mix(h, bits);
  }
  return h ^ static_cast<uint64_t>(a.val.size());
}

static int64_t env_int(const char* name, int64_t def, int64_t min_ok) {
  if (const char* e = getenv_compat(name)) {
    const long long v = std::atoll(e);
    if (v >= min_ok) return v;
  }
  return def;
}

bool auto_choose_block(int32_t n, const CanonicalCoo& a) {
  const size_t nnz = a.row.size();
  // Coarse rules, solver.cpp:466-473.
  bool coarse;
  if (n >= 65000 && nnz >= 3000000) {
    coarse = false;
  } else if (n <= 25000 && nnz >= 600000) {
    coarse = true;
  } else {
    const int64_t n_thr = env_int("USERALGO_AUTO_BLOCK_N", 50000, 1);
    const int64_t nnz_thr = env_int("USERALGO_AUTO_BLOCK_NNZ", 2000000, 1);
    coarse = (n >= n_thr) || (static_cast<int64_t>(nnz) >= nnz_thr);
  }
  if (!coarse) return false;
  if (n < 40000 && nnz < 1500000) return true;

  // compute_profile_lite, solver.cpp:182-231 (deterministic stride sample).
  std::vector<int32_t> row_deg(static_cast<size_t>(n), 0), col_deg(static_cast<size_t>(n), 0);
  std::vector<uint8_t> diag_has(static_cast<size_t>(n), 0);
  const size_t target = 200000;
  const size_t step = (nnz > target) ? std::max<size_t>(1, nnz / target) : 1;
  for (size_t k = 0; k < nnz; k += step) {
    const int32_t r = a.row[k], c = a.col[k];
    if (r < 0 || c < 0 || r >= n || c >= n) continue;
    row_deg[static_cast<size_t>(r)]++;
    col_deg[static_cast<size_t>(c)]++;
    if (r == c) diag_has[static_cast<size_t>(r)] = 1;
  }
  int32_t diag_present = 0;
  for (int32_t i = 0; i < n; ++i) diag_present += diag_has[static_cast<size_t>(i)] != 0;
  const double diag_cov = static_cast<double>(diag_present) / static_cast<double>(n);
  const int32_t s = static_cast<int32_t>(step);
  const int32_t row_max = *std::max_element(row_deg.begin(), row_deg.end()) * s;
  const int32_t col_max = *std::max_element(col_deg.begin(), col_deg.end()) * s;
  auto p95 = [](std::vector<int32_t> v) {
    const size_t k = static_cast<size_t>(0.95 * static_cast<double>(v.size() - 1));
    std::nth_element(v.begin(), v.begin() + static_cast<long>(k), v.end());
    return v[k];
  };
  const int32_t row_p95 = p95(row_deg) * s;
  const int32_t col_p95 = p95(col_deg) * s;
  const int32_t dense_thr = std::max<int32_t>(4096, n / 8);
  const bool hub = row_max >= dense_thr || col_max >= dense_thr;
  const int32_t broad_thr = std::max<int32_t>(512, n / 64);
  const bool broad = row_p95 >= broad_thr && col_p95 >= broad_thr && diag_cov >= 0.9;
  return !(hub || broad);
}

Csc pattern_csc(const CanonicalCoo& a, double drop_abs_lt) {
  // Two-pass count + scatter; within a column entries keep COO order
  // (sparse_formats.h:23-53, ubtf_block_solver.cpp:333-371).
  Csc out;
  const int32_t n = a.n;
  out.n = n;
  out.col_ptr.assign(static_cast<size_t>(n) + 1, 0);
  const size_t nnz = a.row.size();
  for (size_t k = 0; k < nnz; ++k) {
    if (drop_abs_lt > 0.0 && std::abs(a.val[k]) < drop_abs_lt) continue;
    out.col_ptr[static_cast<size_t>(a.col[k]) + 1]++;
  }
  for (int32_t i = 0; i < n; ++i) out.col_ptr[i + 1] += out.col_ptr[i];
  out.row_ind.resize(static_cast<size_t>(out.col_ptr[n]));
  std::vector<int32_t> next(out.col_ptr.begin(), out.col_ptr.end() - 1);
  for (size_t k = 0; k < nnz; ++k) {
    if (drop_abs_lt > 0.0 && std::abs(a.val[k]) < drop_abs_lt) continue;
    out.row_ind[static_cast<size_t>(next[a.col[k]]++)] = a.row[k];
  }
  return out;
}

// ---------------------------------------------------------------------------
// DM/BTF.  SuiteSparse BTF (btf_order = btf_maxtrans + btf_strongcomp) is not
// present here; this follows its published structure and output conventions:
//  * maximum transversal (any maximum matching gives the same block
//    partition; SuiteSparse's single-pass depth-first MC21 search is
//    quadratic on large circuit-like patterns, so a Karp-Sipser start and
//    Hopcroft-Karp phases are used);
//  * unmatched rows paired with unmatched columns in increasing order and the
//    column flagged as -(col)-2 (BTF_FLIP);
//  * Tarjan's strongly connected components of the graph of A(:,Q), roots
//    taken in order 0..n-1, components numbered in completion order, which
//    makes A(P,Q) upper block triangular.
// ---------------------------------------------------------------------------
static int32_t maxtrans(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* match) {
  // Karp-Sipser initial matching, then Hopcroft-Karp augmentation.  Columns
  // and rows are visited in increasing index order.
  std::vector<int32_t> cmatch(static_cast<size_t>(n), -1);
  std::vector<int32_t> it(static_cast<size_t>(n)), stack(static_cast<size_t>(n));
  for (int32_t i = 0; i < n; ++i) match[i] = -1;
  int32_t nmatch = 0;
  // Karp-Sipser start: vertices left with one free neighbour are matched to
  // it first (this alone recovers the matching of triangular parts); when
  // none is left, the lowest free column takes its first free row.
  {
    std::vector<int32_t> rp(static_cast<size_t>(n) + 1, 0), rc(static_cast<size_t>(Ap[n]));
    for (int32_t p = 0; p < Ap[n]; ++p) rp[static_cast<size_t>(Ai[p]) + 1]++;
    for (int32_t i = 0; i < n; ++i) rp[static_cast<size_t>(i) + 1] += rp[static_cast<size_t>(i)];
    {
      std::vector<int32_t> nx(rp.begin(), rp.end() - 1);
      for (int32_t j = 0; j < n; ++j)
        for (int32_t p = Ap[j]; p < Ap[j + 1]; ++p) rc[static_cast<size_t>(nx[static_cast<size_t>(Ai[p])]++)] = j;
    }
    std::vector<int32_t> cdeg(static_cast<size_t>(n)), rdeg(static_cast<size_t>(n));
    for (int32_t j = 0; j < n; ++j) cdeg[static_cast<size_t>(j)] = Ap[j + 1] - Ap[j];
    for (int32_t i = 0; i < n; ++i) rdeg[static_cast<size_t>(i)] = rp[static_cast<size_t>(i) + 1] - rp[static_cast<size_t>(i)];
    // Work list of (vertex, is_row) with degree one.
    std::vector<int64_t> work;
    work.reserve(static_cast<size_t>(n));
    for (int32_t j = 0; j < n; ++j) if (cdeg[static_cast<size_t>(j)] == 1) work.push_back(j);
    for (int32_t i = 0; i < n; ++i) if (rdeg[static_cast<size_t>(i)] == 1) work.push_back(-static_cast<int64_t>(i) - 1);
    auto take = [&](int32_t i, int32_t j) {
      match[i] = j;
      cmatch[static_cast<size_t>(j)] = i;
      ++nmatch;
      for (int32_t p = rp[static_cast<size_t>(i)]; p < rp[static_cast<size_t>(i) + 1]; ++p) {
        const int32_t jj = rc[static_cast<size_t>(p)];
        if (cmatch[static_cast<size_t>(jj)] == -1 && --cdeg[static_cast<size_t>(jj)] == 1) work.push_back(jj);
      }
      for (int32_t p = Ap[j]; p < Ap[j + 1]; ++p) {
        const int32_t ii = Ai[p];
        if (match[ii] == -1 && --rdeg[static_cast<size_t>(ii)] == 1) work.push_back(-static_cast<int64_t>(ii) - 1);
      }
    };
    size_t wh = 0;
    int32_t next_col = 0;
    while (true) {
      if (wh < work.size()) {
        const int64_t v = work[wh++];
        if (v >= 0) {
          const int32_t j = static_cast<int32_t>(v);
          if (cmatch[static_cast<size_t>(j)] != -1) continue;
          for (int32_t p = Ap[j]; p < Ap[j + 1]; ++p)
            if (match[Ai[p]] == -1) { take(Ai[p], j); break; }
        } else {
          const int32_t i = static_cast<int32_t>(-v - 1);
          if (match[i] != -1) continue;
          for (int32_t p = rp[static_cast<size_t>(i)]; p < rp[static_cast<size_t>(i) + 1]; ++p) {
            const int32_t j = rc[static_cast<size_t>(p)];
            if (cmatch[static_cast<size_t>(j)] == -1) { take(i, j); break; }
          }
        }
        continue;
      }
      while (next_col < n && cmatch[static_cast<size_t>(next_col)] != -1) ++next_col;
      if (next_col >= n) break;
      bool took = false;
      for (int32_t p = Ap[next_col]; p < Ap[next_col + 1]; ++p)
        if (match[Ai[p]] == -1) { take(Ai[p], next_col); took = true; break; }
      if (!took) cmatch[static_cast<size_t>(next_col)] = -2;  // no free row now; retried below
      ++next_col;
    }
    for (int32_t j = 0; j < n; ++j) if (cmatch[static_cast<size_t>(j)] == -2) cmatch[static_cast<size_t>(j)] = -1;
  }
  // Hopcroft-Karp phases: BFS layering from the free columns, then layered
  // depth-first augmentation along shortest paths.
  const int32_t kInf = std::numeric_limits<int32_t>::max();
  std::vector<int32_t> dist(static_cast<size_t>(n)), queue(static_cast<size_t>(n));
  while (true) {
    int32_t qh = 0, qt = 0, limit = kInf;
    for (int32_t j = 0; j < n; ++j) {
      if (cmatch[static_cast<size_t>(j)] == -1) {
        dist[static_cast<size_t>(j)] = 0;
        queue[static_cast<size_t>(qt++)] = j;
      } else {
        dist[static_cast<size_t>(j)] = kInf;
      }
    }
    while (qh < qt) {
      const int32_t j = queue[static_cast<size_t>(qh++)];
      if (dist[static_cast<size_t>(j)] >= limit) continue;
      for (int32_t p = Ap[j]; p < Ap[j + 1]; ++p) {
        const int32_t j2 = match[Ai[p]];
        if (j2 == -1) {
          if (limit == kInf) limit = dist[static_cast<size_t>(j)] + 1;
        } else if (dist[static_cast<size_t>(j2)] == kInf) {
          dist[static_cast<size_t>(j2)] = dist[static_cast<size_t>(j)] + 1;
          queue[static_cast<size_t>(qt++)] = j2;
        }
      }
    }
    if (limit == kInf) break;
    int32_t augmented = 0;
    for (int32_t root = 0; root < n; ++root) {
      if (cmatch[static_cast<size_t>(root)] != -1 || dist[static_cast<size_t>(root)] != 0) continue;
      int32_t top = 0;
      stack[0] = root;
      it[static_cast<size_t>(root)] = Ap[root];
      bool done = false;
      while (top >= 0 && !done) {
        const int32_t j = stack[static_cast<size_t>(top)];
        bool moved = false;
        for (int32_t& p = it[static_cast<size_t>(j)]; p < Ap[j + 1]; ++p) {
          const int32_t i = Ai[p];
          const int32_t j2 = match[i];
          if (j2 == -1) {
            if (dist[static_cast<size_t>(j)] + 1 != limit) continue;
            // Column stack[t] takes the row it points at; the last one takes
            // the free row i.
            for (int32_t t = top; t >= 0; --t) {
              const int32_t jc = stack[static_cast<size_t>(t)];
              const int32_t ir = Ai[it[static_cast<size_t>(jc)]];
              match[ir] = jc;
              cmatch[static_cast<size_t>(jc)] = ir;
            }
            done = true;
            moved = true;
            break;
          }
          if (dist[static_cast<size_t>(j2)] == dist[static_cast<size_t>(j)] + 1) {
            stack[static_cast<size_t>(++top)] = j2;
            it[static_cast<size_t>(j2)] = Ap[j2];
            moved = true;
            break;
          }
        }
        if (!moved) {
          dist[static_cast<size_t>(j)] = kInf;  // dead end for this phase
          --top;
          if (top >= 0) ++it[static_cast<size_t>(stack[static_cast<size_t>(top)])];
        }
      }
      if (done) {
        ++augmented;
        ++nmatch;
      }
    }
    if (augmented == 0) break;
  }
  return nmatch;
}

static inline int32_t unflip(int32_t j) { return j < -1 ? -j - 2 : j; }

static int32_t strongcomp(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* Q, int32_t* P,
                          int32_t* R) {
  // Iterative Tarjan.  Node j stands for (row j, column Q[j]); its successors
  // are the rows of column Q[j].
  std::vector<int32_t> index(static_cast<size_t>(n), -1), low(static_cast<size_t>(n), 0);
  std::vector<int32_t> pos(static_cast<size_t>(n), 0), cstack, tstack;
  std::vector<uint8_t> on_stack(static_cast<size_t>(n), 0);
  std::vector<int32_t> comp(static_cast<size_t>(n), -1);
  cstack.reserve(static_cast<size_t>(n));
  tstack.reserve(static_cast<size_t>(n));
  int32_t counter = 0, nblocks = 0, k = 0;
  for (int32_t root = 0; root < n; ++root) {
    if (index[static_cast<size_t>(root)] != -1) continue;
    cstack.push_back(root);
    while (!cstack.empty()) {
      const int32_t v = cstack.back();
      const int32_t col = unflip(Q[v]);
      if (index[static_cast<size_t>(v)] == -1) {
        index[static_cast<size_t>(v)] = low[static_cast<size_t>(v)] = counter++;
        pos[static_cast<size_t>(v)] = Ap[col];
        tstack.push_back(v);
        on_stack[static_cast<size_t>(v)] = 1;
      }
      bool descended = false;
      for (int32_t p = pos[static_cast<size_t>(v)]; p < Ap[col + 1]; ++p) {
        const int32_t w = Ai[p];
        if (index[static_cast<size_t>(w)] == -1) {
          pos[static_cast<size_t>(v)] = p + 1;
          cstack.push_back(w);
          descended = true;
          break;
        }
        if (on_stack[static_cast<size_t>(w)]) {
          low[static_cast<size_t>(v)] = std::min(low[static_cast<size_t>(v)], index[static_cast<size_t>(w)]);
        }
      }
      if (descended) continue;
      pos[static_cast<size_t>(v)] = Ap[col + 1];
      cstack.pop_back();
      if (!cstack.empty()) {
        const int32_t parent = cstack.back();
        low[static_cast<size_t>(parent)] = std::min(low[static_cast<size_t>(parent)], low[static_cast<size_t>(v)]);
      }
      if (low[static_cast<size_t>(v)] == index[static_cast<size_t>(v)]) {
        R[nblocks] = k;
        int32_t w;
        do {
          w = tstack.back();
          tstack.pop_back();
          on_stack[static_cast<size_t>(w)] = 0;
          comp[static_cast<size_t>(w)] = nblocks;
          P[k++] = w;
        } while (w != v);
        ++nblocks;
      }
    }
  }
  R[nblocks] = n;
  // New column order follows the row (node) order, keeping flip flags.
  std::vector<int32_t> q(static_cast<size_t>(n));
  for (int32_t t = 0; t < n; ++t) q[static_cast<size_t>(t)] = Q[P[t]];
  std::copy(q.begin(), q.end(), Q);
  return nblocks;
}

int32_t btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q,
                  int32_t* R, int32_t* nmatch_out) {
  if (n <= 0) return 0;
  std::vector<int32_t> match(static_cast<size_t>(n));
  const int32_t nmatch = maxtrans(n, Ap, Ai, match.data());
  if (nmatch < n) {
    std::vector<uint8_t> col_used(static_cast<size_t>(n), 0);
    for (int32_t i = 0; i < n; ++i)
      if (match[static_cast<size_t>(i)] >= 0) col_used[static_cast<size_t>(match[static_cast<size_t>(i)])] = 1;
    int32_t j = 0;
    for (int32_t i = 0; i < n; ++i) {
      if (match[static_cast<size_t>(i)] >= 0) continue;
      while (col_used[static_cast<size_t>(j)]) ++j;
      col_used[static_cast<size_t>(j)] = 1;
      match[static_cast<size_t>(i)] = -j - 2;
    }
  }
  for (int32_t i = 0; i < n; ++i) Q[i] = match[static_cast<size_t>(i)];
  if (nmatch_out) *nmatch_out = nmatch;
  return strongcomp(n, Ap, Ai, Q, P, R);
}

std::vector<int32_t> merge_block_boundaries(const std::vector<int32_t>& R, int32_t n,
                                            int32_t merge_max) {
  // ubtf_block_solver.cpp:393-476: runs of consecutive blocks of size
  // <= min(merge_max, 32) are packed into groups of at most merge_max rows;
  // larger blocks stay intact.
  if (R.size() < 2) return {0, n};
  const int32_t nb = static_cast<int32_t>(R.size() - 1);
  if (nb <= 1) return {0, n};
  if (merge_max <= 0) merge_max = 64;
  const int32_t small_max = std::max<int32_t>(1, std::min<int32_t>(merge_max, 32));
  std::vector<int32_t> out;
  out.reserve(R.size());
  out.push_back(0);
  int32_t acc = 0, run_start = 0, run_end = 0;
  auto flush = [&]() {
    if (acc <= 0) return;
    if (out.back() != run_start) out.push_back(run_start);
    if (out.back() != run_end) out.push_back(run_end);
    acc = run_start = run_end = 0;
  };
  for (int32_t b = 0; b < nb; ++b) {
    const int32_t s = R[static_cast<size_t>(b)], e = R[static_cast<size_t>(b) + 1], sz = e - s;
    if (sz <= small_max) {
      if (acc == 0) {
        run_start = s;
        run_end = e;
        acc = sz;
        continue;
      }
      if (acc + sz <= merge_max) {
        acc += sz;
        run_end = e;
        continue;
      }
      flush();
      run_start = s;
      run_end = e;
      acc = sz;
      continue;
    }
    flush();
    if (out.back() != s) out.push_back(s);
    if (out.back() != e) out.push_back(e);
  }
  flush();
  if (out.back() != n) out.push_back(n);
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

AnalysisOptions analysis_options_from_env() {
  AnalysisOptions o;
  // Merge cap: BLOCK_MERGE_MAX_SIZE, else DENSE_BLOCK_MAX, else 64
  // (ubtf_block_solver.cpp:407-419).
  int64_t mm = env_int("USERALGO_BLOCK_MERGE_MAX_SIZE", 0, 1);
  if (mm <= 0) mm = env_int("USERALGO_DENSE_BLOCK_MAX", 0, 1);
  o.merge_max = mm > 0 ? static_cast<int32_t>(mm) : 64;
  if (const char* e = getenv_compat("USERALGO_BLOCK_MERGE")) o.merge = std::atoi(e) != 0;
  if (const char* e = getenv_compat("USERALGO_DROP_ABS_LT")) {
    const double v = std::atof(e);
    if (v >= 0.0) o.drop_abs_lt = v;
  }
  return o;
}

double drop_threshold(const AnalysisOptions& opt, int32_t n) {
  return opt.drop_abs_lt >= 0.0 ? opt.drop_abs_lt : ((n >= 50000) ? 1e-20 : 0.0);
}

Decomposition build_decomposition(const CanonicalCoo& a, const AnalysisOptions& opt) {
  Decomposition d;
  const int32_t n = a.n;
  d.n = n;
  const size_t nnz = a.row.size();
  const double drop = drop_threshold(opt, n);

  d.P.resize(static_cast<size_t>(n));
  d.Q.resize(static_cast<size_t>(n));
  std::vector<int32_t> R;
  if (opt.single_block) {
    for (int32_t i = 0; i < n; ++i) d.P[static_cast<size_t>(i)] = d.Q[static_cast<size_t>(i)] = i;
    R = {0, n};
    d.R_raw = R;
    d.nblocks_raw = 1;
    d.nmatch = n;
  } else if (opt.btf) {
    d.P = opt.btf->P;
    d.Q = opt.btf->Q;
    R = opt.btf->R;
    if (static_cast<int32_t>(d.P.size()) != n || static_cast<int32_t>(d.Q.size()) != n || R.size() < 2 ||
        R.front() != 0 || R.back() != n)
      throw std::runtime_error("precomputed BTF ordering does not match the matrix");
    d.nblocks_raw = static_cast<int32_t>(R.size()) - 1;
    d.nmatch = opt.btf->nmatch;
    d.R_raw = R;
    if (opt.merge) R = merge_block_boundaries(R, n, opt.merge_max);
  } else {
    const Csc csc = pattern_csc(a, drop);
    R.assign(static_cast<size_t>(n) + 1, 0);
    int32_t nmatch = 0;
    const int32_t nb = btf_order(n, csc.col_ptr.data(), csc.row_ind.data(), d.P.data(), d.Q.data(),
                                 R.data(), &nmatch);
    if (nb <= 0) throw std::runtime_error("btf_order failed");
    d.nblocks_raw = nb;
    d.nmatch = nmatch;
    for (int32_t k = 0; k < n; ++k) d.Q[static_cast<size_t>(k)] = unflip(d.Q[static_cast<size_t>(k)]);
    R.resize(static_cast<size_t>(nb) + 1);
    d.R_raw = R;
    if (opt.merge) R = merge_block_boundaries(R, n, opt.merge_max);
  }
  d.R = R;
  d.nblocks = static_cast<int32_t>(R.size() - 1);
  d.invP.assign(static_cast<size_t>(n), -1);
  d.invQ.assign(static_cast<size_t>(n), -1);
  for (int32_t i = 0; i < n; ++i) {
    d.invP[static_cast<size_t>(d.P[static_cast<size_t>(i)])] = i;
    d.invQ[static_cast<size_t>(d.Q[static_cast<size_t>(i)])] = i;
  }
  std::vector<int32_t> block_of(static_cast<size_t>(n));
  for (int32_t b = 0; b < d.nblocks; ++b)
    for (int32_t k = R[static_cast<size_t>(b)]; k < R[static_cast<size_t>(b) + 1]; ++k)
      block_of[static_cast<size_t>(k)] = b;

  // UBTF split (ubtf_block_solver.cpp:739-853): count, then fill in canonical order.
  std::vector<int32_t> row_cnt(static_cast<size_t>(n), 0);
  std::vector<int64_t> diag_cnt(static_cast<size_t>(d.nblocks), 0);
  bool violates = false;
  for (size_t k = 0; k < nnz; ++k) {
    if (drop > 0.0 && std::abs(a.val[k]) < drop) continue;
    const int32_t rp = d.invP[static_cast<size_t>(a.row[k])];
    const int32_t cp = d.invQ[static_cast<size_t>(a.col[k])];
    const int32_t br = block_of[static_cast<size_t>(rp)], bc = block_of[static_cast<size_t>(cp)];
    if (bc < br) {
      violates = true;
      continue;
    }
    if (bc == br) diag_cnt[static_cast<size_t>(br)]++;
    else row_cnt[static_cast<size_t>(rp)]++;
  }
  if (violates) throw std::runtime_error("permutation is not UBTF (found lower-block entries)");
  d.off_ptr.assign(static_cast<size_t>(n) + 1, 0);
  for (int32_t i = 0; i < n; ++i) d.off_ptr[static_cast<size_t>(i) + 1] = d.off_ptr[static_cast<size_t>(i)] + row_cnt[static_cast<size_t>(i)];
  d.diag_ptr.assign(static_cast<size_t>(d.nblocks) + 1, 0);
  for (int32_t b = 0; b < d.nblocks; ++b) d.diag_ptr[static_cast<size_t>(b) + 1] = d.diag_ptr[static_cast<size_t>(b)] + diag_cnt[static_cast<size_t>(b)];
  const size_t noff = static_cast<size_t>(d.off_ptr[static_cast<size_t>(n)]);
  const size_t ndiag = static_cast<size_t>(d.diag_ptr[static_cast<size_t>(d.nblocks)]);
  d.off_col.resize(noff);
  d.off_src.resize(noff);
  d.diag_row.resize(ndiag);
  d.diag_col.resize(ndiag);
  d.diag_src.resize(ndiag);
  std::vector<int32_t> onext(d.off_ptr.begin(), d.off_ptr.end() - 1);
  std::vector<int64_t> dnext(d.diag_ptr.begin(), d.diag_ptr.end() - 1);
  for (size_t k = 0; k < nnz; ++k) {
    if (drop > 0.0 && std::abs(a.val[k]) < drop) continue;
    const int32_t rp = d.invP[static_cast<size_t>(a.row[k])];
    const int32_t cp = d.invQ[static_cast<size_t>(a.col[k])];
    const int32_t br = block_of[static_cast<size_t>(rp)], bc = block_of[static_cast<size_t>(cp)];
    if (bc == br) {
      const int64_t q = dnext[static_cast<size_t>(br)]++;
      const int32_t s = R[static_cast<size_t>(br)];
      d.diag_row[static_cast<size_t>(q)] = rp - s;
      d.diag_col[static_cast<size_t>(q)] = cp - s;
      d.diag_src[static_cast<size_t>(q)] = static_cast<int32_t>(k);
    } else {
      const int32_t q = onext[static_cast<size_t>(rp)]++;
      d.off_col[static_cast<size_t>(q)] = cp;
      d.off_src[static_cast<size_t>(q)] = static_cast<int32_t>(k);
    }
  }

  // Block DAG and levels (ubtf_block_solver.cpp:857-909), always built here.
  d.dep_ptr.assign(static_cast<size_t>(d.nblocks) + 1, 0);
  d.dep_idx.clear();
  std::vector<int32_t> seen(static_cast<size_t>(d.nblocks), -1);
  for (int32_t b = 0; b < d.nblocks; ++b) {
    const int32_t s = R[static_cast<size_t>(b)], e = R[static_cast<size_t>(b) + 1];
    for (int32_t r = s; r < e; ++r) {
      for (int32_t p = d.off_ptr[static_cast<size_t>(r)]; p < d.off_ptr[static_cast<size_t>(r) + 1]; ++p) {
        const int32_t c = d.off_col[static_cast<size_t>(p)];
        if (c >= e) {
          const int32_t bc = block_of[static_cast<size_t>(c)];
          if (bc > b && seen[static_cast<size_t>(bc)] != b) {
            seen[static_cast<size_t>(bc)] = b;
            d.dep_idx.push_back(bc);
          }
        }
      }
    }
    d.dep_ptr[static_cast<size_t>(b) + 1] = static_cast<int32_t>(d.dep_idx.size());
  }
  d.level.assign(static_cast<size_t>(d.nblocks), 0);
  d.max_level = 0;
  for (int32_t b = d.nblocks - 1; b >= 0; --b) {
    int32_t lev = 0;
    for (int32_t p = d.dep_ptr[static_cast<size_t>(b)]; p < d.dep_ptr[static_cast<size_t>(b) + 1]; ++p)
      lev = std::max(lev, d.level[static_cast<size_t>(d.dep_idx[static_cast<size_t>(p)])] + 1);
    d.level[static_cast<size_t>(b)] = lev;
    d.max_level = std::max(d.max_level, lev);
  }
  d.level_ptr.assign(static_cast<size_t>(d.max_level) + 2, 0);
  for (int32_t b = 0; b < d.nblocks; ++b) d.level_ptr[static_cast<size_t>(d.level[static_cast<size_t>(b)]) + 1]++;
  for (int32_t l = 0; l <= d.max_level; ++l) d.level_ptr[static_cast<size_t>(l) + 1] += d.level_ptr[static_cast<size_t>(l)];
  d.level_blocks.resize(static_cast<size_t>(d.nblocks));
  std::vector<int32_t> lnext(d.level_ptr.begin(), d.level_ptr.end() - 1);
  for (int32_t b = 0; b < d.nblocks; ++b) d.level_blocks[static_cast<size_t>(lnext[static_cast<size_t>(d.level[static_cast<size_t>(b)])]++)] = b;
  return d;
}

}  // namespace bdlu
