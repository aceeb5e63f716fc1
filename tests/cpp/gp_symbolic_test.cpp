// Independent check of the sparse-LU route's host analysis (gp_plan.cpp):
// the symbolic factorisation of random unit patterns against a dense
// boolean elimination without pivoting, the value positions of the row-wise
// solve tables, and a host emulation of the device kernels' index
// arithmetic over those tables (columns and rows in the kernels' order); and
// the route's configuration from the environment.  Prints "ok" when every
// check passes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "gp.h"
#include "plan.h"

using namespace bdlu;

static int failures = 0;
#define CHECK(c)                                                    \
  do {                                                              \
    if (!(c)) {                                                     \
      std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);       \
      ++failures;                                                   \
    }                                                               \
  } while (0)

// Pattern of L + U of the no-pivot elimination, row-major booleans.
static std::vector<char> dense_fill(int m, const std::vector<int>& r, const std::vector<int>& c) {
  std::vector<char> f(static_cast<size_t>(m) * m, 0);
  for (size_t k = 0; k < r.size(); ++k) f[static_cast<size_t>(r[k]) * m + c[k]] = 1;
  for (int k = 0; k < m; ++k)
    for (int i = k + 1; i < m; ++i) {
      if (!f[static_cast<size_t>(i) * m + k]) continue;
      for (int j = k + 1; j < m; ++j)
        if (f[static_cast<size_t>(k) * m + j]) f[static_cast<size_t>(i) * m + j] = 1;
    }
  return f;
}

// Host emulation of k_gp_factor and k_gp_solve (gp_lu.cu) for unit g with
// the kernels' index expressions, every access bounds-checked against the
// buffers the kernels get; checks that every column (row) the emulation reads
// was finished before (the kernels' flags), L U = A and A x = b.
static void emulate_unit(const Plan& p, int g, int m, const std::vector<int>& r, const std::vector<int>& c,
                         const std::vector<int>& src, const std::vector<double>& a) {
  // The kernel reads vals[asrc]: values indexed by source.
  std::vector<double> vals(static_cast<size_t>(*std::max_element(src.begin(), src.end())) + 1, 0.0);
  for (size_t k = 0; k < src.size(); ++k) vals[static_cast<size_t>(src[k])] = a[k];
  const int64_t nv = p.gp_nnz;
  const size_t na = p.gp_asrc.size();
  std::vector<double> val(static_cast<size_t>(nv), 0.0);
  std::vector<double> x(static_cast<size_t>(p.gp_maxm), 0.0);
  auto IN = [](int64_t i, int64_t n) { return i >= 0 && i < n; };
  const int c0 = p.gp_col0[static_cast<size_t>(g)];
  CHECK(IN(g + 1, static_cast<int64_t>(p.gp_col0.size())));
  std::vector<char> done(static_cast<size_t>(m), 0);
  {
    // Columns ascending: the order every warp's columns follow, and a
    // topological order of the column dependencies.
    for (int j = 0; j < m; ++j) {
      const int cc = c0 + j;
      CHECK(IN(cc + 1, static_cast<int64_t>(p.gp_cptr.size())) && IN(cc + 1, static_cast<int64_t>(p.gp_aptr.size())));
      const int p0 = p.gp_cptr[static_cast<size_t>(cc)], p1 = p.gp_cptr[static_cast<size_t>(cc) + 1];
      const int dp = p.gp_dpos[static_cast<size_t>(cc)];
      CHECK(p0 <= dp && dp < p1 && IN(p1 - 1, nv));
      for (int q = p0; q < p1; ++q) {
        CHECK(IN(p.gp_row[static_cast<size_t>(q)], p.gp_maxm));
        x[static_cast<size_t>(p.gp_row[static_cast<size_t>(q)])] = -0.0;
      }
      for (int q = p.gp_aptr[static_cast<size_t>(cc)]; q < p.gp_aptr[static_cast<size_t>(cc) + 1]; ++q) {
        CHECK(IN(q, static_cast<int64_t>(na)) && IN(p.gp_arow[static_cast<size_t>(q)], p.gp_maxm));
        CHECK(IN(p.gp_asrc[static_cast<size_t>(q)], static_cast<int64_t>(vals.size())));
        x[static_cast<size_t>(p.gp_arow[static_cast<size_t>(q)])] = vals[static_cast<size_t>(p.gp_asrc[static_cast<size_t>(q)])];
      }
      for (int q = p0; q < dp; ++q) {
        const int k = p.gp_row[static_cast<size_t>(q)];
        const double u = x[static_cast<size_t>(k)];
        const int kc = c0 + k;
        CHECK(IN(k, j) && done[static_cast<size_t>(k)]);
        CHECK(IN(kc + 1, static_cast<int64_t>(p.gp_cptr.size())));
        for (int rr = p.gp_dpos[static_cast<size_t>(kc)] + 1; rr < p.gp_cptr[static_cast<size_t>(kc) + 1]; ++rr) {
          CHECK(IN(rr, nv) && IN(p.gp_row[static_cast<size_t>(rr)], p.gp_maxm));
          x[static_cast<size_t>(p.gp_row[static_cast<size_t>(rr)])] -= val[static_cast<size_t>(rr)] * u;
        }
      }
      const double diag = x[static_cast<size_t>(j)];
      for (int q = p0; q < p1; ++q) {
        const double v = x[static_cast<size_t>(p.gp_row[static_cast<size_t>(q)])];
        val[static_cast<size_t>(q)] = q > dp ? v / diag : v;
      }
      done[static_cast<size_t>(j)] = 1;
    }
  }
  // Dense L U against A.
  std::vector<double> L(static_cast<size_t>(m) * m, 0.0), U(static_cast<size_t>(m) * m, 0.0),
      A(static_cast<size_t>(m) * m, 0.0);
  for (size_t k = 0; k < r.size(); ++k) A[static_cast<size_t>(r[k]) * m + c[k]] = a[k];
  for (int j = 0; j < m; ++j) {
    L[static_cast<size_t>(j) * m + j] = 1.0;
    for (int q = p.gp_cptr[static_cast<size_t>(c0 + j)]; q < p.gp_cptr[static_cast<size_t>(c0 + j) + 1]; ++q) {
      const int i = p.gp_row[static_cast<size_t>(q)];
      (i > j ? L : U)[static_cast<size_t>(i) * m + j] = val[static_cast<size_t>(q)];
    }
  }
  double err = 0.0, amax = 0.0;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      double s = 0.0;
      for (int k = 0; k < m; ++k) s += L[static_cast<size_t>(i) * m + k] * U[static_cast<size_t>(k) * m + j];
      err = std::max(err, std::abs(s - A[static_cast<size_t>(i) * m + j]));
      amax = std::max(amax, std::abs(A[static_cast<size_t>(i) * m + j]));
    }
  CHECK(err <= 1e-9 * std::max(1.0, amax));
  // Solve: rows ascending (L), then descending (U), then A x = b.
  std::vector<double> b(static_cast<size_t>(m)), xs;
  for (int i = 0; i < m; ++i) b[static_cast<size_t>(i)] = std::sin(1.0 + i);
  xs = b;
  std::vector<char> ready(static_cast<size_t>(m), 0);
  for (int i = 0; i < m; ++i)
    {
      const int gr = c0 + i;
      double sum = xs[static_cast<size_t>(i)];
      for (int q = p.gp_lrp[static_cast<size_t>(gr)]; q < p.gp_lrp[static_cast<size_t>(gr) + 1]; ++q) {
        CHECK(IN(q, static_cast<int64_t>(p.gp_lci.size())) && IN(p.gp_lpos[static_cast<size_t>(q)], nv));
        CHECK(IN(p.gp_lci[static_cast<size_t>(q)], m) && ready[static_cast<size_t>(p.gp_lci[static_cast<size_t>(q)])]);
        sum -= val[static_cast<size_t>(p.gp_lpos[static_cast<size_t>(q)])] * xs[static_cast<size_t>(p.gp_lci[static_cast<size_t>(q)])];
      }
      xs[static_cast<size_t>(i)] = sum;
      ready[static_cast<size_t>(i)] = 1;
    }
  std::fill(ready.begin(), ready.end(), 0);
  for (int i = m - 1; i >= 0; --i)
    {
      const int gr = c0 + i;
      double sum = xs[static_cast<size_t>(i)];
      for (int q = p.gp_urp[static_cast<size_t>(gr)]; q < p.gp_urp[static_cast<size_t>(gr) + 1]; ++q) {
        CHECK(IN(q, static_cast<int64_t>(p.gp_uci.size())) && IN(p.gp_upos[static_cast<size_t>(q)], nv));
        CHECK(IN(p.gp_uci[static_cast<size_t>(q)], m) && ready[static_cast<size_t>(p.gp_uci[static_cast<size_t>(q)])]);
        sum -= val[static_cast<size_t>(p.gp_upos[static_cast<size_t>(q)])] * xs[static_cast<size_t>(p.gp_uci[static_cast<size_t>(q)])];
      }
      xs[static_cast<size_t>(i)] = sum / val[static_cast<size_t>(p.gp_dpos[static_cast<size_t>(gr)])];
      ready[static_cast<size_t>(i)] = 1;
    }
  double rmax = 0.0;
  for (int i = 0; i < m; ++i) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += A[static_cast<size_t>(i) * m + j] * xs[static_cast<size_t>(j)];
    rmax = std::max(rmax, std::abs(s - b[static_cast<size_t>(i)]));
  }
  CHECK(rmax <= 1e-8);
}

// The route's configuration from the reference's environment knobs
// (ubtf_block_solver.cpp:87-182), BLOCKDAGLU_ names over USERALGO_ ones.
static void check_config() {
  static const char* kNames[] = {"SPARSE_LU_KERNEL", "GP_MAX_N", "GP_FORCE", "DENSE_BLOCK_MAX", "GP_DIAG_TOL",
                                 "GP_PIVOT_TOL", "GP_MIN_ABS_DIAG", "GP_REQUIRE_NO_SWAPS", "GP_SWAP_MAX",
                                 "GP_SWAP_MAX_N", "GP_REQUIRE_NO_TINY_PIVOTS", "GP_SCALE", "GP_DROP_TOL"};
  auto clear = [] {
    for (const char* n : kNames) {
      unsetenv((std::string("USERALGO_") + n).c_str());
      unsetenv((std::string("BLOCKDAGLU_") + n).c_str());
    }
  };
  clear();
  GpConfig c = gp_config_from_env();
  CHECK(c.mode == 0 && c.max_n == 4096 && c.dense_max == 64 && !c.force && !c.unsupported);
  CHECK(c.diag_tol == 1e-3 && c.pivot_tol == 1e-12 && c.min_abs_diag == 1e-12);
  setenv("USERALGO_SPARSE_LU_KERNEL", "GPLU", 1);
  CHECK(gp_config_from_env().mode == 1);
  setenv("BLOCKDAGLU_SPARSE_LU_KERNEL", "klu", 1);
  CHECK(gp_config_from_env().mode == 0);
  unsetenv("BLOCKDAGLU_SPARSE_LU_KERNEL");
  setenv("USERALGO_GP_MAX_N", "80", 1);
  setenv("USERALGO_GP_DIAG_TOL", "0.5", 1);
  setenv("USERALGO_GP_MIN_ABS_DIAG", "-1", 1);  // negative: ignored
  c = gp_config_from_env();
  CHECK(c.max_n == 80 && c.diag_tol == 0.5 && c.min_abs_diag == 1e-12 && !c.unsupported);
  setenv("USERALGO_GP_MAX_N", "0", 1);  // not positive: ignored
  CHECK(gp_config_from_env().max_n == 4096);
  // Settings the device route does not implement turn it off.
  const char* relax[][2] = {{"USERALGO_GP_REQUIRE_NO_SWAPS", "0"}, {"USERALGO_GP_SWAP_MAX", "2"},
                            {"USERALGO_GP_REQUIRE_NO_TINY_PIVOTS", "0"}, {"USERALGO_GP_SCALE", "1"},
                            {"BLOCKDAGLU_GP_DROP_TOL", "1e-3"}};
  for (const auto& kv : relax) {
    setenv(kv[0], kv[1], 1);
    CHECK(gp_config_from_env().unsupported);
    unsetenv(kv[0]);
  }
  CHECK(!gp_config_from_env().unsupported);
  clear();
}

int main() {
  check_config();
  std::mt19937 rng(12345);
  Plan p;
  int units = 0;
  for (int trial = 0; trial < 40; ++trial) {
    const int m = 20 + static_cast<int>(rng() % 180);
    const int per_row = 1 + static_cast<int>(rng() % 4);
    std::vector<int> r, c, src;
    std::vector<char> have(static_cast<size_t>(m) * m, 0);
    auto add = [&](int i, int j) {
      if (have[static_cast<size_t>(i) * m + j]) return;
      have[static_cast<size_t>(i) * m + j] = 1;
      r.push_back(i);
      c.push_back(j);
      src.push_back(static_cast<int>(src.size()) + 1000 * trial);
    };
    for (int i = 0; i < m; ++i) {
      add(i, i);
      add(i, (i + 1) % m);
      for (int t = 0; t < per_row; ++t) add(i, static_cast<int>(rng() % m));
    }
    GpSymbolic s;
    CHECK(gp_symbolic(m, r, c, src, -1, s));
    const std::vector<char> f = dense_fill(m, r, c);
    // Column patterns: exactly the filled entries, rows ascending, diagonal
    // at dpos, A's entries with their sources.
    int64_t nnz = 0;
    for (int j = 0; j < m; ++j) {
      std::vector<int> rows;
      for (int i = 0; i < m; ++i)
        if (f[static_cast<size_t>(i) * m + j]) rows.push_back(i);
      nnz += static_cast<int64_t>(rows.size());
      const int q0 = s.cptr[static_cast<size_t>(j)], q1 = s.cptr[static_cast<size_t>(j) + 1];
      CHECK(static_cast<size_t>(q1 - q0) == rows.size());
      for (int q = q0; q < q1 && static_cast<size_t>(q - q0) < rows.size(); ++q)
        CHECK(s.row[static_cast<size_t>(q)] == rows[static_cast<size_t>(q - q0)]);
      CHECK(s.row[static_cast<size_t>(s.dpos[static_cast<size_t>(j)])] == j);
      for (int q = s.aptr[static_cast<size_t>(j)]; q < s.aptr[static_cast<size_t>(j) + 1]; ++q)
        CHECK(have[static_cast<size_t>(s.arow[static_cast<size_t>(q)]) * m + j]);
    }
    CHECK(s.nnz == nnz);
    CHECK(static_cast<size_t>(s.aptr.back()) == r.size());
    // A fill limit below the pattern stops the symbolic.
    GpSymbolic t;
    CHECK(!gp_symbolic(m, r, c, src, nnz - 1, t));
    // Plan tables: the solve rows reference the right value positions and
    // levels order every dependency.
    const int g = static_cast<int>(p.sparse_units.size());
    gp_append_unit(p, trial, s);
    {
      // Values for the emulation: a dominant diagonal keeps the elimination
      // without pivoting stable.
      std::vector<double> a(r.size());
      for (size_t k = 0; k < r.size(); ++k) a[k] = r[k] == c[k] ? 8.0 + (k % 3) : 0.5 + 0.01 * static_cast<double>(k % 37);
      emulate_unit(p, g, m, r, c, src, a);
    }
    ++units;
    const int c0 = p.gp_col0[static_cast<size_t>(g)];
    CHECK(p.gp_col0[static_cast<size_t>(g) + 1] == c0 + m);
    for (int i = 0; i < m; ++i) {
      int prev = -1;
      for (int q = p.gp_lrp[static_cast<size_t>(c0 + i)]; q < p.gp_lrp[static_cast<size_t>(c0 + i) + 1]; ++q) {
        const int k = p.gp_lci[static_cast<size_t>(q)];
        CHECK(k < i && k > prev && f[static_cast<size_t>(i) * m + k]);
        CHECK(p.gp_row[static_cast<size_t>(p.gp_lpos[static_cast<size_t>(q)])] == i);
        CHECK(p.gp_lpos[static_cast<size_t>(q)] >= p.gp_cptr[static_cast<size_t>(c0 + k)] &&
              p.gp_lpos[static_cast<size_t>(q)] < p.gp_cptr[static_cast<size_t>(c0 + k) + 1]);
        prev = k;
      }
      prev = i;
      for (int q = p.gp_urp[static_cast<size_t>(c0 + i)]; q < p.gp_urp[static_cast<size_t>(c0 + i) + 1]; ++q) {
        const int j = p.gp_uci[static_cast<size_t>(q)];
        CHECK(j > prev && f[static_cast<size_t>(i) * m + j]);
        CHECK(p.gp_row[static_cast<size_t>(p.gp_upos[static_cast<size_t>(q)])] == i);
        CHECK(p.gp_upos[static_cast<size_t>(q)] >= p.gp_cptr[static_cast<size_t>(c0 + j)] &&
              p.gp_upos[static_cast<size_t>(q)] < p.gp_cptr[static_cast<size_t>(c0 + j) + 1]);
        prev = j;
      }
    }
  }
  // A column without its diagonal after fill is refused.
  {
    std::vector<int> r = {1, 0, 2, 1}, c = {0, 1, 1, 2}, src = {0, 1, 2, 3};
    GpSymbolic s;
    CHECK(!gp_symbolic(3, r, c, src, -1, s));
  }
  std::printf("units %d nnz %lld\n", units, static_cast<long long>(p.gp_nnz));
  if (failures) {
    std::printf("%d failures\n", failures);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
