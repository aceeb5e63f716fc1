// C++ API test of the blockdaglu::Solver drop-in (include/blockdaglu/solver.h).
// Mirrors the reference's own test program's cases (apps/tests/main.cpp:93-204:
// input errors, 3x3 solution with duplicates, BLOCK route on known-ones
// systems, export identity) and covers the additions: value-only refactor,
// multi-RHS solve and last_stats().  Prints "ok" and exits 0 on success.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <string>
#include <vector>

#include "blockdaglu/solver.h"

using blockdaglu::CooMatrix;
using blockdaglu::Solver;
using blockdaglu::SolverError;

static int failures = 0;
static void check(bool ok, const std::string& what) {
  if (!ok) {
    ++failures;
    std::fprintf(stderr, "FAIL: %s\n", what.c_str());
  }
}
static bool close(double a, double b, double tol = 1e-9) {
  return std::fabs(a - b) <= tol * std::fmax(1.0, std::fmax(std::fabs(a), std::fabs(b)));
}
static std::vector<double> multiply(const CooMatrix& a, int n, const std::vector<double>& x) {
  std::vector<double> y(static_cast<size_t>(n), 0.0);
  for (const auto& e : a) y[std::get<0>(e)] += std::get<2>(e) * x[std::get<1>(e)];
  return y;
}
static std::vector<double> dense(const CooMatrix& a, int n) {
  std::vector<double> d(static_cast<size_t>(n) * n, 0.0);
  for (const auto& e : a) d[static_cast<size_t>(std::get<0>(e)) * n + std::get<1>(e)] += std::get<2>(e);
  return d;
}

// Tridiagonal-like system of n rows with a coupling column in the middle row.
static CooMatrix chain_matrix(int n, int changed) {
  CooMatrix m;
  for (int r = 0; r < n; ++r) {
    m.emplace_back(r, r, 4.0);
    if (r + 2 < n) m.emplace_back(r, r == n / 2 ? changed : r + 1, 0.25);
    else m.emplace_back(r, r, 0.5);
  }
  return m;
}

int main() {
  {
    Solver s;
    check(s.set_matrix({{-1, 0, 1.0}}), "set_matrix stores a negative index");
    check(!s.analyze() && s.last_error() == SolverError::InvalidIndex, "negative index rejected by analyze");
    Solver t;
    check(t.set_matrix({{0, 0, std::numeric_limits<double>::quiet_NaN()}}), "set_matrix stores NaN");
    check(!t.analyze() && t.last_error() == SolverError::NonFiniteValue, "NaN rejected by analyze");
    Solver u;
    check(!u.factor() && u.last_error() == SolverError::NotPrepared, "factor before analyze");
  }
  {
    setenv("BLOCKDAGLU_MODE", "klu", 1);
    Solver s;
    CooMatrix a{{0, 0, 4.0}, {0, 1, 1.0}, {1, 0, 1.0}, {1, 1, 3.0}, {1, 2, 1.0}, {2, 1, 1.0}, {2, 2, 2.0},
                {0, 0, 1.0}, {0, 0, -1.0}};
    std::vector<double> b{1.0, 2.0, 3.0};
    const double x[3] = {0.2222222222222222, 0.1111111111111111, 1.4444444444444444};
    check(s.set_matrix(a, 3) && s.analyze() && s.factor() && s.solve_in_place(b), "3x3 solve: " + s.last_error_message());
    for (int i = 0; i < 3; ++i) check(close(b[i], x[i]), "3x3 solution entry " + std::to_string(i));
    check(std::string(s.selected_mode()) == "KLU", "MODE=klu selects KLU");
    std::vector<double> bad{1.0, 2.0};
    check(!s.solve_in_place(bad) && s.last_error() == SolverError::InvalidRightHandSide, "wrong rhs size");
  }
  {
    setenv("BLOCKDAGLU_MODE", "block", 1);
    const int n = 1100;
    CooMatrix a = chain_matrix(n, n / 2 + 1);
    Solver s;
    check(s.set_matrix(a, n) && s.analyze() && s.factor(), "block route: " + s.last_error_message());
    check(std::string(s.selected_mode()) == "BLOCK", "MODE=block selects BLOCK");
    std::vector<double> ones(n, 1.0), b = multiply(a, n, ones);
    check(s.solve_in_place(b), "block solve");
    for (int i = 0; i < n; ++i)
      if (!close(b[i], 1.0)) {
        check(false, "block solution entry " + std::to_string(i));
        break;
      }
    // Value-only refactor with doubled values (canonical order = sorted
    // by row then column, duplicates summed).
    CooMatrix sorted;
    {
      std::vector<double> d = dense(a, n);
      for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c)
          if (d[static_cast<size_t>(r) * n + c] != 0.0) sorted.emplace_back(r, c, d[static_cast<size_t>(r) * n + c]);
    }
    std::vector<double> vals;
    for (const auto& e : sorted) vals.push_back(2.0 * std::get<2>(e));
    check(s.refactor_values(vals.data(), vals.size()), "refactor_values: " + s.last_error_message());
    // Three right-hand sides, column-major with leading dimension n + 3.
    const int ldb = n + 3, nrhs = 3;
    std::vector<double> B(static_cast<size_t>(ldb) * nrhs, 0.0);
    for (int k = 0; k < nrhs; ++k) {
      std::vector<double> xk(n, static_cast<double>(k + 1));
      std::vector<double> bk = multiply(a, n, xk);
      for (int i = 0; i < n; ++i) B[static_cast<size_t>(k) * ldb + i] = 2.0 * bk[i];
    }
    check(s.solve_in_place(B.data(), ldb, nrhs), "multi-rhs solve: " + s.last_error_message());
    for (int k = 0; k < nrhs; ++k)
      for (int i = 0; i < n; ++i)
        if (!close(B[static_cast<size_t>(k) * ldb + i], k + 1.0)) {
          check(false, "multi-rhs entry " + std::to_string(k) + "," + std::to_string(i));
          k = nrhs;
          break;
        }
    const auto& st = s.last_stats();
    check(st.n == n && st.residual_inf <= 1e-12, "last_stats: n and residual");
  }
  {
    setenv("BLOCKDAGLU_MODE", "block", 1);
    Solver s;
    CooMatrix a{{0, 0, 100.0}, {0, 1, 20.0}, {0, 2, 7.0}, {1, 0, 30.0}, {1, 1, 80.0}, {1, 3, 5.0},
                {2, 2, 0.25}, {2, 3, 0.05}, {3, 2, 0.10}, {3, 3, 0.50}};
    check(s.set_matrix(a, 4) && s.analyze() && s.factor(), "export factor");
    const auto ra = dense(s.get_rearranged_matrix(), 4), l = dense(s.getL(), 4), u = dense(s.getU(), 4);
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        double v = 0.0;
        for (int k = 0; k < 4; ++k) v += l[r * 4 + k] * u[k * 4 + c];
        check(close(ra[r * 4 + c], v), "export identity at " + std::to_string(r) + "," + std::to_string(c));
      }
    check(!s.getP().empty() && !s.getQ().empty(), "P and Q exports");
  }
  if (failures) {
    std::fprintf(stderr, "%d failure(s)\n", failures);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
