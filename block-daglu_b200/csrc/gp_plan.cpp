// Host side of the sparse-LU route (gp.h): configuration from the
// reference's environment knobs, the symbolic factorisation of a unit and
// the plan tables the device kernels read.
#include "gp.h"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <functional>
#include <queue>
#include <string>

#include "analysis.h"
#include "plan.h"

namespace bdlu {

GpConfig gp_config_from_env() {
  GpConfig c;
  // USERALGO_SPARSE_LU_KERNEL = gp | gplu (ubtf_block_solver.cpp:87-94).
  if (const char* e = getenv_compat("USERALGO_SPARSE_LU_KERNEL")) {
    std::string v(e);
    for (auto& ch : v) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    c.mode = (v == "gp" || v == "gplu") ? 1 : 0;
  }
  if (const char* e = getenv_compat("USERALGO_GP_MAX_N")) {
    const int v = std::atoi(e);
    if (v > 0) c.max_n = v;
  }
  if (const char* e = getenv_compat("USERALGO_GP_FORCE")) c.force = std::atoi(e) != 0;
  if (const char* e = getenv_compat("USERALGO_DENSE_BLOCK_MAX")) {
    const int v = std::atoi(e);
    if (v >= 1) c.dense_max = v;
  }
  if (const char* e = getenv_compat("USERALGO_GP_DIAG_TOL")) {
    const double v = std::atof(e);
    if (v >= 0.0) c.diag_tol = v;
  }
  if (const char* e = getenv_compat("USERALGO_GP_PIVOT_TOL")) {
    const double v = std::atof(e);
    if (v >= 0.0) c.pivot_tol = v;
  }
  if (const char* e = getenv_compat("USERALGO_GP_MIN_ABS_DIAG")) {
    const double v = std::atof(e);
    if (v >= 0.0) c.min_abs_diag = v;
  }
  // The gate's relaxations and the factor's scaling and dropping
  // (ubtf_block_solver.cpp:118-182) are not implemented on the device.
  auto env_int = [](const char* name, int dflt) {
    const char* e = getenv_compat(name);
    return e ? std::atoi(e) : dflt;
  };
  if (env_int("USERALGO_GP_REQUIRE_NO_SWAPS", 1) == 0) c.unsupported = true;
  if (env_int("USERALGO_GP_SWAP_MAX", 0) > 0 && env_int("USERALGO_GP_SWAP_MAX_N", 256) > 0) c.unsupported = true;
  if (env_int("USERALGO_GP_REQUIRE_NO_TINY_PIVOTS", 1) == 0) c.unsupported = true;
  if (env_int("USERALGO_GP_SCALE", 0) != 0) c.unsupported = true;
  if (const char* e = getenv_compat("USERALGO_GP_DROP_TOL"))
    if (std::atof(e) > 0.0) c.unsupported = true;
  return c;
}

bool gp_symbolic(int32_t m, const std::vector<int32_t>& er, const std::vector<int32_t>& ec,
                 const std::vector<int32_t>& esrc, int64_t fill_limit, GpSymbolic& out) {
  out = GpSymbolic{};
  const size_t ne = er.size();
  // A by columns, rows ascending.
  out.aptr.assign(static_cast<size_t>(m) + 1, 0);
  for (size_t k = 0; k < ne; ++k) out.aptr[static_cast<size_t>(ec[k]) + 1]++;
  for (int32_t j = 0; j < m; ++j) out.aptr[static_cast<size_t>(j) + 1] += out.aptr[static_cast<size_t>(j)];
  out.arow.resize(ne);
  out.asrc.resize(ne);
  {
    std::vector<int32_t> nx(out.aptr.begin(), out.aptr.end() - 1);
    for (size_t k = 0; k < ne; ++k) {
      const int32_t q = nx[static_cast<size_t>(ec[k])]++;
      out.arow[static_cast<size_t>(q)] = er[k];
      out.asrc[static_cast<size_t>(q)] = esrc[k];
    }
    for (int32_t j = 0; j < m; ++j) {
      std::vector<std::pair<int32_t, int32_t>> t;
      for (int32_t q = out.aptr[static_cast<size_t>(j)]; q < out.aptr[static_cast<size_t>(j) + 1]; ++q)
        t.emplace_back(out.arow[static_cast<size_t>(q)], out.asrc[static_cast<size_t>(q)]);
      std::sort(t.begin(), t.end());
      for (size_t i = 0; i < t.size(); ++i) {
        out.arow[static_cast<size_t>(out.aptr[static_cast<size_t>(j)]) + i] = t[i].first;
        out.asrc[static_cast<size_t>(out.aptr[static_cast<size_t>(j)]) + i] = t[i].second;
      }
    }
  }
  // Left-looking symbolic: column j's pattern is A(:, j) closed under the
  // L columns of its rows above the diagonal, taken in ascending order (a
  // min-heap: every row an L column adds lies below that column).
  std::vector<std::vector<int32_t>> lcols(static_cast<size_t>(m));
  std::vector<int32_t> mark(static_cast<size_t>(m), -1);
  std::priority_queue<int32_t, std::vector<int32_t>, std::greater<int32_t>> heap;
  std::vector<int32_t> up, lo;
  out.cptr.assign(1, 0);
  out.dpos.resize(static_cast<size_t>(m));
  for (int32_t j = 0; j < m; ++j) {
    up.clear();
    lo.clear();
    bool diag = false;
    auto visit = [&](int32_t i) {
      if (mark[static_cast<size_t>(i)] == j) return;
      mark[static_cast<size_t>(i)] = j;
      if (i < j) heap.push(i);
      else if (i == j) diag = true;
      else lo.push_back(i);
    };
    for (int32_t q = out.aptr[static_cast<size_t>(j)]; q < out.aptr[static_cast<size_t>(j) + 1]; ++q)
      visit(out.arow[static_cast<size_t>(q)]);
    while (!heap.empty()) {
      const int32_t k = heap.top();
      heap.pop();
      up.push_back(k);
      out.flops += 2.0 * static_cast<double>(lcols[static_cast<size_t>(k)].size());
      for (int32_t i : lcols[static_cast<size_t>(k)]) visit(i);
    }
    if (!diag) return false;
    std::sort(lo.begin(), lo.end());
    out.flops += static_cast<double>(lo.size());
    out.dpos[static_cast<size_t>(j)] = out.cptr.back() + static_cast<int32_t>(up.size());
    out.row.insert(out.row.end(), up.begin(), up.end());
    out.row.push_back(j);
    out.row.insert(out.row.end(), lo.begin(), lo.end());
    out.nnz = static_cast<int64_t>(out.row.size());
    if ((fill_limit >= 0 && out.nnz > fill_limit) || out.nnz >= (int64_t{1} << 30)) return false;
    out.cptr.push_back(static_cast<int32_t>(out.nnz));
    lcols[static_cast<size_t>(j)] = lo;
  }
  return true;
}

void gp_append_unit(Plan& p, int32_t u, const GpSymbolic& s) {
  if (p.gp_col0.empty()) {
    for (auto* v : {&p.gp_col0, &p.gp_cptr, &p.gp_aptr, &p.gp_lrp, &p.gp_urp})
      v->assign(1, 0);
  }
  const int32_t m = static_cast<int32_t>(s.cptr.size()) - 1;
  const int32_t base = p.gp_cptr.back();
  const int32_t abase = p.gp_aptr.back();
  p.sparse_units.push_back(u);
  p.gp_col0.push_back(p.gp_col0.back() + m);
  for (int32_t j = 0; j < m; ++j) {
    p.gp_cptr.push_back(base + s.cptr[static_cast<size_t>(j) + 1]);
    p.gp_dpos.push_back(base + s.dpos[static_cast<size_t>(j)]);
    p.gp_aptr.push_back(abase + s.aptr[static_cast<size_t>(j) + 1]);
  }
  p.gp_row.insert(p.gp_row.end(), s.row.begin(), s.row.end());
  p.gp_arow.insert(p.gp_arow.end(), s.arow.begin(), s.arow.end());
  p.gp_asrc.insert(p.gp_asrc.end(), s.asrc.begin(), s.asrc.end());
  // Strict L and strict U by rows, columns ascending (columns are visited in
  // order), with the value positions of the column-compressed factor.
  std::vector<int32_t> lcnt(static_cast<size_t>(m) + 1, 0), ucnt(static_cast<size_t>(m) + 1, 0);
  for (int32_t j = 0; j < m; ++j)
    for (int32_t q = s.cptr[static_cast<size_t>(j)]; q < s.cptr[static_cast<size_t>(j) + 1]; ++q) {
      const int32_t i = s.row[static_cast<size_t>(q)];
      if (i > j) lcnt[static_cast<size_t>(i) + 1]++;
      else if (i < j) ucnt[static_cast<size_t>(i) + 1]++;
    }
  for (int32_t i = 0; i < m; ++i) {
    lcnt[static_cast<size_t>(i) + 1] += lcnt[static_cast<size_t>(i)];
    ucnt[static_cast<size_t>(i) + 1] += ucnt[static_cast<size_t>(i)];
  }
  const int32_t lbase = p.gp_lrp.back(), ubase = p.gp_urp.back();
  for (int32_t i = 0; i < m; ++i) {
    p.gp_lrp.push_back(lbase + lcnt[static_cast<size_t>(i) + 1]);
    p.gp_urp.push_back(ubase + ucnt[static_cast<size_t>(i) + 1]);
  }
  p.gp_lci.resize(static_cast<size_t>(lbase + lcnt[static_cast<size_t>(m)]));
  p.gp_lpos.resize(p.gp_lci.size());
  p.gp_uci.resize(static_cast<size_t>(ubase + ucnt[static_cast<size_t>(m)]));
  p.gp_upos.resize(p.gp_uci.size());
  std::vector<int32_t> ln(lcnt.begin(), lcnt.end() - 1), un(ucnt.begin(), ucnt.end() - 1);
  for (int32_t j = 0; j < m; ++j)
    for (int32_t q = s.cptr[static_cast<size_t>(j)]; q < s.cptr[static_cast<size_t>(j) + 1]; ++q) {
      const int32_t i = s.row[static_cast<size_t>(q)];
      if (i > j) {
        const size_t w = static_cast<size_t>(lbase + ln[static_cast<size_t>(i)]++);
        p.gp_lci[w] = j;
        p.gp_lpos[w] = base + q;
      } else if (i < j) {
        const size_t w = static_cast<size_t>(ubase + un[static_cast<size_t>(i)]++);
        p.gp_uci[w] = j;
        p.gp_upos[w] = base + q;
      }
    }
  p.gp_nnz += s.nnz;
  p.gp_maxm = std::max(p.gp_maxm, m);
  p.gp_flops += s.flops;
}

}  // namespace bdlu
