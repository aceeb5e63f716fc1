// Host-side integration of the sparse-LU route into the device plan
// (plan.cpp build_plan with a GpConfig), on a real decomposition of a small
// block system: which units become sparse, that the dense tables leave them
// out, that every level lists them once, that their entries map back to the
// canonical matrix, and how the fill limit, rejected units and an unsupported
// configuration change the routes.  Prints "ok" when every check passes.
#include <algorithm>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "analysis.h"
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

// Block upper triangular system: irreducible blocks (diagonal, cyclic chain,
// extra entries) with coupling above the blocks.
static CanonicalCoo make_system(const std::vector<int>& sizes, std::mt19937& rng) {
  std::vector<int32_t> r, c;
  std::vector<double> v;
  std::uniform_real_distribution<double> mag(0.5, 2.0);
  int off = 0, n = 0;
  for (int m : sizes) n += m;
  for (int m : sizes) {
    for (int i = 0; i < m; ++i) {
      r.push_back(off + i); c.push_back(off + i); v.push_back(4.0 * mag(rng));
      r.push_back(off + i); c.push_back(off + (i + 1) % m); v.push_back(mag(rng));
      r.push_back(off + i); c.push_back(off + static_cast<int>(rng() % m)); v.push_back(mag(rng));
      if (off + m < n && i % 3 == 0) {
        r.push_back(off + i);
        c.push_back(off + m + static_cast<int>(rng() % (n - off - m)));
        v.push_back(0.1 * mag(rng));
      }
    }
    off += m;
  }
  CanonicalCoo a;
  std::string msg;
  const Status st = canonicalize(r.data(), c.data(), v.data(), static_cast<int64_t>(r.size()), n, a, msg);
  CHECK(st == Status::Ok);
  return a;
}

static int usize(const Plan& p, int u) { return p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]; }

static void check_plan(const Plan& p, const CanonicalCoo& a, const Decomposition& d, const GpConfig& gp) {
  // Routes: sparse exactly for the candidates the symbolic kept.
  int nsparse = 0;
  for (int u = 0; u < p.nunits; ++u) {
    const int m = usize(p, u);
    const bool cand = m > 1 && m > gp.dense_max && m <= gp.max_n;
    const bool sym_rej = std::find(p.gp_symbolic_rejected.begin(), p.gp_symbolic_rejected.end(), u) !=
                         p.gp_symbolic_rejected.end();
    if (p.ukind[static_cast<size_t>(u)] == kUnitSparse) {
      ++nsparse;
      CHECK(cand && !sym_rej);
      CHECK(p.lu_off[static_cast<size_t>(u)] == -1);
      CHECK(p.gp_index[static_cast<size_t>(u)] >= 0 && p.sparse_units[static_cast<size_t>(p.gp_index[static_cast<size_t>(u)])] == u);
    } else {
      CHECK(p.gp_index[static_cast<size_t>(u)] == -1);
    }
  }
  CHECK(nsparse == static_cast<int>(p.sparse_units.size()));
  // The dense tables leave sparse units out; the sparse levels list each once.
  for (int u : p.small_units) CHECK(p.ukind[static_cast<size_t>(u)] == kUnitSmall);
  for (int u : p.large_units) CHECK(p.ukind[static_cast<size_t>(u)] == kUnitLarge);
  for (int u : p.lvl_dense) CHECK(p.ukind[static_cast<size_t>(u)] == kUnitSmall);
  for (int u : p.lvl_large) CHECK(p.ukind[static_cast<size_t>(u)] == kUnitLarge);
  std::vector<int> seen(p.sparse_units.size(), 0);
  const int nl = p.umax_level + 1;
  CHECK(static_cast<int>(p.lvl_sparse_ptr.size()) == nl + 1);
  for (int l = 0; l < nl; ++l)
    for (int q = p.lvl_sparse_ptr[static_cast<size_t>(l)]; q < p.lvl_sparse_ptr[static_cast<size_t>(l) + 1]; ++q) {
      const int g = p.lvl_sparse[static_cast<size_t>(q)];
      seen[static_cast<size_t>(g)]++;
      CHECK(p.ulevel[static_cast<size_t>(p.sparse_units[static_cast<size_t>(g)])] == l);
    }
  for (int x : seen) CHECK(x == 1);
  // The dense arena holds the dense units only.
  int64_t arena = 0;
  for (int u = 0; u < p.nunits; ++u)
    if (p.ukind[static_cast<size_t>(u)] == kUnitSmall || p.ukind[static_cast<size_t>(u)] == kUnitLarge)
      arena += (static_cast<int64_t>(usize(p, u)) * usize(p, u) + 31) / 32 * 32;
  CHECK(arena == p.lu_size);
  // A's entries of a sparse unit point back to canonical entries of its block.
  for (size_t g = 0; g < p.sparse_units.size(); ++g) {
    const int u = p.sparse_units[g];
    const int s0 = p.ustart[static_cast<size_t>(u)], m = usize(p, u);
    const int c0 = p.gp_col0[g];
    CHECK(p.gp_col0[g + 1] - c0 == m);
    int64_t cnt = 0;
    for (int j = 0; j < m; ++j)
      for (int q = p.gp_aptr[static_cast<size_t>(c0 + j)]; q < p.gp_aptr[static_cast<size_t>(c0 + j) + 1]; ++q) {
        const int k = p.gp_asrc[static_cast<size_t>(q)];
        CHECK(d.invP[static_cast<size_t>(a.row[static_cast<size_t>(k)])] == s0 + p.gp_arow[static_cast<size_t>(q)]);
        CHECK(d.invQ[static_cast<size_t>(a.col[static_cast<size_t>(k)])] == s0 + j);
        ++cnt;
      }
    int64_t expect = 0;
    for (size_t k = 0; k < a.row.size(); ++k) {
      const int rp = d.invP[static_cast<size_t>(a.row[k])], cp = d.invQ[static_cast<size_t>(a.col[k])];
      expect += (rp >= s0 && rp < s0 + m && cp >= s0 && cp < s0 + m) ? 1 : 0;
    }
    CHECK(cnt == expect);
  }
}

int main() {
  std::mt19937 rng(7);
  const CanonicalCoo a = make_system({30, 70, 120, 20, 200, 90, 40}, rng);
  AnalysisOptions opt = analysis_options_from_env();
  const Decomposition d = build_decomposition(a, opt);
  const Plan dense = build_plan(a, d, 169, nullptr);
  CHECK(dense.sparse_units.empty());

  GpConfig gp;
  gp.mode = 1;
  const Plan p = build_plan(a, d, 169, &gp);
  check_plan(p, a, d, gp);
  int cands = 0;
  for (int u = 0; u < p.nunits; ++u) cands += (usize(p, u) > gp.dense_max && usize(p, u) <= gp.max_n) ? 1 : 0;
  CHECK(cands >= 3);
  CHECK(static_cast<int>(p.sparse_units.size() + p.gp_symbolic_rejected.size()) == cands);
  CHECK(!p.sparse_units.empty());
  CHECK(p.factor_flops < dense.factor_flops);

  // A unit rejected earlier stays dense.
  GpConfig rej = gp;
  const int u0 = p.sparse_units.front();
  rej.rejected.push_back(p.ustart[static_cast<size_t>(u0)]);
  const Plan pr = build_plan(a, d, 169, &rej);
  check_plan(pr, a, d, rej);
  CHECK(pr.ukind[static_cast<size_t>(u0)] != kUnitSparse);
  CHECK(pr.sparse_units.size() + 1 == p.sparse_units.size());

  // A fill limit below every unit's pattern keeps them all dense, reported.
  GpConfig tight = gp;
  tight.mode = 2;
  tight.fill_max = 1e-6;
  const Plan pt = build_plan(a, d, 169, &tight);
  check_plan(pt, a, d, tight);
  CHECK(pt.sparse_units.empty() && static_cast<int>(pt.gp_symbolic_rejected.size()) == cands);

  // An unsupported configuration turns the route off.
  GpConfig off = gp;
  off.unsupported = true;
  CHECK(build_plan(a, d, 169, &off).sparse_units.empty());

  if (failures) {
    std::printf("%d failures\n", failures);
    return 1;
  }
  std::printf("sparse units %zu of %d candidates\nok\n", p.sparse_units.size(), cands);
  return 0;
}
