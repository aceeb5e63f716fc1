// Builds the per-pattern device plan (see plan.h).
#include "plan.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <map>

#include "gp.h"

namespace bdlu {

static double lu_flops(int64_t m) {
  // Partial-pivoting LU: (m-k-1) divisions and (m-k-1)^2 multiply-subtract
  // pairs at step k.
  double f = 0.0;
  for (int64_t k = 0; k < m; ++k) {
    const double r = static_cast<double>(m - k - 1);
    f += r + 2.0 * r * r;
  }
  return f;
}

int64_t build_rtasks(const std::vector<int32_t>& units, const std::vector<int32_t>& sizes, int64_t max_tasks,
                     std::vector<int32_t>& tasks, int32_t& words) {
  tasks.clear();
  words = 0;
  const size_t nu = units.size();
  std::vector<int64_t> nt(nu), vbase(nu);
  int64_t total = 0, steps = 0, w = 1;
  for (size_t q = 0; q < nu; ++q) {
    nt[q] = (sizes[q] + kRPanel - 1) / kRPanel;
    if (nt[q] > 65535) return -1;
    vbase[q] = w;
    w += nt[q] * nt[q];
    steps = std::max(steps, nt[q]);
    // Per step k: 1 D, 2 (nt - k - 1) strips, ceil((nt - k - 1) / 2) (nt - k - 1) updates.
    for (int64_t k = 0; k < nt[q]; ++k) {
      const int64_t r = nt[q] - k - 1;
      total += 1 + 2 * r + (r + 1) / 2 * r;
    }
  }
  if (nu == 0 || total > max_tasks || w > INT32_MAX) return -1;
  tasks.reserve(static_cast<size_t>(total) * 4);
  auto push = [&](size_t q, int64_t k, int64_t i, int64_t j) {
    tasks.push_back(units[q]);
    tasks.push_back(static_cast<int32_t>(k));
    tasks.push_back(static_cast<int32_t>((i << 16) | j));
    tasks.push_back(static_cast<int32_t>(vbase[q]));
  };
  // Step k's panel: D, then the strips of step k + 1's panel, then the rest.
  auto panel = [&](int64_t k) {
    for (size_t q = 0; q < nu; ++q)
      if (nt[q] > k) push(q, k, k, k);
    for (size_t q = 0; q < nu; ++q) {
      for (int64_t t = k + 1; t < nt[q]; ++t) {
        push(q, k, t, k);
        push(q, k, k, t);
      }
    }
  };
  // Step k's updates of step k + 1's panel: the diagonal pair first, then
  // row pair k + 1 and tile column k + 1 alternately.
  auto critical = [&](int64_t k) {
    for (size_t q = 0; q < nu; ++q) {
      if (nt[q] <= k + 1) continue;
      push(q, k, k + 1, k + 1);
      for (int64_t t = 1;; ++t) {
        const bool row = k + 1 + t < nt[q], col = k + 1 + 2 * t < nt[q];
        if (!row && !col) break;
        if (row) push(q, k, k + 1, k + 1 + t);
        if (col) push(q, k, k + 1 + 2 * t, k + 1);
      }
    }
  };
  // Step k's other updates (row pairs from k + 3, tile columns from k + 2),
  // by the step at which their tiles join a panel.
  std::vector<std::array<int64_t, 3>> rest;
  auto others = [&](int64_t k) {
    for (size_t q = 0; q < nu; ++q) {
      rest.clear();
      for (int64_t i = k + 3; i < nt[q]; i += 2)
        for (int64_t j = k + 2; j < nt[q]; ++j) rest.push_back({std::min(i, j), i, j});
      std::sort(rest.begin(), rest.end());
      for (const auto& r : rest) push(q, k, r[1], r[2]);
    }
  };
  for (int64_t k = 0; k < steps; ++k) {
    panel(k);
    if (k > 0) others(k - 1);
    critical(k);
  }
  if (steps > 0) others(steps - 1);
  words = static_cast<int32_t>(w);
  return static_cast<int64_t>(tasks.size() / 4);
}

Plan build_plan(const CanonicalCoo& a, const Decomposition& d, int32_t small_max, const GpConfig* gp) {
  Plan p;
  const int32_t n = d.n;
  p.n = n;
  p.nnz = a.nnz();
  p.small_max = small_max;
  p.ustart = d.R_raw;
  p.nunits = static_cast<int32_t>(p.ustart.size()) - 1;
  const int32_t nu = p.nunits;
  p.unit_of.resize(static_cast<size_t>(n));
  p.ukind.resize(static_cast<size_t>(nu));
  p.lu_off.assign(static_cast<size_t>(nu), -1);
  for (int32_t u = 0; u < nu; ++u) {
    const int32_t s = p.ustart[static_cast<size_t>(u)], e = p.ustart[static_cast<size_t>(u) + 1];
    const int32_t m = e - s;
    for (int32_t r = s; r < e; ++r) p.unit_of[static_cast<size_t>(r)] = u;
    p.ukind[static_cast<size_t>(u)] = (m == 1) ? kUnitScalar : (m <= small_max ? kUnitSmall : kUnitLarge);
    p.max_unit = std::max(p.max_unit, m);
  }
  const double drop = [&] {
    const AnalysisOptions o = analysis_options_from_env();
    return o.drop_abs_lt < 0.0 ? (n >= 50000 ? 1e-20 : 0.0) : o.drop_abs_lt;
  }();
  // Sparse-LU route (gp.h): the units it tries get their no-pivot symbolic
  // factorisation; a unit whose pattern qualifies becomes a sparse unit.
  std::map<int32_t, GpSymbolic> gp_sym;
  p.gp_index.assign(static_cast<size_t>(nu), -1);
  if (gp && gp->mode > 0 && !gp->unsupported) {
    std::vector<int32_t> cand(static_cast<size_t>(nu), 0);
    bool any = false;
    for (int32_t u = 0; u < nu; ++u) {
      const int32_t s0 = p.ustart[static_cast<size_t>(u)];
      const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - s0;
      if (m <= 1 || m <= gp->dense_max || (!gp->force && m > gp->max_n) || m > kGpMaxRows) continue;
      if (std::find(gp->rejected.begin(), gp->rejected.end(), s0) != gp->rejected.end()) continue;
      cand[static_cast<size_t>(u)] = 1;
      any = true;
    }
    if (any) {
      std::map<int32_t, std::array<std::vector<int32_t>, 3>> ent;  // unit -> local rows, cols, sources
      const size_t nz = static_cast<size_t>(a.nnz());
      for (size_t k = 0; k < nz; ++k) {
        if (drop > 0.0 && std::abs(a.val[k]) < drop) continue;
        const int32_t rp = d.invP[static_cast<size_t>(a.row[k])], cp = d.invQ[static_cast<size_t>(a.col[k])];
        const int32_t ur = p.unit_of[static_cast<size_t>(rp)];
        if (ur != p.unit_of[static_cast<size_t>(cp)] || !cand[static_cast<size_t>(ur)]) continue;
        auto& e = ent[ur];
        const int32_t s0 = p.ustart[static_cast<size_t>(ur)];
        e[0].push_back(rp - s0);
        e[1].push_back(cp - s0);
        e[2].push_back(static_cast<int32_t>(k));
      }
      int64_t total = 0;
      for (int32_t u = 0; u < nu; ++u) {
        if (!cand[static_cast<size_t>(u)]) continue;
        const int64_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
        const int64_t limit = gp->mode == 2 ? static_cast<int64_t>(gp->fill_max * static_cast<double>(m * m)) : -1;
        GpSymbolic sym;
        auto& e = ent[u];
        if (gp_symbolic(static_cast<int32_t>(m), e[0], e[1], e[2], limit, sym) && total + sym.nnz < INT32_MAX) {
          total += sym.nnz;
          p.ukind[static_cast<size_t>(u)] = kUnitSparse;
          gp_sym.emplace(u, std::move(sym));
        } else {
          p.gp_symbolic_rejected.push_back(u);
        }
      }
    }
  }
  // Arena: small units first, then large units contiguously (so one memset
  // clears all large slots).  Slots are padded to 32 doubles.
  int64_t off = 0;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) p.lu_large_begin = off;
    for (int32_t u = 0; u < nu; ++u) {
      const int32_t k = p.ukind[static_cast<size_t>(u)];
      if ((pass == 0 && k != kUnitSmall) || (pass == 1 && k != kUnitLarge)) continue;
      const int64_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
      p.lu_off[static_cast<size_t>(u)] = off;
      off += (m * m + 31) / 32 * 32;
      p.dense_entries += m * m;
      p.factor_flops += lu_flops(m);
      (pass == 0 ? p.small_units : p.large_units).push_back(u);
    }
  }
  p.lu_large_end = off;
  p.lu_size = off;
  {
    // Small units by size, cut into buckets at these row counts.
    auto usz = [&](int32_t u) { return p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]; };
    std::stable_sort(p.small_units.begin(), p.small_units.end(), [&](int32_t x, int32_t y) { return usz(x) < usz(y); });
    static const int32_t kCuts[] = {8, 16, 24, 32, 48, 64, 80, 96, 128};
    p.small_bucket_ptr.assign(1, 0);
    size_t q = 0;
    for (int32_t cut : kCuts) {
      const size_t q0 = q;
      while (q < p.small_units.size() && usz(p.small_units[q]) <= cut) ++q;
      if (q > q0) {
        p.small_bucket_ptr.push_back(static_cast<int32_t>(q));
        p.small_bucket_m.push_back(usz(p.small_units[q - 1]));
      }
    }
    if (q < p.small_units.size()) {
      p.small_bucket_ptr.push_back(static_cast<int32_t>(p.small_units.size()));
      p.small_bucket_m.push_back(usz(p.small_units.back()));
    }
  }

  // Split entries into unit-diagonal entries and coupling, canonical order.
  p.sdiag_src.assign(static_cast<size_t>(n), -1);
  for (int32_t u = 0; u < nu; ++u)
    if (p.ukind[static_cast<size_t>(u)] == kUnitScalar) p.sdiag_src[static_cast<size_t>(p.ustart[static_cast<size_t>(u)])] = -2;
  std::vector<int64_t> dcnt(static_cast<size_t>(nu), 0);
  std::vector<int32_t> ccnt(static_cast<size_t>(n), 0);
  const size_t nnz = static_cast<size_t>(a.nnz());
  for (size_t k = 0; k < nnz; ++k) {
    if (drop > 0.0 && std::abs(a.val[k]) < drop) continue;
    const int32_t rp = d.invP[static_cast<size_t>(a.row[k])], cp = d.invQ[static_cast<size_t>(a.col[k])];
    const int32_t ur = p.unit_of[static_cast<size_t>(rp)], uc = p.unit_of[static_cast<size_t>(cp)];
    if (ur == uc) {
      if (p.ukind[static_cast<size_t>(ur)] == kUnitScalar) p.sdiag_src[static_cast<size_t>(rp)] = static_cast<int32_t>(k);
      else dcnt[static_cast<size_t>(ur)]++;
    } else {
      ccnt[static_cast<size_t>(rp)]++;
    }
  }
  p.dent_ptr.assign(static_cast<size_t>(nu) + 1, 0);
  for (int32_t u = 0; u < nu; ++u) p.dent_ptr[static_cast<size_t>(u) + 1] = p.dent_ptr[static_cast<size_t>(u)] + dcnt[static_cast<size_t>(u)];
  p.cpl_ptr.assign(static_cast<size_t>(n) + 1, 0);
  for (int32_t r = 0; r < n; ++r) p.cpl_ptr[static_cast<size_t>(r) + 1] = p.cpl_ptr[static_cast<size_t>(r)] + ccnt[static_cast<size_t>(r)];
  p.dent_pos.resize(static_cast<size_t>(p.dent_ptr[static_cast<size_t>(nu)]));
  p.dent_src.resize(p.dent_pos.size());
  p.cpl_col.resize(static_cast<size_t>(p.cpl_ptr[static_cast<size_t>(n)]));
  p.cpl_src.resize(p.cpl_col.size());
  std::vector<int64_t> dnext(p.dent_ptr.begin(), p.dent_ptr.end() - 1);
  std::vector<int32_t> cnext(p.cpl_ptr.begin(), p.cpl_ptr.end() - 1);
  for (size_t k = 0; k < nnz; ++k) {
    if (drop > 0.0 && std::abs(a.val[k]) < drop) continue;
    const int32_t rp = d.invP[static_cast<size_t>(a.row[k])], cp = d.invQ[static_cast<size_t>(a.col[k])];
    const int32_t ur = p.unit_of[static_cast<size_t>(rp)], uc = p.unit_of[static_cast<size_t>(cp)];
    if (ur == uc) {
      if (p.ukind[static_cast<size_t>(ur)] == kUnitScalar) continue;
      const int32_t s = p.ustart[static_cast<size_t>(ur)];
      const int32_t m = p.ustart[static_cast<size_t>(ur) + 1] - s;
      const int64_t q = dnext[static_cast<size_t>(ur)]++;
      // Small units are column-major, large units row-major.
      p.dent_pos[static_cast<size_t>(q)] = (p.ukind[static_cast<size_t>(ur)] == kUnitLarge)
                                               ? (rp - s) * m + (cp - s)
                                               : (cp - s) * m + (rp - s);
      p.dent_src[static_cast<size_t>(q)] = static_cast<int32_t>(k);
    } else {
      const int32_t q = cnext[static_cast<size_t>(rp)]++;
      p.cpl_col[static_cast<size_t>(q)] = cp;
      p.cpl_src[static_cast<size_t>(q)] = static_cast<int32_t>(k);
    }
  }

  // Unit DAG levels from the coupling (dependencies point to higher units).
  p.ulevel.assign(static_cast<size_t>(nu), 0);
  p.umax_level = 0;
  for (int32_t u = nu - 1; u >= 0; --u) {
    int32_t lev = 0;
    for (int32_t r = p.ustart[static_cast<size_t>(u)]; r < p.ustart[static_cast<size_t>(u) + 1]; ++r)
      for (int32_t q = p.cpl_ptr[static_cast<size_t>(r)]; q < p.cpl_ptr[static_cast<size_t>(r) + 1]; ++q)
        lev = std::max(lev, p.ulevel[static_cast<size_t>(p.unit_of[static_cast<size_t>(p.cpl_col[static_cast<size_t>(q)])])] + 1);
    p.ulevel[static_cast<size_t>(u)] = lev;
    p.umax_level = std::max(p.umax_level, lev);
  }
  const int32_t nl = p.umax_level + 1;
  p.lvl_scalar_ptr.assign(static_cast<size_t>(nl) + 1, 0);
  p.lvl_dense_ptr.assign(static_cast<size_t>(nl) + 1, 0);
  p.lvl_large_ptr.assign(static_cast<size_t>(nl) + 1, 0);
  for (int32_t u = 0; u < nu; ++u) {
    const int32_t l = p.ulevel[static_cast<size_t>(u)];
    const int32_t k = p.ukind[static_cast<size_t>(u)];
    if (k == kUnitScalar) p.lvl_scalar_ptr[static_cast<size_t>(l) + 1]++;
    else if (k == kUnitSmall) p.lvl_dense_ptr[static_cast<size_t>(l) + 1]++;
    else if (k == kUnitLarge) p.lvl_large_ptr[static_cast<size_t>(l) + 1]++;
  }
  // Sparse units by level (g indices, in unit order).
  p.lvl_sparse_ptr.assign(static_cast<size_t>(nl) + 1, 0);
  for (const auto& kv : gp_sym) {
    p.gp_index[static_cast<size_t>(kv.first)] = static_cast<int32_t>(p.sparse_units.size());
    gp_append_unit(p, kv.first, kv.second);
    p.lvl_sparse_ptr[static_cast<size_t>(p.ulevel[static_cast<size_t>(kv.first)]) + 1]++;
  }
  for (int32_t l = 0; l < nl; ++l) p.lvl_sparse_ptr[static_cast<size_t>(l) + 1] += p.lvl_sparse_ptr[static_cast<size_t>(l)];
  p.lvl_sparse.resize(p.sparse_units.size());
  {
    std::vector<int32_t> gn(p.lvl_sparse_ptr.begin(), p.lvl_sparse_ptr.end() - 1);
    for (size_t g = 0; g < p.sparse_units.size(); ++g)
      p.lvl_sparse[static_cast<size_t>(gn[static_cast<size_t>(p.ulevel[static_cast<size_t>(p.sparse_units[g])])]++)] =
          static_cast<int32_t>(g);
  }
  p.factor_flops += p.gp_flops;
  for (int32_t l = 0; l < nl; ++l) {
    p.lvl_scalar_ptr[static_cast<size_t>(l) + 1] += p.lvl_scalar_ptr[static_cast<size_t>(l)];
    p.lvl_dense_ptr[static_cast<size_t>(l) + 1] += p.lvl_dense_ptr[static_cast<size_t>(l)];
    p.lvl_large_ptr[static_cast<size_t>(l) + 1] += p.lvl_large_ptr[static_cast<size_t>(l)];
  }
  p.lvl_scalar.resize(static_cast<size_t>(p.lvl_scalar_ptr[static_cast<size_t>(nl)]));
  p.lvl_dense.resize(static_cast<size_t>(p.lvl_dense_ptr[static_cast<size_t>(nl)]));
  p.lvl_large.resize(static_cast<size_t>(p.lvl_large_ptr[static_cast<size_t>(nl)]));
  {
    std::vector<int32_t> sn(p.lvl_scalar_ptr.begin(), p.lvl_scalar_ptr.end() - 1);
    std::vector<int32_t> dn(p.lvl_dense_ptr.begin(), p.lvl_dense_ptr.end() - 1);
    std::vector<int32_t> ln(p.lvl_large_ptr.begin(), p.lvl_large_ptr.end() - 1);
    for (int32_t u = 0; u < nu; ++u) {
      const int32_t l = p.ulevel[static_cast<size_t>(u)];
      const int32_t k = p.ukind[static_cast<size_t>(u)];
      if (k == kUnitScalar)
        p.lvl_scalar[static_cast<size_t>(sn[static_cast<size_t>(l)]++)] = p.ustart[static_cast<size_t>(u)];
      else if (k == kUnitSmall)
        p.lvl_dense[static_cast<size_t>(dn[static_cast<size_t>(l)]++)] = u;
      else if (k == kUnitLarge)
        p.lvl_large[static_cast<size_t>(ln[static_cast<size_t>(l)]++)] = u;
    }
  }
  p.lvl_dense_maxm.assign(static_cast<size_t>(nl), 0);
  for (int32_t l = 0; l < nl; ++l)
    for (int32_t q = p.lvl_dense_ptr[static_cast<size_t>(l)]; q < p.lvl_dense_ptr[static_cast<size_t>(l) + 1]; ++q) {
      const int32_t u = p.lvl_dense[static_cast<size_t>(q)];
      p.lvl_dense_maxm[static_cast<size_t>(l)] =
          std::max(p.lvl_dense_maxm[static_cast<size_t>(l)], p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]);
    }
  // Large units of a level: largest first, so the longest tile chain claims
  // its CTAs first.
  auto usize = [&](int32_t u) { return p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]; };
  for (int32_t l = 0; l < nl; ++l)
    std::stable_sort(p.lvl_large.begin() + p.lvl_large_ptr[static_cast<size_t>(l)],
                     p.lvl_large.begin() + p.lvl_large_ptr[static_cast<size_t>(l) + 1],
                     [&](int32_t a, int32_t b) { return usize(a) > usize(b); });
  p.lvl_large_tile0.assign(p.lvl_large.size() + 1, 0);
  for (size_t q = 0; q < p.lvl_large.size(); ++q)
    p.lvl_large_tile0[q + 1] = p.lvl_large_tile0[q] + (usize(p.lvl_large[q]) + kSolveTile - 1) / kSolveTile;
  p.large_tiles = p.lvl_large_tile0.back();

  // Blocked-LU step tables for large units.
  int32_t max_large = 0;
  for (int32_t u : p.large_units) max_large = std::max(max_large, p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]);
  p.nsteps = (max_large + kPanel - 1) / kPanel;
  p.step_ptr.assign(static_cast<size_t>(p.nsteps) + 1, 0);
  for (int32_t st = 0; st < p.nsteps; ++st) {
    const int32_t k0 = st * kPanel;
    int32_t tpre = 0, gpre = 0, rows = 0;
    for (int32_t u : p.large_units) {
      const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
      if (m <= k0) continue;
      rows = std::max(rows, m - k0);
      const int32_t nb = std::min(kPanel, m - k0);
      const int32_t rest = m - k0 - nb;
      p.step_unit.push_back(u);
      p.step_trsm_pref.push_back(tpre);
      p.step_gemm_pref.push_back(gpre);
      tpre += (m + kTrsmCols - 1) / kTrsmCols;
      const int32_t t = (rest + kGemmTile - 1) / kGemmTile;
      gpre += t * t;
    }
    p.step_ptr[static_cast<size_t>(st) + 1] = static_cast<int32_t>(p.step_unit.size());
    p.step_trsm_total.push_back(tpre);
    p.step_gemm_total.push_back(gpre);
    p.step_max_rows.push_back(rows);
  }

  // Value-only refactor steps (kRPanel columns).
  p.rsteps = (max_large + kRPanel - 1) / kRPanel;
  p.rstep_ptr.assign(static_cast<size_t>(p.rsteps) + 1, 0);
  for (int32_t st = 0; st < p.rsteps; ++st) {
    const int32_t k0 = st * kRPanel;
    int32_t spre = 0, apre = 0, bpre = 0, act = 0;
    for (int32_t u : p.large_units) {
      const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
      if (m <= k0) continue;
      const int32_t rest = m - k0 - std::min(kRPanel, m - k0);
      const int32_t chunks = (rest + kRPanel - 1) / kRPanel;
      const int32_t nti = (rest + kRTileM - 1) / kRTileM, ntj = (rest + kRTileN - 1) / kRTileN;
      p.rstep_unit.push_back(u);
      p.rstep_strip_pref.push_back(spre);
      p.rstep_ga_pref.push_back(apre);
      p.rstep_gb_pref.push_back(bpre);
      spre += std::max(1, 2 * chunks);        // at least one CTA factors the diagonal block
      apre += rest > 0 ? nti + ntj - 1 : 1;   // part a places the factored block
      bpre += rest > 0 ? (nti - 1) * (ntj - 1) : 0;
      ++act;
    }
    p.rstep_ptr[static_cast<size_t>(st) + 1] = static_cast<int32_t>(p.rstep_unit.size());
    p.rstep_strip_total.push_back(spre);
    p.rstep_ga_total.push_back(apre);
    p.rstep_gb_total.push_back(bpre);
    p.rmax_active = std::max(p.rmax_active, act);
  }

  {
    std::vector<int32_t> sizes;
    for (int32_t u : p.large_units)
      sizes.push_back(p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]);
    const int64_t nt = build_rtasks(p.large_units, sizes, kRTaskMax, p.rtask, p.rt_words);
    p.rtasks = nt > 0 ? static_cast<int32_t>(nt) : 0;
  }

  // Canonical CSR row pointer (original coordinates) for the residual.
  p.csr_ptr.assign(static_cast<size_t>(n) + 1, 0);
  for (size_t k = 0; k < nnz; ++k) p.csr_ptr[static_cast<size_t>(a.row[k]) + 1]++;
  for (int32_t r = 0; r < n; ++r) p.csr_ptr[static_cast<size_t>(r) + 1] += p.csr_ptr[static_cast<size_t>(r)];
  return p;
}

}  // namespace bdlu
