// Seeded synthetic sparse systems standing in for the reference's private
// benchmark set.  Each generator builds A in block-ordered coordinates with
// irreducible diagonal blocks and strictly-upper block coupling, applies random
// row and column permutations (which BTF must undo) and returns the canonical
// COO (sorted by (row, col), no duplicates), x_true and b = A x_true.
//
// Builder choices (the matrix families follow the workload descriptions; the
// reference ships no generator):
//  * RNG: xoshiro256** seeded through splitmix64; uniform doubles use the top
//    53 bits; normals use Box-Muller.
//  * "block"   family: m ~ U{10..90} rescaled (largest remainder) to sum n;
//    cycle i->(i+1) mod m plus 4 random intra-block entries per row, N(0,1);
//    one coupling entry per row into a strictly later block, N(0, 0.1^2);
//    a_ii = 0.5 * sum_j!=i |a_ij| + N(0, 0.1^2).
//  * "circuit" family: Pareto(alpha = 1.5, x_m = 10) block sizes clipped to
//    [1, 20000] plus 1x1 blocks up to n, shuffled; Pareto rows get cycle + 3
//    random intra entries + 1 coupling entry, 1x1 rows 5 coupling entries
//    (average 6 per row); 50 bus rows (early blocks) and 50 bus columns (late
//    blocks) with 500 extra coupling entries each; off-diagonal values have
//    log-uniform magnitude in [1e-3, 1e3] and random sign; diagonal as above.
//  * "precision" family: nbig dense-ish blocks of U{lo..hi} rows with ~20
//    entries per row, plus Pareto small blocks for ~10% of the rows; the
//    diagonal of the large blocks is scaled by a per-row geometric ramp so
//    that the block condition grows to about the requested kappa.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "bdlu.h"

namespace {

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t z = seed;
    for (auto& w : s) {
      z += 0x9e3779b97f4a7c15ull;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
      x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
      w = x ^ (x >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }  // [0,1)
  double uniform_pos() { return (static_cast<double>(next() >> 11) + 1.0) * 0x1.0p-53; }  // (0,1]
  int64_t below(int64_t k) { return static_cast<int64_t>(uniform() * static_cast<double>(k)); }
  double normal() {
    const double u1 = uniform_pos(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct RowEntry {
  int32_t col;
  double val;
};

}  // namespace

struct bdlu_synth {
  int32_t n = 0;
  int32_t nrhs = 1;
  uint64_t seed = 0;
  std::vector<int32_t> row, col;
  std::vector<double> val;
  std::vector<double> x_true;  // n * nrhs, column-major
  std::vector<double> b;       // n * nrhs
  std::vector<int32_t> block_sizes;  // generator block sizes in generator order
};

namespace {

void dedupe_row(std::vector<RowEntry>& r) {
  std::stable_sort(r.begin(), r.end(), [](const RowEntry& a, const RowEntry& b) { return a.col < b.col; });
  size_t w = 0;
  for (size_t i = 0; i < r.size(); ++i) {
    if (w > 0 && r[w - 1].col == r[i].col) continue;
    r[w++] = r[i];
  }
  r.resize(w);
}

// Finishes a generator: diagonal rule, permutation, canonical order, x_true, b.
void finish(bdlu_synth& s, std::vector<std::vector<RowEntry>>& rows, Rng& rng,
            const std::vector<double>* diag_scale) {
  const int32_t n = s.n;
  for (int32_t i = 0; i < n; ++i) {
    auto& r = rows[static_cast<size_t>(i)];
    dedupe_row(r);
    double sum = 0.0;
    for (const auto& e : r) sum += std::fabs(e.val);
    const double noise = 0.1 * rng.normal();
    double d = 0.5 * sum + (diag_scale ? noise * (*diag_scale)[static_cast<size_t>(i)] : noise);
    if (d == 0.0) d = 1.0;
    r.push_back(RowEntry{i, d});
  }
  std::vector<int32_t> pr(static_cast<size_t>(n)), pc(static_cast<size_t>(n));
  std::iota(pr.begin(), pr.end(), 0);
  std::iota(pc.begin(), pc.end(), 0);
  for (int32_t i = n - 1; i > 0; --i) std::swap(pr[static_cast<size_t>(i)], pr[static_cast<size_t>(rng.below(i + 1))]);
  for (int32_t i = n - 1; i > 0; --i) std::swap(pc[static_cast<size_t>(i)], pc[static_cast<size_t>(rng.below(i + 1))]);
  // Row pr[i] of the output holds generator row i; column pc[j] holds column j.
  std::vector<int32_t> inv_pr(static_cast<size_t>(n));
  for (int32_t i = 0; i < n; ++i) inv_pr[static_cast<size_t>(pr[static_cast<size_t>(i)])] = i;
  size_t nnz = 0;
  for (const auto& r : rows) nnz += r.size();
  s.row.clear();
  s.col.clear();
  s.val.clear();
  s.row.reserve(nnz);
  s.col.reserve(nnz);
  s.val.reserve(nnz);
  std::vector<RowEntry> tmp;
  for (int32_t out_r = 0; out_r < n; ++out_r) {
    const auto& r = rows[static_cast<size_t>(inv_pr[static_cast<size_t>(out_r)])];
    tmp.clear();
    for (const auto& e : r) tmp.push_back(RowEntry{pc[static_cast<size_t>(e.col)], e.val});
    std::sort(tmp.begin(), tmp.end(), [](const RowEntry& a, const RowEntry& b) { return a.col < b.col; });
    for (const auto& e : tmp) {
      s.row.push_back(out_r);
      s.col.push_back(e.col);
      s.val.push_back(e.val);
    }
  }
  s.x_true.resize(static_cast<size_t>(n) * static_cast<size_t>(s.nrhs));
  for (auto& x : s.x_true) x = 2.0 * rng.uniform() - 1.0;
  s.b.assign(static_cast<size_t>(n) * static_cast<size_t>(s.nrhs), 0.0);
  for (int32_t k = 0; k < s.nrhs; ++k) {
    const double* x = s.x_true.data() + static_cast<size_t>(k) * static_cast<size_t>(n);
    double* bb = s.b.data() + static_cast<size_t>(k) * static_cast<size_t>(n);
    for (size_t p = 0; p < s.row.size(); ++p) bb[s.row[p]] += s.val[p] * x[s.col[p]];
  }
}

std::vector<int32_t> rescaled_uniform_sizes(Rng& rng, int32_t n, int32_t nb, int32_t lo, int32_t hi) {
  if (nb > n) nb = n;
  if (nb < 1) nb = 1;
  std::vector<double> raw(static_cast<size_t>(nb));
  double tot = 0.0;
  for (auto& r : raw) {
    r = static_cast<double>(lo + rng.below(hi - lo + 1));
    tot += r;
  }
  std::vector<int32_t> sz(static_cast<size_t>(nb));
  std::vector<std::pair<double, int32_t>> frac(static_cast<size_t>(nb));
  int64_t used = 0;
  for (int32_t i = 0; i < nb; ++i) {
    const double t = raw[static_cast<size_t>(i)] * static_cast<double>(n) / tot;
    int32_t f = static_cast<int32_t>(std::floor(t));
    if (f < 1) f = 1;
    sz[static_cast<size_t>(i)] = f;
    used += f;
    frac[static_cast<size_t>(i)] = {t - std::floor(t), i};
  }
  std::stable_sort(frac.begin(), frac.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  int64_t rem = n - used;
  for (size_t k = 0; rem > 0; k = (k + 1) % frac.size(), --rem) sz[static_cast<size_t>(frac[k].second)]++;
  for (size_t k = sz.size(); rem < 0 && k-- > 0;) {
    while (rem < 0 && sz[k] > 1) {
      sz[k]--;
      rem++;
    }
  }
  return sz;
}

void gen_block_family(bdlu_synth& s, Rng& rng, int32_t n, int32_t nb) {
  s.n = n;
  const std::vector<int32_t> sz = rescaled_uniform_sizes(rng, n, nb, 10, 90);
  s.block_sizes = sz;
  std::vector<int32_t> off(sz.size() + 1, 0);
  for (size_t b = 0; b < sz.size(); ++b) off[b + 1] = off[b] + sz[b];
  std::vector<std::vector<RowEntry>> rows(static_cast<size_t>(n));
  for (size_t b = 0; b < sz.size(); ++b) {
    const int32_t m = sz[b], o = off[b];
    for (int32_t i = 0; i < m; ++i) {
      auto& r = rows[static_cast<size_t>(o + i)];
      if (m > 1) r.push_back(RowEntry{o + (i + 1) % m, rng.normal()});
      for (int t = 0; t < 4 && m > 1; ++t) {
        const int32_t c = static_cast<int32_t>(rng.below(m));
        const double v = rng.normal();
        if (c != i) r.push_back(RowEntry{o + c, v});
      }
      if (b + 1 < sz.size()) {
        const int32_t lo = off[b + 1];
        const int32_t c = lo + static_cast<int32_t>(rng.below(n - lo));
        r.push_back(RowEntry{c, 0.1 * rng.normal()});
      }
    }
  }
  finish(s, rows, rng, nullptr);
}

double loguniform_signed(Rng& rng) {
  const double mag = std::pow(10.0, -3.0 + 6.0 * rng.uniform());
  return (rng.next() >> 63) ? -mag : mag;
}

// Pareto(alpha=1.5, x_m=10) sizes clipped to [1, clip]; at most `budget` rows.
std::vector<int32_t> pareto_sizes(Rng& rng, int32_t count, int32_t clip, int64_t budget) {
  std::vector<int32_t> out;
  int64_t used = 0;
  for (int32_t k = 0; k < count; ++k) {
    double x = 10.0 / std::pow(rng.uniform_pos(), 1.0 / 1.5);
    int32_t m = static_cast<int32_t>(std::min<double>(std::floor(x), clip));
    if (m < 1) m = 1;
    if (used + m > budget) break;
    out.push_back(m);
    used += m;
  }
  return out;
}

void gen_circuit_family(bdlu_synth& s, Rng& rng, int32_t n, int32_t npareto, int32_t nbus) {
  s.n = n;
  std::vector<int32_t> sizes = pareto_sizes(rng, npareto, 20000, static_cast<int64_t>(n) * 9 / 10);
  int64_t used = 0;
  for (int32_t m : sizes) used += m;
  for (int64_t k = used; k < n; ++k) sizes.push_back(1);
  for (size_t i = sizes.size() - 1; i > 0; --i) std::swap(sizes[i], sizes[static_cast<size_t>(rng.below(static_cast<int64_t>(i) + 1))]);
  s.block_sizes = sizes;
  const size_t nb = sizes.size();
  std::vector<int32_t> off(nb + 1, 0);
  for (size_t b = 0; b < nb; ++b) off[b + 1] = off[b] + sizes[b];
  std::vector<std::vector<RowEntry>> rows(static_cast<size_t>(n));
  auto couple = [&](std::vector<RowEntry>& r, size_t b) {
    if (b + 1 >= nb) return;
    const int32_t lo = off[b + 1];
    r.push_back(RowEntry{lo + static_cast<int32_t>(rng.below(n - lo)), loguniform_signed(rng)});
  };
  for (size_t b = 0; b < nb; ++b) {
    const int32_t m = sizes[b], o = off[b];
    for (int32_t i = 0; i < m; ++i) {
      auto& r = rows[static_cast<size_t>(o + i)];
      if (m > 1) {
        r.push_back(RowEntry{o + (i + 1) % m, loguniform_signed(rng)});
        for (int t = 0; t < 3; ++t) {
          const int32_t c = static_cast<int32_t>(rng.below(m));
          const double v = loguniform_signed(rng);
          if (c != i) r.push_back(RowEntry{o + c, v});
        }
        couple(r, b);
      } else {
        for (int t = 0; t < 5; ++t) couple(r, b);
      }
    }
  }
  // Bus rows in the first 10% of blocks, bus columns in the last 10%.
  const size_t early = std::max<size_t>(1, nb / 10);
  const size_t late0 = nb - std::max<size_t>(1, nb / 10);
  for (int32_t k = 0; k < nbus; ++k) {
    const size_t b = static_cast<size_t>(rng.below(static_cast<int64_t>(early)));
    const int32_t r = off[b] + static_cast<int32_t>(rng.below(sizes[b]));
    const int32_t lo = off[b + 1];
    if (lo >= n) continue;
    for (int t = 0; t < 500; ++t)
      rows[static_cast<size_t>(r)].push_back(RowEntry{lo + static_cast<int32_t>(rng.below(n - lo)), loguniform_signed(rng)});
  }
  for (int32_t k = 0; k < nbus; ++k) {
    const size_t b = late0 + static_cast<size_t>(rng.below(static_cast<int64_t>(nb - late0)));
    const int32_t c = off[b] + static_cast<int32_t>(rng.below(sizes[b]));
    const int32_t hi = off[b];
    if (hi <= 0) continue;
    for (int t = 0; t < 500; ++t)
      rows[static_cast<size_t>(rng.below(hi))].push_back(RowEntry{c, loguniform_signed(rng)});
  }
  finish(s, rows, rng, nullptr);
}

void gen_precision_family(bdlu_synth& s, Rng& rng, int32_t nbig, int32_t lo, int32_t hi, double kappa) {
  std::vector<int32_t> big(static_cast<size_t>(nbig));
  int64_t nb_rows = 0;
  for (auto& m : big) {
    m = lo + static_cast<int32_t>(rng.below(hi - lo + 1));
    nb_rows += m;
  }
  std::vector<int32_t> small = pareto_sizes(rng, 1 << 30, 2000, nb_rows / 9);
  std::vector<int32_t> sizes = big;
  sizes.insert(sizes.end(), small.begin(), small.end());
  for (size_t i = sizes.size() - 1; i > 0; --i) std::swap(sizes[i], sizes[static_cast<size_t>(rng.below(static_cast<int64_t>(i) + 1))]);
  int64_t n64 = 0;
  for (int32_t m : sizes) n64 += m;
  s.n = static_cast<int32_t>(n64);
  s.block_sizes = sizes;
  const int32_t n = s.n;
  const size_t nb = sizes.size();
  std::vector<int32_t> off(nb + 1, 0);
  for (size_t b = 0; b < nb; ++b) off[b + 1] = off[b] + sizes[b];
  std::vector<std::vector<RowEntry>> rows(static_cast<size_t>(n));
  std::vector<double> scale(static_cast<size_t>(n), 1.0);
  for (size_t b = 0; b < nb; ++b) {
    const int32_t m = sizes[b], o = off[b];
    const bool large = m >= lo;
    const int intra = large ? 18 : 3;
    for (int32_t i = 0; i < m; ++i) {
      auto& r = rows[static_cast<size_t>(o + i)];
      if (m > 1) {
        r.push_back(RowEntry{o + (i + 1) % m, rng.normal()});
        for (int t = 0; t < intra; ++t) {
          const int32_t c = static_cast<int32_t>(rng.below(m));
          const double v = rng.normal();
          if (c != i) r.push_back(RowEntry{o + c, v});
        }
      }
      if (b + 1 < nb) {
        const int32_t l2 = off[b + 1];
        r.push_back(RowEntry{l2 + static_cast<int32_t>(rng.below(n - l2)), 0.1 * rng.normal()});
      }
      // Geometric row ramp over the block: rows are scaled down by up to
      // 1/kappa, which raises the block condition number towards kappa.
      if (large && kappa > 1.0) {
        const double t = (m > 1) ? static_cast<double>(i) / static_cast<double>(m - 1) : 0.0;
        const double f = std::pow(kappa, -t);
        for (auto& e : r) e.val *= f;
        scale[static_cast<size_t>(o + i)] = f;
      }
    }
  }
  finish(s, rows, rng, &scale);
}

}  // namespace

extern "C" {

bdlu_synth* bdlu_synth_create(int32_t family, uint64_t seed, int32_t n, int32_t param, int32_t nrhs) {
  auto* s = new bdlu_synth();
  s->seed = seed;
  s->nrhs = nrhs > 0 ? nrhs : 1;
  Rng rng(seed);
  switch (family) {
    case BDLU_SYNTH_BLOCK:
      gen_block_family(*s, rng, n, param > 0 ? param : std::max<int32_t>(1, n / 50));
      break;
    case BDLU_SYNTH_CIRCUIT:
      gen_circuit_family(*s, rng, n, param > 0 ? param : std::max<int32_t>(1, static_cast<int32_t>(1000LL * n / 200000)), 50);
      break;
    case BDLU_SYNTH_PRECISION: {
      // n: number of large blocks; param: kappa exponent (4 or 8).
      const double kappa = std::pow(10.0, param > 0 ? param : 4);
      gen_precision_family(*s, rng, n > 0 ? n : 200, 2000, 8000, kappa);
      break;
    }
    default:
      delete s;
      return nullptr;
  }
  return s;
}

void bdlu_synth_destroy(bdlu_synth* s) { delete s; }
int32_t bdlu_synth_n(const bdlu_synth* s) { return s ? s->n : 0; }
int64_t bdlu_synth_nnz(const bdlu_synth* s) { return s ? static_cast<int64_t>(s->row.size()) : 0; }
int32_t bdlu_synth_nrhs(const bdlu_synth* s) { return s ? s->nrhs : 0; }
int32_t bdlu_synth_nblocks(const bdlu_synth* s) { return s ? static_cast<int32_t>(s->block_sizes.size()) : 0; }

void bdlu_synth_copy(const bdlu_synth* s, int32_t* rows, int32_t* cols, double* vals, double* x_true,
                     double* b) {
  if (!s) return;
  if (rows) std::memcpy(rows, s->row.data(), s->row.size() * sizeof(int32_t));
  if (cols) std::memcpy(cols, s->col.data(), s->col.size() * sizeof(int32_t));
  if (vals) std::memcpy(vals, s->val.data(), s->val.size() * sizeof(double));
  if (x_true) std::memcpy(x_true, s->x_true.data(), s->x_true.size() * sizeof(double));
  if (b) std::memcpy(b, s->b.data(), s->b.size() * sizeof(double));
}

void bdlu_synth_block_sizes(const bdlu_synth* s, int32_t* sizes) {
  if (s && sizes) std::memcpy(sizes, s->block_sizes.data(), s->block_sizes.size() * sizeof(int32_t));
}

void bdlu_synth_perturb(const bdlu_synth* s, uint64_t seed, double* vals_out) {
  // values x (1 + U(-0.1, 0.1)), one draw per stored entry.
  if (!s || !vals_out) return;
  Rng rng(seed);
  for (size_t k = 0; k < s->val.size(); ++k) vals_out[k] = s->val[k] * (1.0 + 0.2 * rng.uniform() - 0.1);
}

}  // extern "C"
