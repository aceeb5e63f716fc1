// Checks the task list of the tile-graph refactor (bdlu::build_rtasks) on the
// CPU, independently of the kernel: replaying the list in ticket order, every
// task finds its input tiles at exactly the versions the kernel waits for,
// every tile receives each step's update once and in step order, and every
// tile ends at version min(i, j) + 1.  In-order replay succeeding means that
// each task depends only on tasks with smaller tickets, which is what keeps
// the persistent kernel free of deadlock.  Prints "ok" on success.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "plan.h"

namespace {

int fail(const char* what, long a, long b) {
  std::printf("FAIL: %s (%ld, %ld)\n", what, a, b);
  return 1;
}

// plant > 0 moves the diagonal task of step 1 of the first unit to just
// after step 0's diagonal task, before its inputs: the replay must reject it.
int check(const std::vector<int32_t>& sizes, int plant = 0) {
  std::vector<int32_t> units;
  for (size_t q = 0; q < sizes.size(); ++q) units.push_back(static_cast<int32_t>(1000 + 7 * q));
  std::vector<int32_t> tasks;
  int32_t words = 0;
  const int64_t n = bdlu::build_rtasks(units, sizes, int64_t{1} << 30, tasks, words);
  if (plant > 0) {
    for (int64_t t = 1; t < n; ++t) {
      const int32_t* e = tasks.data() + 4 * t;
      if (e[0] == units[0] && e[1] == 1 && e[2] == ((1 << 16) | 1)) {
        std::vector<int32_t> d(e, e + 4);
        tasks.erase(tasks.begin() + 4 * t, tasks.begin() + 4 * t + 4);
        tasks.insert(tasks.begin() + 4, d.begin(), d.end());
        break;
      }
    }
  }
  std::vector<int64_t> nt(sizes.size()), base(sizes.size());
  int64_t expect = 0, w = 1;
  for (size_t q = 0; q < sizes.size(); ++q) {
    nt[q] = (sizes[q] + bdlu::kRPanel - 1) / bdlu::kRPanel;
    base[q] = w;
    w += nt[q] * nt[q];
    for (int64_t k = 0; k < nt[q]; ++k) {
      const int64_t r = nt[q] - k - 1;
      expect += 1 + 2 * r + (r + 1) / 2 * r;
    }
  }
  if (n != expect || static_cast<int64_t>(tasks.size()) != 4 * expect) return fail("task count", n, expect);
  if (words != w) return fail("version words", words, w);
  std::vector<std::vector<int32_t>> ver(sizes.size());
  for (size_t q = 0; q < sizes.size(); ++q) ver[q].assign(static_cast<size_t>(nt[q] * nt[q]), 0);
  for (int64_t t = 0; t < n; ++t) {
    const int32_t* e = tasks.data() + 4 * t;
    size_t q = 0;
    while (q < units.size() && units[q] != e[0]) ++q;
    if (q == units.size()) return fail("unknown unit", t, e[0]);
    if (e[3] != base[q]) return fail("version base", t, e[3]);
    const int64_t k = e[1], i = e[2] >> 16, j = e[2] & 0xffff, m = nt[q];
    auto v = [&](int64_t a, int64_t b) -> int32_t& { return ver[q][static_cast<size_t>(a * m + b)]; };
    if (k < 0 || k >= m || i < k || j < k || i >= m || j >= m) return fail("task out of range", t, k);
    if (i == k && j == k) {
      if (v(k, k) != k) return fail("D input", t, k);
      v(k, k) = static_cast<int32_t>(k + 1);
    } else if (j == k) {
      if (v(k, k) != k + 1 || v(i, k) != k) return fail("L input", t, i);
      v(i, k) = static_cast<int32_t>(k + 1);
    } else if (i == k) {
      if (v(k, k) != k + 1 || v(k, j) != k) return fail("U input", t, j);
      v(k, j) = static_cast<int32_t>(k + 1);
    } else {
      if ((i - k - 1) % 2 != 0) return fail("row pair alignment", t, i);
      if (v(i, k) != k + 1 || v(k, j) != k + 1 || v(i, j) != k) return fail("G input", t, i * m + j);
      v(i, j) = static_cast<int32_t>(k + 1);
      if (i + 1 < m) {
        if (v(i + 1, k) != k + 1 || v(i + 1, j) != k) return fail("G input (second row tile)", t, i * m + j);
        v(i + 1, j) = static_cast<int32_t>(k + 1);
      }
    }
  }
  for (size_t q = 0; q < sizes.size(); ++q)
    for (int64_t i = 0; i < nt[q]; ++i)
      for (int64_t j = 0; j < nt[q]; ++j)
        if (ver[q][static_cast<size_t>(i * nt[q] + j)] != (i < j ? i : j) + 1) return fail("final version", i, j);
  return 0;
}

}  // namespace

int main() {
  const std::vector<std::vector<int32_t>> cases = {
      {170}, {192}, {193}, {4233}, {320, 171}, {4233, 1000, 200, 170, 640, 641}, {64 * 9 + 1, 64 * 10}};
  for (const auto& c : cases)
    if (check(c)) return 1;
  std::printf("planted misorder: ");
  if (check({320}, 1) == 0) {
    std::printf("not detected\n");
    return 1;
  }
  // The size cap empties the list.
  std::vector<int32_t> tasks;
  int32_t words = 0;
  if (bdlu::build_rtasks({1}, {4233}, 1000, tasks, words) != -1 || !tasks.empty())
    return fail("task cap", static_cast<long>(tasks.size()), 0);
  std::printf("ok\n");
  return 0;
}
