// Serving loop (bdlu_server_*, include/bdlu.h): value-only refactor + solve
// requests over resident patterns, with continuous batching.
//
// The reference serves one system at a time per Solver; a caller with many
// patterns and a stream of requests keeps a Solver per pattern and calls
// refactor + solve for each request in turn.  Here every pattern keeps its
// analysis on the host and its plan, factors and work space on the device
// (one engine per pattern).  `slots` worker threads each own a CUDA stream;
// a free worker takes the oldest queued request whose pattern is not being
// served, so requests for different patterns run side by side on the device
// (their kernels overlap), and requests for one pattern run in arrival order.
// Patterns are admitted under a device-memory budget: before a pattern is
// uploaded, idle resident patterns are released least recently used first
// until the estimate fits; a pattern that cannot fit even alone fails its
// request.  Latency is taken from submission to the result being in the
// caller's buffer.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bdlu.h"
#include "capi_internal.h"
#include "plan.h"

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Pattern {
  bdlu_solver* h = nullptr;
  int32_t n = 0;
  int64_t nnz = 0;     // canonical entries (values per request)
  bool resident = false;
  bool busy = false;
  int64_t bytes = 0;   // device bytes when resident (measured), else the estimate
  uint64_t last_use = 0;
};

struct Request {
  int64_t id = 0;
  int32_t pattern = 0;
  const double* vals = nullptr;
  double* B = nullptr;
  int32_t ldb = 0, nrhs = 0;
  bool device = false;  // vals and B are device pointers (device-resident request)
  double t_submit = 0.0, t_done = 0.0;
  int status = BDLU_OK;
  double residual = 0.0;
  std::string message;
  bool done = false;
};

}  // namespace

struct bdlu_server {
  int64_t budget = 0;
  std::vector<std::unique_ptr<Pattern>> patterns;
  std::deque<Request*> queue;
  std::unordered_map<int64_t, std::unique_ptr<Request>> requests;
  int64_t next_id = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::thread> workers;
  bool stop = false;
  int64_t resident_bytes = 0;
  int64_t evictions = 0;
  int32_t running = 0, peak_running = 0;
  uint64_t tick = 0;
  std::vector<double> latencies;
  double t_first = -1.0, t_last = 0.0;
  int64_t completed = 0, failed = 0;
  int64_t kernel_launches = 0;
  double factor_flops = 0.0;
  double stage_ms = 0.0, factor_ms = 0.0, solve_ms = 0.0;  // worker wall time per phase, summed
  std::string last_message;
  int last_error = BDLU_OK;
  double precision = 0.0;  // "precision" option of every pattern's handle
  int64_t max_nnz = 0;     // largest pattern: sizes the workers' page-locked staging once
  int32_t max_n = 0;
};

namespace {

// Device bytes of a pattern before its first upload: LU arena, values,
// coupling and unit tables, 16 right-hand sides of work space.
int64_t estimate_bytes(const bdlu::Plan& p) {
  const int64_t n = p.n;
  return 8 * p.lu_size + 16 * p.nnz + 16 * static_cast<int64_t>(p.cpl_col.size()) + 64 * n + 4 * 8 * n * 16 +
         (16 << 20);
}

// Picks a request to run (lock held): the oldest queued request whose pattern
// is idle and fits the budget after releasing idle patterns.  Returns nullptr
// if none can start now.  Fails requests whose pattern cannot fit at all.
Request* pick(bdlu_server* s) {
  for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
    Request* r = *it;
    Pattern& p = *s->patterns[static_cast<size_t>(r->pattern)];
    if (p.busy) continue;
    if (!p.resident) {
      if (p.bytes > s->budget) {
        r->status = BDLU_BACKEND_UNAVAILABLE;
        r->message = "pattern needs " + std::to_string(p.bytes) + " device bytes, above the server budget";
        r->done = true;
        r->t_done = now_ms();
        ++s->failed;
        s->queue.erase(it);
        s->cv_done.notify_all();
        return pick(s);
      }
      // Release idle resident patterns, least recently used first.
      while (s->resident_bytes + p.bytes > s->budget) {
        Pattern* victim = nullptr;
        for (auto& q : s->patterns)
          if (q->resident && !q->busy && (!victim || q->last_use < victim->last_use)) victim = q.get();
        if (!victim) break;
        bdlu_device_release(victim->h);
        victim->resident = false;
        s->resident_bytes -= victim->bytes;
        ++s->evictions;
      }
      if (s->resident_bytes + p.bytes > s->budget) continue;  // wait for a busy pattern to finish
      p.resident = true;                                        // reserved; uploaded by the worker
      s->resident_bytes += p.bytes;
    }
    p.busy = true;
    p.last_use = ++s->tick;
    s->queue.erase(it);
    return r;
  }
  return nullptr;
}

// Page-locked host staging of one worker (copies from pageable memory are
// staged by the driver and do not overlap with other streams' work).
struct Staging {
  double* buf = nullptr;
  size_t cap = 0;  // doubles
  // `hint`: the size the largest pattern needs, allocated at once so the
  // buffer is not regrown request after request (cudaMallocHost and
  // cudaFreeHost are slow and cudaFreeHost synchronises the device).
  double* get(size_t count, size_t hint) {
    if (count <= cap) return buf;
    if (buf) cudaFreeHost(buf);
    buf = nullptr;
    cap = 0;
    const size_t want = std::max(count, hint);
    if (cudaMallocHost(reinterpret_cast<void**>(&buf), want * sizeof(double)) != cudaSuccess) return nullptr;
    cap = want;
    return buf;
  }
  ~Staging() {
    if (buf) cudaFreeHost(buf);
  }
};

void worker(bdlu_server* s) {
  cudaStream_t stream = nullptr;
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  Staging vstage, bstage;
  while (true) {
    Request* r = nullptr;
    Pattern* pp = nullptr;
    size_t hint_v = 0, hint_b = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || (r = pick(s)) != nullptr; });
      if (!r) break;
      s->peak_running = std::max(s->peak_running, ++s->running);
      pp = s->patterns[static_cast<size_t>(r->pattern)].get();
      hint_v = static_cast<size_t>(s->max_nnz);
      hint_b = static_cast<size_t>(s->max_n) * 16;
    }
    Pattern& p = *pp;
    int st = BDLU_OK;
    const double t_start = now_ms();
    double t_staged = t_start, t_factored = t_start;
    const int64_t reserved = p.bytes;
    if (!bdlu_engine_ready(p.h)) st = bdlu_device_restore(p.h);
    if (r->device) {
      // Device-resident request: values and right-hand sides never leave HBM.
      t_staged = now_ms();
      if (st == BDLU_OK) st = bdlu_refactor_values_device_on(p.h, r->vals, p.nnz, stream);
      t_factored = now_ms();
      if (st == BDLU_OK) st = bdlu_solve_checked_on(p.h, r->B, r->ldb, r->nrhs, stream, true);
    } else {
      const size_t nb = static_cast<size_t>(p.n) * static_cast<size_t>(r->nrhs);
      double* sv = vstage.get(static_cast<size_t>(p.nnz), hint_v);
      double* sb = bstage.get(nb, hint_b);
      if (st == BDLU_OK && (!sv || !sb)) st = -1;
      // One pass per input: the copy into page-locked staging checks for
      // NaN and infinity on the way; the checks fail the request where
      // bdlu_refactor_solve's would (values before the refactor, right-hand
      // sides after it).
      bool finite_b = true;
      if (st == BDLU_OK) {
        if (!bdlu_copy_finite(sv, r->vals, p.nnz))
          st = bdlu_fail(p.h, BDLU_NON_FINITE_VALUE, "matrix contains NaN or infinity");
        for (int32_t k = 0; k < r->nrhs && st == BDLU_OK; ++k)
          finite_b &= bdlu_copy_finite(sb + static_cast<size_t>(k) * p.n, r->B + static_cast<size_t>(k) * r->ldb, p.n);
        t_staged = now_ms();
        if (st == BDLU_OK) st = bdlu_refactor_values_on(p.h, sv, p.nnz, stream, true);
      }
      t_factored = now_ms();
      if (st == BDLU_OK && !finite_b)
        st = bdlu_fail(p.h, BDLU_NON_FINITE_VALUE, "right-hand side contains NaN or infinity");
      if (st == BDLU_OK) st = bdlu_solve_checked_on(p.h, sb, p.n, r->nrhs, stream, false, true);
      if (st == BDLU_OK)
        for (int32_t k = 0; k < r->nrhs; ++k)
          std::copy(sb + static_cast<size_t>(k) * p.n, sb + static_cast<size_t>(k + 1) * p.n,
                    r->B + static_cast<size_t>(k) * r->ldb);
    }
    char buf[512] = "host staging allocation failed";
    if (st > 0) bdlu_last_error(p.h, buf, sizeof(buf));
    if (st < 0) st = BDLU_BACKEND_UNAVAILABLE;
    bdlu_stats stats{};
    bdlu_get_stats(p.h, &stats);
    const int64_t actual = bdlu_device_bytes(p.h);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (actual > 0) {
        s->resident_bytes += actual - reserved;
        p.bytes = actual;
      } else {
        // The upload failed: give the reservation back.
        s->resident_bytes -= reserved;
        p.resident = false;
      }
      p.busy = false;
      p.last_use = ++s->tick;
      r->status = st;
      r->residual = stats.residual_inf;
      if (st != BDLU_OK) r->message = buf;
      r->t_done = now_ms();
      r->done = true;
      --s->running;
      s->kernel_launches += static_cast<int64_t>(stats.factor_launches) + stats.solve_launches;
      s->stage_ms += t_staged - t_start;
      s->factor_ms += t_factored - t_staged;
      s->solve_ms += now_ms() - t_factored;
      if (st == BDLU_OK) {
        s->factor_flops += stats.factor_flops;
        ++s->completed;
        s->latencies.push_back(r->t_done - r->t_submit);
        s->t_last = std::max(s->t_last, r->t_done);
      } else {
        ++s->failed;
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
  cudaStreamDestroy(stream);
}

int sfail(bdlu_server* s, int code, std::string msg) {
  s->last_error = code;
  s->last_message = std::move(msg);
  return code;
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * static_cast<double>(v.size() - 1);
  const size_t lo = static_cast<size_t>(pos);
  const size_t hi = std::min(v.size() - 1, lo + 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - static_cast<double>(lo));
}

}  // namespace

extern "C" {

bdlu_server* bdlu_server_create(int64_t memory_budget_bytes, int32_t slots) {
  if (memory_budget_bytes <= 0 || slots <= 0) return nullptr;
  try {
    auto* s = new bdlu_server();
    s->budget = memory_budget_bytes;
    for (int32_t i = 0; i < slots; ++i) s->workers.emplace_back(worker, s);
    return s;
  } catch (...) {
    return nullptr;
  }
}

void bdlu_server_destroy(bdlu_server* s) {
  if (!s) return;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->queue.empty() && s->running == 0; });
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& p : s->patterns) bdlu_destroy(p->h);
  delete s;
}

int32_t bdlu_server_add_pattern(bdlu_server* s, const int32_t* rows, const int32_t* cols, const double* vals,
                                int64_t nnz, int32_t n) {
  if (!s) return -BDLU_NOT_PREPARED;
  auto p = std::make_unique<Pattern>();
  p->h = bdlu_create();
  if (!p->h) return -sfail(s, BDLU_BACKEND_UNAVAILABLE, "bdlu_create failed");
  int st = bdlu_set_coo(p->h, rows, cols, vals, nnz, n);
  // Host analysis only; the device upload happens when a request is admitted.
  if (st == BDLU_OK) st = bdlu_set_option(p->h, "analysis_only", 1);
  if (st == BDLU_OK) st = bdlu_analyze(p->h);
  if (st == BDLU_OK) st = bdlu_set_option(p->h, "analysis_only", 0);
  // The step chain for every served pattern: the tile task graph's
  // persistent kernel waits on its own tiles, and with other requests'
  // kernels on the GPU its CTAs lose the SMs they wait for (measured: tens of
  // milliseconds to seconds per refactor while the chain takes a few).
  if (st == BDLU_OK) st = bdlu_set_option(p->h, "refactor_schedule", 0);
  // Many workers wait for the device at once: they sleep on blocking-sync
  // events instead of each spinning a host core.
  if (st == BDLU_OK) st = bdlu_set_option(p->h, "blocking_sync", 1);
  // Plain stream order for the solve levels: with many request streams in
  // flight, a level launched ahead as a programmatic dependent holds SM
  // slots while it waits, which the other streams' ready work could use.
  if (st == BDLU_OK) st = bdlu_set_option(p->h, "programmatic_launch", 0);
  if (st == BDLU_OK) {
    std::lock_guard<std::mutex> lk(s->mu);
    st = bdlu_set_option(p->h, "precision", s->precision);
  }
  if (st != BDLU_OK) {
    char buf[512];
    bdlu_last_error(p->h, buf, sizeof(buf));
    bdlu_destroy(p->h);
    return -sfail(s, st, buf);
  }
  p->n = bdlu_n(p->h);
  p->nnz = bdlu_canonical_pattern(p->h, nullptr, nullptr);
  try {
    p->bytes = estimate_bytes(bdlu::build_plan(p->h->coo, p->h->dec, bdlu::small_unit_max()));
  } catch (const std::exception& e) {
    bdlu_destroy(p->h);
    return -sfail(s, BDLU_ANALYSIS_FAILED, e.what());
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->max_nnz = std::max(s->max_nnz, p->nnz);
  s->max_n = std::max(s->max_n, p->n);
  s->patterns.push_back(std::move(p));
  return static_cast<int32_t>(s->patterns.size()) - 1;
}

int64_t bdlu_server_pattern_nnz(bdlu_server* s, int32_t pattern) {
  if (!s) return -1;
  std::lock_guard<std::mutex> lk(s->mu);
  if (pattern < 0 || pattern >= static_cast<int32_t>(s->patterns.size())) return -1;
  return s->patterns[static_cast<size_t>(pattern)]->nnz;
}

int64_t bdlu_server_pattern_bytes(bdlu_server* s, int32_t pattern) {
  if (!s) return -1;
  std::lock_guard<std::mutex> lk(s->mu);
  if (pattern < 0 || pattern >= static_cast<int32_t>(s->patterns.size())) return -1;
  return s->patterns[static_cast<size_t>(pattern)]->bytes;
}

static int64_t submit_request(bdlu_server* s, int32_t pattern, const double* vals, int64_t nnz, double* B,
                              int32_t ldb, int32_t nrhs, bool device) {
  if (!s) return -BDLU_NOT_PREPARED;
  std::lock_guard<std::mutex> lk(s->mu);
  if (pattern < 0 || pattern >= static_cast<int32_t>(s->patterns.size()))
    return -sfail(s, BDLU_INVALID_INDEX, "unknown pattern");
  const Pattern& p = *s->patterns[static_cast<size_t>(pattern)];
  if (!vals || nnz != p.nnz) return -sfail(s, BDLU_INVALID_INDEX, "value count does not match the pattern");
  if (!B || nrhs < 1 || ldb < p.n) return -sfail(s, BDLU_INVALID_RHS, "right-hand side size does not match the pattern");
  auto r = std::make_unique<Request>();
  r->id = s->next_id++;
  r->pattern = pattern;
  r->vals = vals;
  r->B = B;
  r->ldb = ldb;
  r->nrhs = nrhs;
  r->device = device;
  r->t_submit = now_ms();
  if (s->t_first < 0.0) s->t_first = r->t_submit;
  s->queue.push_back(r.get());
  const int64_t id = r->id;
  s->requests.emplace(id, std::move(r));
  s->cv_work.notify_one();
  return id;
}

int64_t bdlu_server_submit(bdlu_server* s, int32_t pattern, const double* vals, int64_t nnz, double* B, int32_t ldb,
                           int32_t nrhs) {
  return submit_request(s, pattern, vals, nnz, B, ldb, nrhs, false);
}

int64_t bdlu_server_submit_device(bdlu_server* s, int32_t pattern, const double* d_vals, int64_t nnz, double* d_B,
                                  int32_t ldb, int32_t nrhs) {
  return submit_request(s, pattern, d_vals, nnz, d_B, ldb, nrhs, true);
}

int bdlu_server_wait(bdlu_server* s, int64_t request, double* residual, double* latency_ms) {
  if (!s) return BDLU_NOT_PREPARED;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(request);
  if (it == s->requests.end()) return sfail(s, BDLU_INVALID_INDEX, "unknown request");
  Request* r = it->second.get();
  s->cv_done.wait(lk, [&] { return r->done; });
  if (residual) *residual = r->residual;
  if (latency_ms) *latency_ms = r->t_done - r->t_submit;
  const int st = r->status;
  if (st != BDLU_OK) sfail(s, st, r->message);
  s->requests.erase(it);
  return st;
}

int bdlu_server_drain(bdlu_server* s) {
  if (!s) return BDLU_NOT_PREPARED;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->queue.empty() && s->running == 0; });
  return BDLU_OK;
}

int bdlu_server_get_stats(bdlu_server* s, bdlu_server_stats* out) {
  if (!s || !out) return BDLU_NOT_PREPARED;
  std::lock_guard<std::mutex> lk(s->mu);
  out->completed = s->completed;
  out->failed = s->failed;
  out->p50_ms = percentile(s->latencies, 0.50);
  out->p99_ms = percentile(s->latencies, 0.99);
  out->max_ms = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(), s->latencies.end());
  double sum = 0.0;
  for (double v : s->latencies) sum += v;
  out->mean_ms = s->latencies.empty() ? 0.0 : sum / static_cast<double>(s->latencies.size());
  const double span = s->t_last - s->t_first;
  out->throughput = span > 0.0 ? 1000.0 * static_cast<double>(s->completed) / span : 0.0;
  out->resident_bytes = s->resident_bytes;
  out->evictions = s->evictions;
  out->peak_concurrency = s->peak_running;
  out->kernel_launches = s->kernel_launches;
  out->factor_flops = s->factor_flops;
  const double done = static_cast<double>(std::max<int64_t>(1, s->completed + s->failed));
  out->mean_stage_ms = s->stage_ms / done;
  out->mean_factor_ms = s->factor_ms / done;
  out->mean_solve_ms = s->solve_ms / done;
  return BDLU_OK;
}

int bdlu_server_reset_stats(bdlu_server* s) {
  if (!s) return BDLU_NOT_PREPARED;
  std::lock_guard<std::mutex> lk(s->mu);
  s->latencies.clear();
  s->completed = s->failed = 0;
  s->kernel_launches = 0;
  s->factor_flops = 0.0;
  s->stage_ms = s->factor_ms = s->solve_ms = 0.0;
  s->t_first = -1.0;
  s->t_last = 0.0;
  s->peak_running = s->running;
  s->evictions = 0;
  return BDLU_OK;
}

int bdlu_server_set_option(bdlu_server* s, const char* key, double value) {
  if (!s || !key) return BDLU_NOT_PREPARED;
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->queue.empty() || s->running > 0) return sfail(s, BDLU_NOT_PREPARED, "requests are queued or running");
  const std::string k(key);
  if (k != "precision" || (value != 0.0 && value != 1.0 && value != 2.0))
    return sfail(s, BDLU_INVALID_DIMENSION, "unknown server option or value");
  for (auto& p : s->patterns)
    if (const int st = bdlu_set_option(p->h, "precision", value)) return sfail(s, st, "precision option refused");
  s->precision = value;
  return BDLU_OK;
}

int bdlu_server_last_error(const bdlu_server* s, char* buf, int64_t len) {
  if (!s) return BDLU_NOT_PREPARED;
  if (buf && len > 0) {
    const size_t m = std::min<size_t>(static_cast<size_t>(len - 1), s->last_message.size());
    std::copy(s->last_message.begin(), s->last_message.begin() + static_cast<std::ptrdiff_t>(m), buf);
    buf[m] = '\0';
  }
  return s->last_error;
}

}  // extern "C"
