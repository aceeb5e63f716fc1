// Autotuner cache (tuner.h): per-process choices, persisted per GPU as JSON.
#include "tuner.h"

#include <cuda_runtime_api.h>
#include <sys/stat.h>

#include <cctype>
#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

namespace bdlu {

namespace {

struct SmallChoice {
  int threads = 0;
  std::vector<int> widths;
  std::vector<float> ms;
};

struct ScheduleChoice {
  int schedule = -1;
  float ms_chain = 0.0f, ms_graph = 0.0f;
};

std::mutex g_mu;
std::map<int32_t, SmallChoice> g_small;
std::map<uint64_t, ScheduleChoice> g_sched;
std::map<uint64_t, ScheduleChoice> g_mode;  // small-unit launch mode (0 buckets, 1 queue) and both times

std::string sanitize(const std::string& s) {
  std::string out;
  for (char c : s) out += (std::isalnum(static_cast<unsigned char>(c)) || c == '-' || c == '_') ? c : '_';
  return out;
}

void make_dirs(const std::string& path) {
  for (size_t i = 1; i < path.size(); ++i)
    if (path[i] == '/') {
      const std::string d = path.substr(0, i);
      if (mkdir(d.c_str(), 0755) != 0 && errno != EEXIST) return;
    }
}

}  // namespace

Tuner& Tuner::get() {
  static Tuner t;
  return t;
}

Tuner::Tuner() {
  if (const char* e = std::getenv("BDLU_AUTOTUNE")) enabled_ = std::strcmp(e, "0") != 0;
  int dev = 0, sms = 0;
  cudaDeviceProp prop{};
  std::string name = "no-device";
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    name = prop.name;
    sms = prop.multiProcessorCount;
  }
  device_ = name + " sm" + std::to_string(prop.major) + std::to_string(prop.minor) + " x" + std::to_string(sms);
  if (const char* p = std::getenv("BDLU_TUNE_CACHE")) {
    path_ = p;
  } else if (const char* h = std::getenv("HOME")) {
    path_ = std::string(h) + "/.cache/bdlu/tune-" + sanitize(device_) + ".json";
  }
  load();
}

void Tuner::load() {
  if (path_.empty()) return;
  std::ifstream f(path_);
  if (!f) return;
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string t = ss.str();
  // The file is one this class wrote; entries are read by their keys.
  if (t.find("\"device\": \"" + device_ + "\"") == std::string::npos) return;
  std::lock_guard<std::mutex> lk(g_mu);
  for (size_t p = t.find("\"bucket_m\":"); p != std::string::npos; p = t.find("\"bucket_m\":", p + 1)) {
    int m = 0, th = 0;
    if (std::sscanf(t.c_str() + p, "\"bucket_m\": %d, \"threads\": %d", &m, &th) == 2 && m > 0 &&
        (th == 1 || th == 32 || th == 64 || th == 128 || th == 256))
      g_small[m].threads = th;
  }
  for (size_t p = t.find("\"mode_sig\":"); p != std::string::npos; p = t.find("\"mode_sig\":", p + 1)) {
    unsigned long long sig = 0;
    int mode = -1;
    float a = 0.0f, b = 0.0f;
    if (std::sscanf(t.c_str() + p, "\"mode_sig\": \"%llx\", \"mode\": %d, \"ms_buckets\": %f, \"ms_queue\": %f",
                    &sig, &mode, &a, &b) >= 2 &&
        (mode == 0 || mode == 1)) {
      ScheduleChoice& c = g_mode[static_cast<uint64_t>(sig)];
      c.schedule = mode;
      c.ms_chain = a;
      c.ms_graph = b;
    }
  }
  for (size_t p = t.find("\"sig\":"); p != std::string::npos; p = t.find("\"sig\":", p + 1)) {
    unsigned long long sig = 0;
    int sch = -1;
    float a = 0.0f, b = 0.0f;
    if (std::sscanf(t.c_str() + p, "\"sig\": \"%llx\", \"schedule\": %d, \"ms_chain\": %f, \"ms_graph\": %f", &sig, &sch,
                    &a, &b) >= 2 &&
        (sch == 0 || sch == 1)) {
      ScheduleChoice& c = g_sched[static_cast<uint64_t>(sig)];
      c.schedule = sch;
      c.ms_chain = a;
      c.ms_graph = b;
    }
  }
}

std::string Tuner::report() {
  std::lock_guard<std::mutex> lk(g_mu);
  std::ostringstream o;
  o << "{\"device\": \"" << device_ << "\", \"enabled\": " << (enabled_ ? "true" : "false") << ", \"cache\": \""
    << path_ << "\",\n \"lu_small_threads\": [";
  bool first = true;
  for (const auto& kv : g_small) {
    o << (first ? "\n  " : ",\n  ") << "{\"bucket_m\": " << kv.first << ", \"threads\": " << kv.second.threads;
    if (!kv.second.widths.empty()) {
      o << ", \"widths\": [";
      for (size_t i = 0; i < kv.second.widths.size(); ++i) o << (i ? ", " : "") << kv.second.widths[i];
      o << "], \"ms\": [";
      for (size_t i = 0; i < kv.second.ms.size(); ++i) o << (i ? ", " : "") << kv.second.ms[i];
      o << "]";
    }
    o << "}";
    first = false;
  }
  o << "],\n \"refactor_schedule\": [";
  first = true;
  for (const auto& kv : g_sched) {
    char sig[32];
    std::snprintf(sig, sizeof(sig), "%016" PRIx64, kv.first);
    o << (first ? "\n  " : ",\n  ") << "{\"sig\": \"" << sig << "\", \"schedule\": " << kv.second.schedule
      << ", \"ms_chain\": " << kv.second.ms_chain << ", \"ms_graph\": " << kv.second.ms_graph << "}";
    first = false;
  }
  o << "],\n \"small_mode\": [";
  first = true;
  for (const auto& kv : g_mode) {
    char sig[32];
    std::snprintf(sig, sizeof(sig), "%016" PRIx64, kv.first);
    o << (first ? "\n  " : ",\n  ") << "{\"mode_sig\": \"" << sig << "\", \"mode\": " << kv.second.schedule
      << ", \"ms_buckets\": " << kv.second.ms_chain << ", \"ms_queue\": " << kv.second.ms_graph << "}";
    first = false;
  }
  o << "]}\n";
  return o.str();
}

int Tuner::lu_small_threads(int32_t bucket_m) {
  std::lock_guard<std::mutex> lk(g_mu);
  const auto it = g_small.find(bucket_m);
  return it == g_small.end() ? 0 : it->second.threads;
}

static void write_file(const std::string& path, const std::string& text) {
  if (path.empty()) return;
  make_dirs(path);
  const std::string tmp = path + ".tmp" + std::to_string(static_cast<long long>(reinterpret_cast<uintptr_t>(&text)));
  {
    std::ofstream f(tmp);
    if (!f) return;
    f << text;
  }
  std::rename(tmp.c_str(), path.c_str());
}

void Tuner::set_lu_small_threads(int32_t bucket_m, int threads, const float* ms, const int* widths, int count) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    SmallChoice& c = g_small[bucket_m];
    c.threads = threads;
    c.widths.assign(widths, widths + count);
    c.ms.assign(ms, ms + count);
  }
  write_file(path_, report());
}

int Tuner::small_mode(uint64_t sig) {
  std::lock_guard<std::mutex> lk(g_mu);
  const auto it = g_mode.find(sig);
  return it == g_mode.end() ? -1 : it->second.schedule;
}

void Tuner::set_small_mode(uint64_t sig, int mode, float ms_buckets, float ms_queue) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ScheduleChoice& c = g_mode[sig];
    c.schedule = mode;
    c.ms_chain = ms_buckets;
    c.ms_graph = ms_queue;
  }
  write_file(path_, report());
}

int Tuner::refactor_schedule(uint64_t sig) {
  std::lock_guard<std::mutex> lk(g_mu);
  const auto it = g_sched.find(sig);
  return it == g_sched.end() ? -1 : it->second.schedule;
}

void Tuner::set_refactor_schedule(uint64_t sig, int schedule, float ms_chain, float ms_graph) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ScheduleChoice& c = g_sched[sig];
    c.schedule = schedule;
    c.ms_chain = ms_chain;
    c.ms_graph = ms_graph;
  }
  write_file(path_, report());
}

}  // namespace bdlu
