// Autotuner: launch-shape and schedule choices measured on the device the
// engine runs on, kept per process and in a per-GPU cache file.
//
// Choices (every candidate computes bit-identical results, so a choice only
// changes the time):
//   * CTA width of the shared-memory LU (k_lu_small) per size bucket: 64,
//     128 or 256 threads, timed on the bucket's own units at the first
//     factor that meets the bucket on this GPU;
//   * per pattern signature, the small units as per-bucket launches or as one
//     persistent launch over a task queue, timed at the pattern's first factor;
//   * schedule of a pattern's value-only refactor of large units: the step
//     chain or the tile task graph, timed on the pattern's first two
//     refactors and keyed by its pattern signature.
// The reference tunes these by hand through environment knobs
// (blockdaglu/src/ubtf_block_solver.cpp:35-568).
//
// Cache file: $BDLU_TUNE_CACHE if set, else $HOME/.cache/bdlu/tune-<gpu>.json;
// BDLU_AUTOTUNE=0 turns tuning off (fixed defaults).
#pragma once

#include <cstdint>
#include <string>

namespace bdlu {

class Tuner {
 public:
  static Tuner& get();
  bool enabled() const { return enabled_; }
  // Launch width chosen for buckets of units up to `bucket_m` rows (1: one
  // thread per row, 32: one warp per unit, else threads per CTA); 0 if none.
  int lu_small_threads(int32_t bucket_m);
  void set_lu_small_threads(int32_t bucket_m, int threads, const float* ms, const int* widths, int count);
  // Small-unit launch mode for pattern `sig`: 0 per-bucket launches, 1 one
  // persistent launch; -1 if none yet.
  int small_mode(uint64_t sig);
  void set_small_mode(uint64_t sig, int mode, float ms_buckets, float ms_queue);
  // Refactor schedule chosen for pattern `sig`: 0 / 1, or -1 if none yet.
  int refactor_schedule(uint64_t sig);
  void set_refactor_schedule(uint64_t sig, int schedule, float ms_chain, float ms_graph);
  // JSON of the device key and every choice with its timings.
  std::string report();

 private:
  Tuner();
  void load();
  bool enabled_ = true;
  std::string path_;
  std::string device_;
};

}  // namespace bdlu
