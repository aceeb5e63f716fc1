// Device helpers shared by the engine's kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace bdlu {

constexpr int kFailZeroPivot = 1;
constexpr int kFailReusedPivot = 2;  // a reused pivot order met a zero pivot
constexpr int kFailSync = 3;         // a bounded wait of the solve ran out
constexpr int kFailRefactorSync = 4; // a bounded wait of the tile-graph refactor ran out
constexpr int kFailSparseReject = 6; // a sparse-LU unit failed the pivot test (gp.h): factor it dense
constexpr int kFailSparseSync = 7;   // a bounded wait between sparse-LU columns ran out

__device__ __forceinline__ void report_failure(int32_t* status, int32_t unit) {
  if (atomicCAS(status, 0, kFailZeroPivot) == 0) status[1] = unit;
}

// (value, index) maximum with the reference's tie rule: the smallest index
// among equal maxima, i.e. the first strict maximum of an ascending scan
// (ubtf_block_solver.cpp:1460-1468).  `none` marks an empty candidate.
__device__ __forceinline__ void pivot_combine(double& best, int& bi, double ob, int oi, int none) {
  if (oi == none) return;
  if (bi == none || ob > best || (ob == best && oi < bi)) {
    best = ob;
    bi = oi;
  }
}

__device__ __forceinline__ void warp_pivot_reduce(double& best, int& bi, int none) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
    pivot_combine(best, bi, ob, oi, none);
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

}  // namespace bdlu
