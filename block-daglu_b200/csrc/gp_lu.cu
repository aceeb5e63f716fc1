// sm_100a kernels of the sparse-LU route (gp.h).  Both are dataflow kernels
// inside one CTA per sparse unit: the warps take columns (rows) round-robin
// in dependency order and wait, with a bounded poll, on per-column (per-row)
// flags in shared memory for exactly the columns (rows) they read, so a
// column's early updates overlap the columns it waits for and a warp's
// global loads for its next column are issued long before its inputs land.
// The smallest unfinished column (row) never waits on anything unfinished,
// so the CTA always progresses.
//   k_gp_factor  a warp forms column j in its shared-memory work vector (A's
//                entries, then x -= L(:,k) x[k] for each row k above the
//                diagonal in ascending order, read as coalesced runs of the
//                column-compressed L), applies the reference's pivot test
//                (gp_lu.cpp:164-218) and writes the column back (U, pivot,
//                L = x / pivot).  Updates are unfused (__dmul_rn, __dsub_rn):
//                each entry sees the multiply-subtracts of gp_lu_factor in its
//                order, and fill entries start at -0.0 so a first update
//                yields the reference's (-l) * u bit for bit.
//   k_gp_solve   right-hand sides with the coupling to later units, then the
//                unit-lower sweep (rows ascending) and the upper sweep (rows
//                descending), a warp per row, the unknowns of up to
//                kGpSolveRhs right-hand sides in shared memory.
#include "gp_dev.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "device_util.cuh"

namespace bdlu {

namespace {

constexpr int kGpWarps = 8;
constexpr int kGpSolveWarps = 8;
constexpr int kGpSolveRhs = 4;  // right-hand sides per pass of the solve
size_t g_gp_smem = 0;           // dynamic shared memory a CTA can have

// Flag states: column (row) pending, done, or the CTA gave up.
constexpr int kPending = 0, kDone = 1, kGiveUp = 2;

// Lane 0 polls flag[k] until it leaves kPending or `abort` is raised, at most
// `limit` polls (with a short sleep between polls after the first 64: the
// default limit then bounds a wait to about a quarter second); the state
// (kGiveUp after the limit) is broadcast to the warp.
__device__ __forceinline__ int warp_wait(const volatile int* flag, int k, const volatile int* abort, int limit) {
  int st = kPending;
  if ((threadIdx.x & 31) == 0) {
    for (int it = 0;; ++it) {
      st = flag[k];
      if (st != kPending) break;
      if (*abort || it >= limit) {
        st = kGiveUp;
        break;
      }
      if (it > 64) __nanosleep(64);
    }
  }
  st = __shfl_sync(0xffffffffu, st, 0);
  __threadfence_block();
  return st;
}

__global__ void __launch_bounds__(32 * kGpWarps) k_gp_factor(GpDev g, const double* __restrict__ vals,
                                                              int32_t* status) {
  extern __shared__ double gp_work[];
  __shared__ int s_abort;
  const int gi = blockIdx.x;
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = g.col0[gi], m = g.col0[gi + 1] - c0;
  double* x = gp_work + static_cast<size_t>(warp) * g.maxm;
  volatile int* done = reinterpret_cast<volatile int*>(gp_work + static_cast<size_t>(nw) * g.maxm);
  volatile int* abort_flag = &s_abort;
  for (int j = threadIdx.x; j < m; j += blockDim.x) done[j] = kPending;
  if (threadIdx.x == 0) s_abort = 0;
  __syncthreads();
  for (int j = warp; j < m; j += nw) {
    const int c = c0 + j;
    const int p0 = g.cptr[c], p1 = g.cptr[c + 1], dp = g.dpos[c];
    for (int q = p0 + lane; q < p1; q += 32) x[g.row[q]] = -0.0;
    __syncwarp();
    for (int q = g.aptr[c] + lane; q < g.aptr[c + 1]; q += 32) x[g.arow[q]] = vals[g.asrc[q]];
    __syncwarp();
    int st = kDone;
    for (int q = p0; q < dp; ++q) {
      const int k = g.row[q];
      st = warp_wait(done, k, abort_flag, g.wait_limit);
      if (st != kDone) break;
      const double u = x[k];
      const int kc = c0 + k;
      const int l1 = g.cptr[kc + 1];
      for (int r = g.dpos[kc] + 1 + lane; r < l1; r += 32) {
        const int i = g.row[r];
        x[i] = __dsub_rn(x[i], __dmul_rn(g.val[r], u));
      }
      __syncwarp();
    }
    if (st != kDone) {
      // A column this one reads failed, or the wait ran out: stop, and make
      // every warp waiting on this column stop too.
      if (lane == 0) {
        if (!*abort_flag) {
          atomicCAS(g.gstat + gi, 0, kGpReasonSync);
          s_abort = 1;
        }
        __threadfence_block();
        done[j] = kGiveUp;
      }
      break;
    }
    // The reference's step j: the largest |entry| on and below the diagonal
    // (an entry wins only if strictly larger, so NaNs never do).
    double best = 0.0;
    for (int q = dp + lane; q < p1; q += 32) {
      const double a = fabs(x[g.row[q]]);
      best = a > best ? a : best;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_xor_sync(0xffffffffu, best, off);
      best = o > best ? o : best;
    }
    const double diag = x[j];
    const double da = fabs(diag);
    int reason = 0;
    if (!(best > 0.0)) reason = 1;  // no nonzero candidate: zero pivot
    else if (!(da >= __dmul_rn(g.diag_tol, best) || da == best)) reason = 2;  // would swap rows
    else if (g.pivot_tol > 0.0 && da < g.pivot_tol) reason = 3;  // tiny pivot
    else if (diag == 0.0) reason = 1;
    else if (g.min_abs_diag > 0.0 && !(da >= g.min_abs_diag)) reason = 4;
    if (reason) {
      if (lane == 0) {
        atomicExch(g.gstat + gi, reason);
        s_abort = 1;
        __threadfence_block();
        done[j] = kGiveUp;
      }
      break;
    }
    for (int q = p0 + lane; q < p1; q += 32) {
      const double v = x[g.row[q]];
      g.val[q] = q > dp ? __ddiv_rn(v, diag) : v;
    }
    __syncwarp();
    __threadfence_block();
    if (lane == 0) done[j] = kDone;
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_abort) {
    const int code = g.gstat[gi] == kGpReasonSync ? kFailSparseSync : kFailSparseReject;
    if (atomicCAS(status, 0, code) == 0) status[1] = g.units[gi];
  }
}

// Uniform poll until every lane with `need` sees ready[col] leave kPending,
// at most `limit` polls; false if a wait gave up, the CTA aborted, or an
// unknown it waited for was given up.
__device__ __forceinline__ bool warp_wait_cols(bool need, int col, const volatile int* ready, const volatile int* abort,
                                               int limit) {
  for (int it = 0;; ++it) {
    if (__all_sync(0xffffffffu, !need || ready[col] != kPending)) break;
    if (*abort || it >= limit) return false;
    if (it > 64) __nanosleep(64);
  }
  if (__any_sync(0xffffffffu, need && ready[col] != kDone)) return false;
  __threadfence_block();
  return true;
}

// Warp-wide sum of v * x[c] over the entries [q0, q1) of one row (column
// indices ci[q], values at positions pos[q]); each entry's unknown is waited
// for through ready[].  The entries whose unknowns are final when the row
// starts are summed and reduced across the warp first; an entry still
// pending (usually the one row the row was waiting for) is kept by its lane
// and added after its wait, so the reduction is off the dependent chain.
// Returns false if a wait gave up.
__device__ __forceinline__ bool row_dot(const GpDev& g, const int32_t* __restrict__ ci,
                                        const int32_t* __restrict__ pos, int q0, int q1, const double* xs, int ld,
                                        int nk, const volatile int* ready, const volatile int* abort,
                                        double (&acc)[kGpSolveRhs]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int kk = 0; kk < kGpSolveRhs; ++kk) acc[kk] = 0.0;
  int lcol = -1;  // this lane's deferred entry
  double lv = 0.0;
  for (int q = q0; q < q1; q += 32) {
    const bool in = q + lane < q1;
    const int col = in ? ci[q + lane] : 0;
    const double v = in ? g.val[pos[q + lane]] : 0.0;
    const int st = in ? ready[col] : kDone;
    if (__any_sync(0xffffffffu, st == kGiveUp)) return false;
    bool defer = in && st == kPending && lcol < 0;
    if (defer) {
      lcol = col;
      lv = v;
    }
    // A lane that already defers one entry waits for its next pending one.
    if (!warp_wait_cols(in && st == kPending && !defer, col, ready, abort, g.wait_limit)) return false;
    __threadfence_block();
#pragma unroll
    for (int kk = 0; kk < kGpSolveRhs; ++kk)
      if (kk < nk && in && !defer) acc[kk] = fma(v, xs[kk * ld + col], acc[kk]);
  }
#pragma unroll
  for (int kk = 0; kk < kGpSolveRhs; ++kk) acc[kk] = warp_sum(acc[kk]);
  const unsigned late = __ballot_sync(0xffffffffu, lcol >= 0);
  if (late == 0u) return true;
  if (!warp_wait_cols(lcol >= 0, lcol, ready, abort, g.wait_limit)) return false;
  double t[kGpSolveRhs];
#pragma unroll
  for (int kk = 0; kk < kGpSolveRhs; ++kk) t[kk] = (kk < nk && lcol >= 0) ? lv * xs[kk * ld + lcol] : 0.0;
  if (__popc(late) == 1) {
    const int who = __ffs(late) - 1;
#pragma unroll
    for (int kk = 0; kk < kGpSolveRhs; ++kk) acc[kk] += __shfl_sync(0xffffffffu, t[kk], who);
  } else {
#pragma unroll
    for (int kk = 0; kk < kGpSolveRhs; ++kk) acc[kk] += warp_sum(t[kk]);
  }
  return true;
}

__global__ void __launch_bounds__(32 * kGpSolveWarps) k_gp_solve(DevPlan dp, GpDev g, const int32_t* __restrict__ glist,
                                                                 const double* __restrict__ rhs, int32_t ldr,
                                                                 double* xp, const int32_t* __restrict__ nrhs_p) {
  extern __shared__ double gs_x[];
  __shared__ int s_abort;
  const int gi = glist[blockIdx.x];
  const int u = g.units[gi];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nrhs = *nrhs_p;
  const size_t n = static_cast<size_t>(dp.n);
  const int c0 = g.col0[gi];
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ld = g.maxm;
  volatile int* ready = reinterpret_cast<volatile int*>(gs_x + static_cast<size_t>(kGpSolveRhs) * ld);
  volatile int* abort_flag = &s_abort;
  if (threadIdx.x == 0) s_abort = 0;
  for (int k0 = 0; k0 < nrhs; k0 += kGpSolveRhs) {
    const int nk = min(kGpSolveRhs, nrhs - k0);
    // Right-hand sides: b (original row order) minus the coupling to the
    // units solved before this one.
    for (int idx = threadIdx.x; idx < m * nk; idx += blockDim.x) {
      const int i = idx % m, kk = idx / m;
      const size_t k = static_cast<size_t>(k0 + kk);
      const int r = s + i;
      double acc = 0.0;
      for (int q = dp.cpl_ptr[r]; q < dp.cpl_ptr[r + 1]; ++q) acc = fma(dp.cpl_val[q], xp[dp.cpl_col[q] + k * n], acc);
      gs_x[kk * ld + i] = rhs[dp.P[r] + k * static_cast<size_t>(ldr)] - acc;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) ready[i] = kPending;
    __syncthreads();
    // y = L^{-1} rhs, rows ascending.
    double acc[kGpSolveRhs];
    for (int i = warp; i < m; i += nw) {
      const int gr = c0 + i;
      const bool ok = row_dot(g, g.lci, g.lpos, g.lrp[gr], g.lrp[gr + 1], gs_x, ld, nk, ready, abort_flag, acc);
      if (lane == 0) {
        if (ok) {
          for (int kk = 0; kk < nk; ++kk) gs_x[kk * ld + i] -= acc[kk];
        } else {
          s_abort = 1;
        }
        __threadfence_block();
        ready[i] = ok ? kDone : kGiveUp;
      }
      if (!ok) break;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) ready[i] = kPending;
    __syncthreads();
    // x = U^{-1} y, rows descending.
    if (!*abort_flag) {
      for (int t = warp; t < m; t += nw) {
        const int i = m - 1 - t;
        const int gr = c0 + i;
        const bool ok = row_dot(g, g.uci, g.upos, g.urp[gr], g.urp[gr + 1], gs_x, ld, nk, ready, abort_flag, acc);
        if (lane == 0) {
          if (ok) {
            const double d = g.val[g.dpos[gr]];
            for (int kk = 0; kk < nk; ++kk) gs_x[kk * ld + i] = __ddiv_rn(gs_x[kk * ld + i] - acc[kk], d);
          } else {
            s_abort = 1;
          }
          __threadfence_block();
          ready[i] = ok ? kDone : kGiveUp;
        }
        if (!ok) break;
      }
    }
    __syncthreads();
    if (*abort_flag) {
      if (threadIdx.x == 0 && atomicCAS(dp.status, 0, kFailSync) == 0) dp.status[1] = u;
      return;
    }
    for (int idx = threadIdx.x; idx < m * nk; idx += blockDim.x) {
      const int i = idx % m, kk = idx / m;
      xp[s + i + static_cast<size_t>(k0 + kk) * n] = gs_x[kk * ld + i];
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t gp_setup() {
  static std::once_flag once;
  static cudaError_t err = cudaSuccess;
  std::call_once(once, [] {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const int dyn = std::max(0, optin - 2048);
    err = cudaFuncSetAttribute(k_gp_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(k_gp_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    g_gp_smem = static_cast<size_t>(dyn);
  });
  return err;
}

cudaError_t gp_factor_launch(const GpDev& g, int32_t count, const double* vals, int32_t* status,
                             cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  // Per warp a work vector of maxm doubles; one flag word per column.
  const size_t per_warp = static_cast<size_t>(g.maxm) * sizeof(double);
  const size_t flags = static_cast<size_t>(g.maxm) * sizeof(int);
  if (per_warp + flags > g_gp_smem) return cudaErrorInvalidValue;
  const int w = static_cast<int>(std::min<size_t>(kGpWarps, (g_gp_smem - flags) / per_warp));
  k_gp_factor<<<count, 32 * w, static_cast<size_t>(w) * per_warp + flags, stream>>>(g, vals, status);
  return cudaGetLastError();
}

cudaError_t gp_solve_launch(const DevPlan& dp, const GpDev& g, const int32_t* glist, int32_t count,
                            const double* rhs, int32_t ldr, double* xp, const int32_t* nrhs, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const size_t smem = static_cast<size_t>(g.maxm) * (kGpSolveRhs * sizeof(double) + sizeof(int));
  if (smem > g_gp_smem) return cudaErrorInvalidValue;
  k_gp_solve<<<count, 32 * kGpSolveWarps, smem, stream>>>(dp, g, glist, rhs, ldr, xp, nrhs);
  return cudaGetLastError();
}

}  // namespace bdlu
