// sm_100a kernels of the sparse-LU route (gp.h):
//   k_gp_factor  one CTA per sparse unit; its columns are taken level by
//                level (a column depends only on columns of earlier levels),
//                one warp per column: the column is formed in the warp's
//                shared-memory work vector (A's entries, then for each row k
//                above the diagonal in ascending order x -= L(:,k) x[k],
//                read as coalesced runs of the column-compressed L), the
//                reference's pivot test is applied (gp_lu.cpp:164-218) and
//                the column is written back (U, pivot, L = x / pivot).
//                Updates are unfused (__dmul_rn, __dsub_rn): each entry sees
//                the multiply-subtracts of gp_lu_factor in its order, and
//                fill entries start at -0.0 so a first update yields the
//                reference's (-l) * u bit for bit.
//   k_gp_solve   one CTA per sparse unit of a solve level: right-hand sides
//                with the coupling to later units, then the unit-lower and
//                upper sweeps by row levels, one thread per (row, rhs), sums
//                in ascending column order as gp_lu_solve_inplace_strided
//                (gp_lu.cpp:242-306).
#include "gp_dev.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "device_util.cuh"

namespace bdlu {

namespace {

constexpr int kGpWarps = 8;
constexpr int kGpSolveThreads = 256;
size_t g_gp_smem = 0;  // dynamic shared memory available to k_gp_factor

__global__ void __launch_bounds__(32 * kGpWarps) k_gp_factor(GpDev g, const double* __restrict__ vals,
                                                              int32_t* status) {
  extern __shared__ double gp_work[];
  __shared__ int s_fail;
  const int gi = blockIdx.x;
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* x = gp_work + static_cast<size_t>(warp) * g.maxm;
  if (threadIdx.x == 0) s_fail = 0;
  __syncthreads();
  const int c0 = g.col0[gi];
  for (int t = g.clvl0[gi]; t < g.clvl0[gi + 1]; ++t) {
    const int b = g.clvlb[t], e = g.clvlb[t + 1];
    for (int idx = b + warp; idx < e; idx += nw) {
      const int j = g.corder[idx];
      const int c = c0 + j;
      const int p0 = g.cptr[c], p1 = g.cptr[c + 1], dp = g.dpos[c];
      for (int q = p0 + lane; q < p1; q += 32) x[g.row[q]] = -0.0;
      __syncwarp();
      for (int q = g.aptr[c] + lane; q < g.aptr[c + 1]; q += 32) x[g.arow[q]] = vals[g.asrc[q]];
      __syncwarp();
      for (int q = p0; q < dp; ++q) {
        const int k = g.row[q];
        const double u = x[k];
        const int kc = c0 + k;
        const int l1 = g.cptr[kc + 1];
        for (int r = g.dpos[kc] + 1 + lane; r < l1; r += 32) {
          const int i = g.row[r];
          x[i] = __dsub_rn(x[i], __dmul_rn(g.val[r], u));
        }
        __syncwarp();
      }
      // The reference's step j: the largest |entry| on and below the
      // diagonal (an entry wins only if strictly larger, so NaNs never do).
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
          atomicCAS(g.gstat + gi, 0, reason);
          s_fail = 1;
        }
        __syncwarp();
        continue;
      }
      for (int q = p0 + lane; q < p1; q += 32) {
        const double v = x[g.row[q]];
        g.val[q] = q > dp ? __ddiv_rn(v, diag) : v;
      }
      __syncwarp();
    }
    __syncthreads();
    if (s_fail) break;
  }
  if (threadIdx.x == 0 && s_fail) {
    if (atomicCAS(status, 0, kFailSparseReject) == 0) status[1] = g.units[gi];
  }
}

__global__ void __launch_bounds__(kGpSolveThreads) k_gp_solve(DevPlan dp, GpDev g, const int32_t* __restrict__ glist,
                                                              const double* __restrict__ rhs, int32_t ldr,
                                                              double* xp, const int32_t* __restrict__ nrhs_p) {
  const int gi = glist[blockIdx.x];
  const int u = g.units[gi];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nrhs = *nrhs_p;
  const size_t n = static_cast<size_t>(dp.n);
  const int c0 = g.col0[gi];
  // Right-hand sides: b (original row order) minus the coupling to the
  // units solved before this one.
  for (long long idx = threadIdx.x; idx < static_cast<long long>(m) * nrhs; idx += blockDim.x) {
    const int i = static_cast<int>(idx % m);
    const size_t k = static_cast<size_t>(idx / m);
    const int r = s + i;
    double acc = 0.0;
    for (int q = dp.cpl_ptr[r]; q < dp.cpl_ptr[r + 1]; ++q) acc = fma(dp.cpl_val[q], xp[dp.cpl_col[q] + k * n], acc);
    xp[r + k * n] = rhs[dp.P[r] + k * static_cast<size_t>(ldr)] - acc;
  }
  __syncthreads();
  double* xu = xp + s;
  // y = L^{-1} rhs: row i after the rows its L row reads.
  for (int t = g.flvl0[gi]; t < g.flvl0[gi + 1]; ++t) {
    const int b = g.flvlb[t], cnt = g.flvlb[t + 1] - b;
    for (long long idx = threadIdx.x; idx < static_cast<long long>(cnt) * nrhs; idx += blockDim.x) {
      const int i = g.frow[b + static_cast<int>(idx % cnt)];
      double* xk = xu + static_cast<size_t>(idx / cnt) * n;
      const int gr = c0 + i;
      double sum = xk[i];
      for (int q = g.lrp[gr]; q < g.lrp[gr + 1]; ++q) sum = __dsub_rn(sum, __dmul_rn(g.val[g.lpos[q]], xk[g.lci[q]]));
      xk[i] = sum;
    }
    __syncthreads();
  }
  // x = U^{-1} y: row i after the rows its U row reads.
  for (int t = g.blvl0[gi]; t < g.blvl0[gi + 1]; ++t) {
    const int b = g.blvlb[t], cnt = g.blvlb[t + 1] - b;
    for (long long idx = threadIdx.x; idx < static_cast<long long>(cnt) * nrhs; idx += blockDim.x) {
      const int i = g.brow[b + static_cast<int>(idx % cnt)];
      double* xk = xu + static_cast<size_t>(idx / cnt) * n;
      const int gr = c0 + i;
      double sum = xk[i];
      for (int q = g.urp[gr]; q < g.urp[gr + 1]; ++q) sum = __dsub_rn(sum, __dmul_rn(g.val[g.upos[q]], xk[g.uci[q]]));
      xk[i] = __ddiv_rn(sum, g.val[g.dpos[gr]]);
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
    g_gp_smem = static_cast<size_t>(dyn);
  });
  return err;
}

cudaError_t gp_factor_launch(const GpDev& g, int32_t count, const double* vals, int32_t* status,
                             cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const size_t per_warp = static_cast<size_t>(g.maxm) * sizeof(double);
  if (per_warp > g_gp_smem) return cudaErrorInvalidValue;
  const int w = static_cast<int>(std::min<size_t>(kGpWarps, g_gp_smem / per_warp));
  k_gp_factor<<<count, 32 * w, static_cast<size_t>(w) * per_warp, stream>>>(g, vals, status);
  return cudaGetLastError();
}

cudaError_t gp_solve_launch(const DevPlan& dp, const GpDev& g, const int32_t* glist, int32_t count,
                            const double* rhs, int32_t ldr, double* xp, const int32_t* nrhs, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  k_gp_solve<<<count, kGpSolveThreads, 0, stream>>>(dp, g, glist, rhs, ldr, xp, nrhs);
  return cudaGetLastError();
}

}  // namespace bdlu
