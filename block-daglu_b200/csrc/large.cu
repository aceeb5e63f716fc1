// Large units (dense blocks above the shared-memory limit): blocked
// right-looking partial-pivoting LU and block-triangular solves.
//
// Layout: a large unit's slot in the LU arena is ROW-major m x m (row swaps
// are contiguous; every kernel reads whole row segments).
//
// Factor, per step of kPanel columns (k0 = step * kPanel), batched over all
// large units still active at that step:
//   k_panel_cluster   the panel A[k0:m, k0:k0+nb] of each unit is held in the
//                     shared memory of a thread-block cluster (C <= 8 CTAs,
//                     rows split contiguously).  Per column: each CTA finds
//                     its local pivot candidate (first strict maximum, the
//                     reference's rule), pushes the candidate's value, index
//                     and full panel row into every peer's shared memory
//                     (DSMEM), and the owner of the diagonal row pushes that
//                     row; one cluster barrier later every CTA holds all
//                     candidates, picks the same pivot, performs its part of
//                     the swap locally and applies the rank-1 update to its
//                     rows.  Candidate buffers alternate by column parity, so
//                     one barrier per column suffices.
//   k_panel_global    the same for units too tall for a cluster (one CTA,
//                     panel in global memory; correctness fallback)
//   k_swap_trsm_rm    the panel's row swaps applied to every other column and
//                     U12 = L11^{-1} A12, one thread per column (coalesced)
//   k_gemm_rm         A22 -= L21 * U12, FP64, 128 x 128 output tile per CTA,
//                     8 x 8 accumulators per thread
//   k_large_perm      final row order of each unit from its pivot sequence
// Solve (per level holding large units):
//   k_large_rhs       rhs of every row in pivot order: b - A_cpl x, gathered
//                     through the unit's final row order
//   k_large_single    units up to kLargeSingleMax rows: one CTA, forward and
//                     backward sweeps by 64-row tiles (row-major GEMV + a
//                     64 x 64 triangle in shared memory)
//   k_trsv_fwd_rm / k_trsv_bwd_rm
//                     taller units: one launch per 64-row tile; the CTAs of
//                     the later tiles apply the finished tile's update and the
//                     next tile's CTA solves its diagonal triangle
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "device_util.cuh"
#include "large.h"

namespace cg = cooperative_groups;

namespace bdlu {

namespace {

constexpr int kPT = 512;                  // panel kernel threads
constexpr int kPStride = kPanel + 1;      // shared-memory row stride of the panel (doubles)
constexpr int kClusterMaxCtas = 8;        // portable cluster size
constexpr int kPanelRowsMax = 800;        // panel rows one CTA holds (800 * 33 * 8 = 211,200 B)
constexpr int kGT = 128;                  // GEMM output tile
constexpr int kGThreads = 256;
constexpr int kTile = 64;                 // solve tile
constexpr int kSolveThreads = 256;

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPT) k_panel_cluster(DevPlan dp, int32_t k0, int32_t ubase, int32_t csize) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ double P[];
  __shared__ double cand[2][kClusterMaxCtas][kPanel + 2];
  __shared__ double jbuf[2][kPanel];
  __shared__ double s_best[kPT / 32];
  __shared__ int s_bi[kPT / 32];
  __shared__ double s_cbest;
  __shared__ int s_cbi;
  const int rank = static_cast<int>(cl.block_rank());
  const int u = dp.step_unit[ubase + blockIdx.x / csize];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kPanel, m - k0);
  double* A = dp.lu + dp.lu_off[u];
  const int R = m - k0;
  const int chunk = (R + csize - 1) / csize;
  const int r0 = k0 + rank * chunk;
  const int r1 = min(m, r0 + chunk);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // Load my rows of the panel.
  for (int t = tid; t < (r1 > r0 ? (r1 - r0) : 0) * kPanel; t += kPT) {
    const int i = t / kPanel, c = t - i * kPanel;
    P[i * kPStride + c] = (c < nb) ? A[static_cast<size_t>(r0 + i) * m + k0 + c] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const int jj = k0 + j;
    const int par = j & 1;
    // Local candidate among rows >= jj.
    double best = 0.0;
    int bi = m;
    for (int i = max(r0, jj) + tid; i < r1; i += kPT) {
      const double a = fabs(P[(i - r0) * kPStride + j]);
      if (bi == m || a > best) {
        best = a;
        bi = i;
      }
    }
    warp_pivot_reduce(best, bi, m);
    if (lane == 0) {
      s_best[warp] = best;
      s_bi[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      best = (lane < kPT / 32) ? s_best[lane] : 0.0;
      bi = (lane < kPT / 32) ? s_bi[lane] : m;
      warp_pivot_reduce(best, bi, m);
      if (lane == 0) {
        s_cbest = best;
        s_cbi = bi;
      }
    }
    __syncthreads();
    // Push the candidate (row, value, index) to every CTA of the cluster;
    // the owner of row jj pushes that row as well.
    const int oj = (jj - k0) / chunk;
    if (warp < csize) {
      const int q = warp;
      double* dst = cl.map_shared_rank(&cand[par][rank][0], q);
      const int cbi = s_cbi;
      if (lane < kPanel) dst[lane] = (cbi != m) ? P[(cbi - r0) * kPStride + lane] : 0.0;
      if (lane == 0) {
        dst[kPanel] = s_cbest;
        dst[kPanel + 1] = static_cast<double>(cbi);
      }
    } else if (rank == oj && warp >= kClusterMaxCtas && warp < kClusterMaxCtas + csize) {
      const int q = warp - kClusterMaxCtas;
      double* dst = cl.map_shared_rank(&jbuf[par][0], q);
      if (lane < kPanel) dst[lane] = P[(jj - r0) * kPStride + lane];
    }
    cl.sync();
    // Every CTA combines the candidates in rank order: the same pivot.
    best = cand[par][0][kPanel];
    bi = static_cast<int>(cand[par][0][kPanel + 1]);
    int owner = 0;
    for (int q = 1; q < csize; ++q) {
      const double ob = cand[par][q][kPanel];
      const int oi = static_cast<int>(cand[par][q][kPanel + 1]);
      const int before = bi;
      pivot_combine(best, bi, ob, oi, m);
      if (bi != before) owner = q;
    }
    if (bi == m || best == 0.0) {
      if (rank == 0 && tid == 0) report_failure(dp.status, u);
      cl.sync();
      return;
    }
    const int p = bi;
    const double* U = cand[par][owner];
    if (rank == 0 && tid == 0) dp.piv[s + jj] = p;
    if (rank == oj && tid < nb) P[(jj - r0) * kPStride + tid] = U[tid];
    if (rank == owner && p != jj && tid < nb) P[(p - r0) * kPStride + tid] = jbuf[par][tid];
    __syncthreads();
    const double d = U[j];
    for (int i = max(r0, jj + 1) + tid; i < r1; i += kPT) {
      double* row = P + (i - r0) * kPStride;
      const double l = row[j] / d;
      row[j] = l;
      for (int c = j + 1; c < nb; ++c) row[c] = fma(-l, U[c], row[c]);
    }
    __syncthreads();
  }
  for (int t = tid; t < (r1 > r0 ? (r1 - r0) : 0) * nb; t += kPT) {
    const int i = t / nb, c = t - i * nb;
    A[static_cast<size_t>(r0 + i) * m + k0 + c] = P[i * kPStride + c];
  }
  cl.sync();
}

// Fallback panel for units taller than a cluster holds: one CTA, global memory.
__global__ void __launch_bounds__(kPT) k_panel_global(DevPlan dp, int32_t k0, int32_t ubase) {
  __shared__ double s_best[kPT / 32];
  __shared__ int s_bi[kPT / 32];
  __shared__ int s_piv;
  __shared__ double s_pbest;
  __shared__ double urow[kPanel];
  const int u = dp.step_unit[ubase + blockIdx.x];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kPanel, m - k0);
  double* A = dp.lu + dp.lu_off[u];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = 0; j < nb; ++j) {
    const int jj = k0 + j;
    double best = 0.0;
    int bi = m;
    for (int i = jj + tid; i < m; i += kPT) {
      const double a = fabs(A[static_cast<size_t>(i) * m + jj]);
      if (bi == m || a > best) {
        best = a;
        bi = i;
      }
    }
    warp_pivot_reduce(best, bi, m);
    if (lane == 0) {
      s_best[warp] = best;
      s_bi[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      best = (lane < kPT / 32) ? s_best[lane] : 0.0;
      bi = (lane < kPT / 32) ? s_bi[lane] : m;
      warp_pivot_reduce(best, bi, m);
      if (lane == 0) {
        s_piv = bi;
        s_pbest = best;
      }
    }
    __syncthreads();
    const int p = s_piv;
    if (s_pbest == 0.0) {
      if (tid == 0) report_failure(dp.status, u);
      return;
    }
    if (tid == 0) dp.piv[s + jj] = p;
    if (tid < nb) {
      double* rj = A + static_cast<size_t>(jj) * m + k0;
      double* rp = A + static_cast<size_t>(p) * m + k0;
      const double t = rj[tid];
      rj[tid] = rp[tid];
      rp[tid] = t;
      urow[tid] = rj[tid];
    }
    __syncthreads();
    const double d = urow[j];
    for (int i = jj + 1 + tid; i < m; i += kPT) {
      double* row = A + static_cast<size_t>(i) * m + k0;
      const double l = row[j] / d;
      row[j] = l;
      for (int c = j + 1; c < nb; ++c) row[c] = fma(-l, urow[c], row[c]);
    }
    __syncthreads();
  }
}

// Row swaps of the panel applied to all other columns, then U12 for the
// columns right of the panel.  One thread per column.
__global__ void __launch_bounds__(kTrsmCols) k_swap_trsm_rm(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact) {
  __shared__ double L11[kPanel][kPanel + 1];
  __shared__ int spiv[kPanel];
  int a = 0;
  while (a + 1 < nact && dp.step_trsm_pref[ubase + a + 1] <= static_cast<int>(blockIdx.x)) ++a;
  const int u = dp.step_unit[ubase + a];
  const int chunk = blockIdx.x - dp.step_trsm_pref[ubase + a];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kPanel, m - k0);
  double* A = dp.lu + dp.lu_off[u];
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
    const int r = t / nb, q = t - r * nb;
    L11[r][q] = A[static_cast<size_t>(k0 + r) * m + k0 + q];
  }
  if (threadIdx.x < nb) spiv[threadIdx.x] = dp.piv[s + k0 + threadIdx.x];
  __syncthreads();
  const int j = chunk * kTrsmCols + threadIdx.x;
  if (j >= m || (j >= k0 && j < k0 + nb)) return;
  for (int r = 0; r < nb; ++r) {
    const int p = spiv[r];
    if (p != k0 + r) {
      double* x = A + static_cast<size_t>(k0 + r) * m + j;
      double* y = A + static_cast<size_t>(p) * m + j;
      const double t = *x;
      *x = *y;
      *y = t;
    }
  }
  if (j < k0 + nb) return;
  double x[kPanel];
#pragma unroll
  for (int r = 0; r < kPanel; ++r) x[r] = (r < nb) ? A[static_cast<size_t>(k0 + r) * m + j] : 0.0;
#pragma unroll
  for (int r = 1; r < kPanel; ++r) {
    double v = x[r];
#pragma unroll
    for (int q = 0; q < r; ++q) v = fma(-L11[r][q], x[q], v);
    x[r] = v;
  }
#pragma unroll
  for (int r = 0; r < kPanel; ++r)
    if (r < nb) A[static_cast<size_t>(k0 + r) * m + j] = x[r];
}

// A22 -= L21 * U12 on row-major storage; the panel depth is staged in two
// halves of kKC columns.
constexpr int kKC = 16;
__global__ void __launch_bounds__(kGThreads, 1) k_gemm_rm(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact) {
  __shared__ double As[kKC][kGT + 1];
  __shared__ double Bs[kKC][kGT];
  int a = 0;
  while (a + 1 < nact && dp.step_gemm_pref[ubase + a + 1] <= static_cast<int>(blockIdx.x)) ++a;
  const int u = dp.step_unit[ubase + a];
  const int tile = blockIdx.x - dp.step_gemm_pref[ubase + a];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kPanel, m - k0);
  const int base = k0 + nb;
  const int rest = m - base;
  const int nt = (rest + kGT - 1) / kGT;
  const int ti = tile % nt, tj = tile / nt;
  const int i0 = base + ti * kGT, j0 = base + tj * kGT;
  double* A = dp.lu + dp.lu_off[u];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  double acc[8][8];
#pragma unroll
  for (int x = 0; x < 8; ++x)
#pragma unroll
    for (int y = 0; y < 8; ++y) acc[x][y] = 0.0;
  for (int h = 0; h < kPanel; h += kKC) {
    for (int t = tid; t < kGT * kKC; t += kGThreads) {
      const int i = t / kKC, q = t - i * kKC;
      As[q][i] = (h + q < nb && i0 + i < m) ? A[static_cast<size_t>(i0 + i) * m + k0 + h + q] : 0.0;
    }
    for (int t = tid; t < kKC * kGT; t += kGThreads) {
      const int q = t / kGT, jj = t - q * kGT;
      Bs[q][jj] = (h + q < nb && j0 + jj < m) ? A[static_cast<size_t>(k0 + h + q) * m + j0 + jj] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < kKC; ++q) {
      double av[8], bv[8];
#pragma unroll
      for (int x = 0; x < 8; ++x) av[x] = As[q][ty + 16 * x];
#pragma unroll
      for (int y = 0; y < 8; ++y) bv[y] = Bs[q][tx + 16 * y];
#pragma unroll
      for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int y = 0; y < 8; ++y) acc[x][y] = fma(av[x], bv[y], acc[x][y]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 8; ++x) {
    const int i = i0 + ty + 16 * x;
    if (i >= m) continue;
    double* row = A + static_cast<size_t>(i) * m;
#pragma unroll
    for (int y = 0; y < 8; ++y) {
      const int j = j0 + tx + 16 * y;
      if (j < m) row[j] -= acc[x][y];
    }
  }
}

// Final row order of each large unit: row k of its factor is local row perm[k].
__global__ void k_large_perm(DevPlan dp, const int32_t* __restrict__ units, int32_t count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int u = units[t];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  int32_t* perm = dp.lperm + s;
  for (int k = 0; k < m; ++k) perm[k] = k;
  for (int k = 0; k < m; ++k) {
    const int p = dp.piv[s + k];
    if (p != k) {
      const int32_t tmp = perm[k];
      perm[k] = perm[p];
      perm[p] = tmp;
    }
  }
}

// rhs of each row in pivot order: xp[s + k] = b[P[s + perm[k]]] - A_cpl x.
__global__ void __launch_bounds__(kSolveThreads) k_large_rhs(DevPlan dp, const int32_t* __restrict__ units,
                                                             const double* __restrict__ rhs, int32_t ldr,
                                                             double* __restrict__ xp, int32_t nrhs) {
  const int u = units[blockIdx.y];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int lane = threadIdx.x & 31;
  const int n = dp.n;
  const int nw = kSolveThreads / 32;
  for (int k = blockIdx.x * nw + (threadIdx.x >> 5); k < m; k += gridDim.x * nw) {
    const int r = s + dp.lperm[s + k];
    const int p0 = dp.cpl_ptr[r], p1 = dp.cpl_ptr[r + 1];
    for (int c = 0; c < nrhs; ++c) {
      const double* xc = xp + static_cast<size_t>(c) * n;
      double acc = 0.0;
      for (int q = p0 + lane; q < p1; q += 32) acc = fma(dp.cpl_val[q], xc[dp.cpl_col[q]], acc);
      acc = warp_sum(acc);
      if (lane == 0) xp[s + k + static_cast<size_t>(c) * n] = rhs[dp.P[r] + static_cast<size_t>(c) * ldr] - acc;
    }
  }
}

// 64 x 64 triangle of tile `t0` (rows/cols t0..t0+w) solved in place on x.
// Warp-level, the tile staged in shared memory.  lower: unit-lower forward;
// else upper backward with division by the diagonal.
__device__ void tile_triangle(const double* LU, int m, int t0, int w, double* x, double* Ts, bool lower) {
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
    const int i = t / w, c = t - i * w;
    Ts[i * kTile + c] = LU[static_cast<size_t>(t0 + i) * m + t0 + c];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (lower) {
      for (int r = 0; r < w; ++r) {
        const double xr = x[t0 + r];
        __syncwarp();
        for (int i = r + 1 + lane; i < w; i += 32) x[t0 + i] = fma(-Ts[i * kTile + r], xr, x[t0 + i]);
        __syncwarp();
      }
    } else {
      for (int r = w - 1; r >= 0; --r) {
        const double xr = x[t0 + r] / Ts[r * kTile + r];
        __syncwarp();
        if (lane == 0) x[t0 + r] = xr;
        for (int i = lane; i < r; i += 32) x[t0 + i] = fma(-Ts[i * kTile + r], xr, x[t0 + i]);
        __syncwarp();
      }
    }
  }
  __syncthreads();
}

// Units up to kLargeSingleMax rows: the whole solve in one CTA.
__global__ void __launch_bounds__(kSolveThreads) k_large_single(DevPlan dp, const int32_t* __restrict__ units,
                                                                double* __restrict__ xp, int32_t nrhs) {
  extern __shared__ double sm[];
  double* Ts = sm;                  // kTile * kTile
  double* x = sm + kTile * kTile;   // m
  const int u = units[blockIdx.x];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const double* LU = dp.lu + dp.lu_off[u];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = kSolveThreads / 32;
  const int nt = (m + kTile - 1) / kTile;
  for (int c = 0; c < nrhs; ++c) {
    double* xg = xp + static_cast<size_t>(c) * dp.n + s;
    for (int i = threadIdx.x; i < m; i += kSolveThreads) x[i] = xg[i];
    __syncthreads();
    for (int I = 0; I < nt; ++I) {
      const int t0 = I * kTile, w = min(kTile, m - t0);
      for (int i = t0 + warp; i < t0 + w; i += nw) {
        const double* row = LU + static_cast<size_t>(i) * m;
        double acc = 0.0;
        for (int q = lane; q < t0; q += 32) acc = fma(row[q], x[q], acc);
        acc = warp_sum(acc);
        if (lane == 0) x[i] -= acc;
      }
      __syncthreads();
      tile_triangle(LU, m, t0, w, x, Ts, true);
    }
    for (int I = nt - 1; I >= 0; --I) {
      const int t0 = I * kTile, w = min(kTile, m - t0);
      for (int i = t0 + warp; i < t0 + w; i += nw) {
        const double* row = LU + static_cast<size_t>(i) * m;
        double acc = 0.0;
        for (int q = t0 + w + lane; q < m; q += 32) acc = fma(row[q], x[q], acc);
        acc = warp_sum(acc);
        if (lane == 0) x[i] -= acc;
      }
      __syncthreads();
      tile_triangle(LU, m, t0, w, x, Ts, false);
    }
    for (int i = threadIdx.x; i < m; i += kSolveThreads) xg[i] = x[i];
    __syncthreads();
  }
}

// Forward sweep step J of a tall unit: tiles I > J take x_J's update; tile
// J + 1 then solves its triangle.  J = -1 solves tile 0 only.
__global__ void __launch_bounds__(kSolveThreads) k_trsv_fwd_rm(DevPlan dp, int32_t u, int32_t J,
                                                               double* __restrict__ xp, int32_t nrhs) {
  __shared__ double Ts[kTile * kTile];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const double* LU = dp.lu + dp.lu_off[u];
  const int I = J + 1 + blockIdx.x;
  const int t0 = I * kTile, w = min(kTile, m - t0);
  const int j0 = J * kTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < nrhs; ++c) {
    double* x = xp + static_cast<size_t>(c) * dp.n + s;
    if (J >= 0) {
      for (int i = t0 + warp; i < t0 + w; i += kSolveThreads / 32) {
        const double* row = LU + static_cast<size_t>(i) * m + j0;
        double acc = 0.0;
        for (int q = lane; q < kTile; q += 32) acc = fma(row[q], x[j0 + q], acc);
        acc = warp_sum(acc);
        if (lane == 0) x[i] -= acc;
      }
      __syncthreads();
    }
    if (I == J + 1) tile_triangle(LU, m, t0, w, x, Ts, true);
  }
}

// Backward sweep step J of a tall unit: tiles I < J take x_J's update; tile
// J - 1 then solves its triangle.  J = nt solves the last tile only.
__global__ void __launch_bounds__(kSolveThreads) k_trsv_bwd_rm(DevPlan dp, int32_t u, int32_t J, int32_t nt,
                                                               double* __restrict__ xp, int32_t nrhs) {
  __shared__ double Ts[kTile * kTile];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const double* LU = dp.lu + dp.lu_off[u];
  const int I = J - 1 - blockIdx.x;
  const int t0 = I * kTile, w = min(kTile, m - t0);
  const int j0 = J * kTile, jw = (J < nt) ? min(kTile, m - j0) : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < nrhs; ++c) {
    double* x = xp + static_cast<size_t>(c) * dp.n + s;
    if (J < nt) {
      for (int i = t0 + warp; i < t0 + w; i += kSolveThreads / 32) {
        const double* row = LU + static_cast<size_t>(i) * m + j0;
        double acc = 0.0;
        for (int q = lane; q < jw; q += 32) acc = fma(row[q], x[j0 + q], acc);
        acc = warp_sum(acc);
        if (lane == 0) x[i] -= acc;
      }
      __syncthreads();
    }
    if (I == J - 1) tile_triangle(LU, m, t0, w, x, Ts, false);
  }
}

int cluster_size_for(int rows) {
  int c = (rows + kPanelRowsMax - 1) / kPanelRowsMax;
  return std::max(1, c);
}

}  // namespace

cudaError_t large_setup() {
  static std::once_flag once;
  static cudaError_t err = cudaSuccess;
  std::call_once(once, [] {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    err = cudaFuncSetAttribute(k_panel_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 8 * 1024);
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_large_single, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (kTile * kTile + kLargeSingleMax) * static_cast<int>(sizeof(double)));
  });
  return err;
}

cudaError_t large_factor(const DevPlan& dp, const Plan& p, const int32_t* d_large_units, cudaStream_t stream,
                         int32_t* launches) {
  cudaError_t e = large_setup();
  if (e != cudaSuccess) return e;
  for (int32_t st = 0; st < p.nsteps; ++st) {
    const int32_t ub = p.step_ptr[static_cast<size_t>(st)];
    const int32_t na = p.step_ptr[static_cast<size_t>(st) + 1] - ub;
    if (na <= 0) continue;
    const int32_t k0 = st * kPanel;
    const int32_t rows = p.step_max_rows[static_cast<size_t>(st)];
    const int csize = cluster_size_for(rows);
    if (csize <= kClusterMaxCtas) {
      const int chunk = (rows + csize - 1) / csize;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(static_cast<unsigned>(na * csize));
      cfg.blockDim = dim3(kPT);
      cfg.dynamicSmemBytes = static_cast<size_t>(chunk) * kPStride * sizeof(double);
      cfg.stream = stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = static_cast<unsigned>(csize);
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      e = cudaLaunchKernelEx(&cfg, k_panel_cluster, dp, k0, ub, static_cast<int32_t>(csize));
      if (e != cudaSuccess) return e;
    } else {
      k_panel_global<<<na, kPT, 0, stream>>>(dp, k0, ub);
    }
    k_swap_trsm_rm<<<p.step_trsm_total[static_cast<size_t>(st)], kTrsmCols, 0, stream>>>(dp, k0, ub, na);
    *launches += 2;
    if (p.step_gemm_total[static_cast<size_t>(st)] > 0) {
      k_gemm_rm<<<p.step_gemm_total[static_cast<size_t>(st)], kGThreads, 0, stream>>>(dp, k0, ub, na);
      ++*launches;
    }
  }
  const int nl = static_cast<int>(p.large_units.size());
  if (nl > 0) {
    k_large_perm<<<(nl + 127) / 128, 128, 0, stream>>>(dp, d_large_units, nl);
    ++*launches;
  }
  return cudaGetLastError();
}

cudaError_t large_solve_level(const DevPlan& dp, const Plan& p, const int32_t* d_units, const int32_t* h_units,
                              int32_t count, const double* rhs, int32_t ldr, double* xp, int32_t nrhs,
                              cudaStream_t stream, int32_t* launches) {
  if (count <= 0) return cudaSuccess;
  int32_t mmax = 0;
  for (int32_t k = 0; k < count; ++k) {
    const int32_t u = h_units[k];
    mmax = std::max(mmax, p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]);
  }
  const int gx = std::min<int32_t>((mmax + 63) / 64, 64);
  k_large_rhs<<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(count)), kSolveThreads, 0, stream>>>(
      dp, d_units, rhs, ldr, xp, nrhs);
  ++*launches;
  // Units are grouped by the solve they take: one CTA for the shorter ones, a
  // tile-by-tile launch sequence per tall unit.
  int32_t nsingle = 0;
  for (int32_t k = 0; k < count; ++k) {
    const int32_t u = h_units[k];
    const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
    if (m <= kLargeSingleMax) ++nsingle;
  }
  if (nsingle > 0) {
    // d_units is ordered with the single-CTA units first (see plan.cpp).
    k_large_single<<<nsingle, kSolveThreads, (kTile * kTile + kLargeSingleMax) * sizeof(double), stream>>>(
        dp, d_units, xp, nrhs);
    ++*launches;
  }
  for (int32_t k = nsingle; k < count; ++k) {
    const int32_t u = h_units[k];
    const int32_t m = p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)];
    const int32_t nt = (m + kTile - 1) / kTile;
    for (int32_t J = -1; J < nt - 1; ++J) {
      k_trsv_fwd_rm<<<(J < 0) ? 1 : nt - J - 1, kSolveThreads, 0, stream>>>(dp, u, J, xp, nrhs);
      ++*launches;
    }
    for (int32_t J = nt; J > 0; --J) {
      k_trsv_bwd_rm<<<(J == nt) ? 1 : J, kSolveThreads, 0, stream>>>(dp, u, J, nt, xp, nrhs);
      ++*launches;
    }
  }
  return cudaGetLastError();
}

}  // namespace bdlu
