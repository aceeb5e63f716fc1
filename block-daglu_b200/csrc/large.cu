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
//   k_large_perm      final row order of each unit (and its inverse) from its
//                     pivot sequence
// Refactor with the stored pivot order (value-only refactor; the pivot order
// of KLU's klu_refactor is reused the same way):
//   k_scatter_large_perm  values scattered with rows already permuted
//   k_rpanel / k_rgemm
//                     64-column blocked LU without pivot search, trailing
//                     update split for one step of lookahead (see below)
// Solve (per level holding large units):
//   k_trsv_tiles<fwd/bwd>
//                     one CTA per 64-row tile, ticket-ordered, ready flags
//                     between tiles (see below)
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "device_util.cuh"
#include "large.h"
#include "tc_update.cuh"

namespace cg = cooperative_groups;

namespace bdlu {

namespace {

constexpr int kPT = 512;                  // panel kernel threads
constexpr int kPStride = kPanel + 1;      // shared-memory row stride of the panel (doubles)
constexpr int kClusterMaxCtas = 8;        // portable cluster size
constexpr int kPanelRowsMax = 640;        // panel rows one CTA holds (one per thread)
constexpr int kGT = 128;                  // GEMM output tile
constexpr int kGThreads = 256;
constexpr int kTile = 64;                 // solve tile
constexpr int kTS = kTile + 1;            // shared-memory row stride of a staged tile
constexpr int kSolveThreads = 256;

// ---------------------------------------------------------------------------
// Panel factorisation in a thread-block cluster.  Each thread of a CTA holds
// one panel row in registers (the column loop is unrolled, so register indices
// are static).  Row swaps are logical: a thread carries the current position
// of its row, and a swap of positions jj and p exchanges the two position
// registers; rows are written to their final positions at the end.  Per
// column: every warp finds its pivot candidate (largest |a|, ties to the
// smallest position: the reference's first strict maximum) and stages that
// row in shared memory; after one CTA barrier warp 0 pushes the CTA's
// candidate row, value and position to every CTA of the cluster (DSMEM);
// after one cluster barrier every warp combines the cluster's candidates
// lane-parallel, and each thread applies the rank-1 update to its row.
// Candidate buffers alternate by column parity, so one CTA and one cluster
// barrier per column suffice.  Multipliers use the reciprocal of the pivot, as
// LAPACK's dgetf2 does.
constexpr int kPanelThreads = 640;
constexpr int kPanelWarps = kPanelThreads / 32;

// Warp arg-max over (value >= 0, position): the largest value, ties to the
// smallest position.  Lanes with valid == false do not take part.  Returns the
// winning lane (or -1 when no lane is valid); best/bpos hold the winner.
__device__ __forceinline__ int warp_argmax(double val, int pos, bool valid, double& best, int& bpos) {
  double mx = valid ? val : -1.0;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  const bool tie = valid && val == mx;
  const int mn = __reduce_min_sync(0xffffffffu, tie ? pos : 0x7fffffff);
  const unsigned who = __ballot_sync(0xffffffffu, tie && pos == mn);
  best = mx;
  bpos = mn;
  return who ? __ffs(who) - 1 : -1;
}

__global__ void __launch_bounds__(kPanelThreads, 1) k_panel_cluster(DevPlan dp, int32_t k0, int32_t ubase,
                                                                    int32_t csize) {
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double cand[2][kClusterMaxCtas][kPanel + 2];
  __shared__ double wrow[kPanelWarps][kPanel];
  __shared__ double wbest[kPanelWarps];
  __shared__ int wpos[kPanelWarps];
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
  const bool has = r0 + tid < r1;
  int pos = has ? r0 + tid : m;             // current position of this thread's row
  double v[kPanel];
#pragma unroll
  for (int c = 0; c < kPanel; ++c) v[c] = (has && c < nb) ? A[static_cast<size_t>(r0 + tid) * m + k0 + c] : 0.0;
#pragma unroll
  for (int j = 0; j < kPanel; ++j) {
    if (j >= nb) break;
    const int jj = k0 + j;
    const int par = j & 1;
    {
      double best;
      int bpos;
      const int wl = warp_argmax(fabs(v[j]), pos, has && pos >= jj, best, bpos);
      if (wl == lane) {
#pragma unroll
        for (int c = 0; c < kPanel; ++c) wrow[warp][c] = v[c];
      }
      if (lane == 0) {
        wbest[warp] = best;
        wpos[warp] = (wl >= 0) ? bpos : m;
      }
    }
    __syncthreads();
    if (warp == 0) {
      const bool ok = lane < kPanelWarps && wpos[lane] != m;
      double best;
      int bpos;
      const int ww = warp_argmax(ok ? wbest[lane] : 0.0, ok ? wpos[lane] : m, ok, best, bpos);
      const double val = (ww >= 0) ? wrow[ww][lane] : 0.0;
      for (int q = 0; q < csize; ++q) {
        double* dst = cl.map_shared_rank(&cand[par][rank][0], q);
        dst[lane] = val;
        if (lane == 0) {
          dst[kPanel] = (ww >= 0) ? best : -1.0;
          dst[kPanel + 1] = static_cast<double>((ww >= 0) ? bpos : m);
        }
      }
    }
    cl.sync();
    double gbest;
    int gpos;
    const bool cok = lane < csize && cand[par][lane][kPanel] >= 0.0;
    const int owner = warp_argmax(cok ? cand[par][lane][kPanel] : 0.0,
                                  cok ? static_cast<int>(cand[par][lane][kPanel + 1]) : m, cok, gbest, gpos);
    if (owner < 0 || gbest == 0.0) {
      if (rank == 0 && tid == 0) report_failure(dp.status, u);
      cl.sync();
      return;
    }
    if (rank == 0 && tid == 0) dp.piv[s + jj] = gpos;
    // Logical swap of positions jj and gpos; the row now at jj is final.
    if (pos == jj) pos = gpos;
    else if (pos == gpos) pos = jj;
    if (has && pos > jj) {
      const double* U = cand[par][owner];
      const double l = v[j] * (1.0 / U[j]);
#pragma unroll
      for (int c = j + 1; c < kPanel; ++c) v[c] = fma(-l, U[c], v[c]);
      v[j] = l;
    }
  }
  if (has) {
#pragma unroll
    for (int c = 0; c < kPanel; ++c)
      if (c < nb) A[static_cast<size_t>(pos) * m + k0 + c] = v[c];
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
// columns right of the panel.  One thread per column.  The nb sequential swaps
// touch at most 2*nb rows; their net permutation is formed once per CTA in
// shared memory, so each thread loads every touched value before it stores.
__global__ void __launch_bounds__(kTrsmCols) k_swap_trsm_rm(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact) {
  __shared__ double L11[kPanel][kPanel + 1];
  __shared__ int rows[2 * kPanel];  // touched rows: k0..k0+nb-1 first, then the others
  __shared__ int src[2 * kPanel];   // new value of rows[q] = old value of rows[src[q]]
  __shared__ int s_cnt;
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
  if (threadIdx.x == 0) {
    int cnt = nb;
    for (int r = 0; r < nb; ++r) {
      rows[r] = k0 + r;
      src[r] = r;
    }
    // Simulate the swaps on positions: pos_of[row] via linear search (<= 64).
    for (int r = 0; r < nb; ++r) {
      const int p = dp.piv[s + k0 + r];
      if (p == k0 + r) continue;
      int qp = -1;
      for (int q = nb; q < cnt; ++q)
        if (rows[q] == p) qp = q;
      if (p < k0 + nb) qp = p - k0;
      if (qp < 0) {
        qp = cnt++;
        rows[qp] = p;
        src[qp] = qp;
      }
      const int t = src[r];
      src[r] = src[qp];
      src[qp] = t;
    }
    s_cnt = cnt;
  }
  __syncthreads();
  const int j = chunk * kTrsmCols + threadIdx.x;
  if (j >= m || (j >= k0 && j < k0 + nb)) return;
  const int cnt = s_cnt;
  // Gather every touched row's new value (all loads first), then store.
  double nv[2 * kPanel];
#pragma unroll
  for (int q = 0; q < 2 * kPanel; ++q)
    if (q < cnt) nv[q] = A[static_cast<size_t>(rows[src[q]]) * m + j];
#pragma unroll
  for (int q = kPanel; q < 2 * kPanel; ++q)
    if (q < cnt) A[static_cast<size_t>(rows[q]) * m + j] = nv[q];
  double x[kPanel];
#pragma unroll
  for (int r = 0; r < kPanel; ++r) x[r] = (r < nb) ? nv[r] : 0.0;
  if (j < k0 + nb) {
#pragma unroll
    for (int r = 0; r < kPanel; ++r)
      if (r < nb) A[static_cast<size_t>(k0 + r) * m + j] = x[r];
    return;
  }
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

// A22 -= L21 * U12 on row-major storage, the whole panel depth staged in
// shared memory.  All loads of the C tile precede its stores (a store may
// alias a later load, which would serialise the round trips).
constexpr int kAStride = kPanel + 1;   // As[i][q]
constexpr int kBStride = kGT + 4;      // Bs[q][j]
constexpr size_t kGemmSmem = (static_cast<size_t>(kGT) * kAStride + static_cast<size_t>(kPanel) * kBStride) * sizeof(double);
__global__ void __launch_bounds__(kGThreads, 1) k_gemm_rm(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact) {
  extern __shared__ double gsm[];
  double* As = gsm;
  double* Bs = gsm + kGT * kAStride;
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
  for (int t = tid; t < kGT * kPanel; t += kGThreads) {
    const int i = t / kPanel, q = t - i * kPanel;
    As[i * kAStride + q] = (q < nb && i0 + i < m) ? A[static_cast<size_t>(i0 + i) * m + k0 + q] : 0.0;
  }
  for (int t = tid; t < kPanel * kGT; t += kGThreads) {
    const int q = t / kGT, jj = t - q * kGT;
    Bs[q * kBStride + jj] = (q < nb && j0 + jj < m) ? A[static_cast<size_t>(k0 + q) * m + j0 + jj] : 0.0;
  }
  __syncthreads();
  double acc[8][8];
#pragma unroll
  for (int x = 0; x < 8; ++x)
#pragma unroll
    for (int y = 0; y < 8; ++y) acc[x][y] = 0.0;
#pragma unroll 4
  for (int q = 0; q < kPanel; ++q) {
    double av[8], bv[8];
#pragma unroll
    for (int x = 0; x < 8; ++x) av[x] = As[(ty + 16 * x) * kAStride + q];
#pragma unroll
    for (int y = 0; y < 8; ++y) bv[y] = Bs[q * kBStride + tx + 16 * y];
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
      for (int y = 0; y < 8; ++y) acc[x][y] = fma(av[x], bv[y], acc[x][y]);
  }
#pragma unroll
  for (int x = 0; x < 8; ++x) {
    const int i = i0 + ty + 16 * x;
    const double* row = A + static_cast<size_t>(min(i, m - 1)) * m;
#pragma unroll
    for (int y = 0; y < 8; ++y) {
      const int j = j0 + tx + 16 * y;
      acc[x][y] = (i < m && j < m) ? row[j] - acc[x][y] : 0.0;
    }
  }
#pragma unroll
  for (int x = 0; x < 8; ++x) {
    const int i = i0 + ty + 16 * x;
    if (i >= m) continue;
    double* row = A + static_cast<size_t>(i) * m;
#pragma unroll
    for (int y = 0; y < 8; ++y) {
      const int j = j0 + tx + 16 * y;
      if (j < m) row[j] = acc[x][y];
    }
  }
}

// Final row order of each large unit and its inverse: row k of the factor is
// local row perm[k], local row r sits at iperm[r].  The sequential swaps run
// on a shared-memory copy (one CTA per unit).
__global__ void k_large_perm(DevPlan dp, const int32_t* __restrict__ units) {
  extern __shared__ int32_t ord[];
  const int u = units[blockIdx.x];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  for (int k = threadIdx.x; k < m; k += blockDim.x) ord[k] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < m; ++k) {
      const int p = dp.piv[s + k];
      if (p != k) {
        const int32_t tmp = ord[k];
        ord[k] = ord[p];
        ord[p] = tmp;
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    dp.lperm[s + k] = ord[k];
    dp.liperm[s + ord[k]] = k;
  }
}

// Value scatter of large units into their slots with rows already in the
// stored pivot order (refactor with the previous pivot sequence).
__global__ void k_scatter_large_perm(DevPlan dp, const double* __restrict__ vals, const int32_t* __restrict__ units) {
  const int u = units[blockIdx.y];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  double* A = dp.lu + dp.lu_off[u];
  for (int64_t e = dp.dent_ptr[u] + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < dp.dent_ptr[u + 1];
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int pos = dp.dent_pos[e];
    const int r = pos / m, c = pos - (pos / m) * m;
    A[static_cast<size_t>(dp.liperm[s + r]) * m + c] = vals[dp.dent_src[e]];
  }
}

// ---------------------------------------------------------------------------
// Triangular solves of large units without a launch per tile.  The unit's
// rows are cut into kTile-row tiles; each CTA takes a ticket (atomic counter,
// so every tile with a smaller ticket belongs to a CTA that is already
// running) and solves one tile: forward sweeps take the unit's tiles in
// order, backward sweeps in reverse.  A CTA forms its rows' right-hand sides
// (forward: b - A_cpl x through the unit's final row order; backward: the
// forward result), then for every finished tile J it stages the kTile x kTile
// block (I, J) of the factor in shared memory, waits for tile J's ready flag
// and accumulates block(I, J) * x_J; finally it subtracts, solves its
// diagonal triangle (one warp per right-hand side, unknowns in registers,
// shuffle broadcasts), stores x_I and publishes its flag.  Flags count the
// finished right-hand-side passes.  Every wait is bounded: a wait that runs
// out records kFailSync in the status word and publishes kAbortFlag, so the
// tiles behind it stop too.
// Right-hand sides per pass: kernels exist for 8 and 16 (the 16-wide one
// reads each factor block once for up to 16 right-hand sides; the 8-wide one
// keeps fewer registers and a shorter tile chain for few right-hand sides).
constexpr int32_t kAbortFlag = 1 << 30;
constexpr int kTLoads = kTile * kTile / kSolveThreads;  // block entries each thread stages
template <int kRC>
constexpr size_t trsv_smem() {
  return (static_cast<size_t>(kTile) * kTS + 2 * static_cast<size_t>(kTile) * kRC) * sizeof(double);
}

// Waits until *f >= need, at most `limit` polls (DevPlan::wait_limit).
__device__ __forceinline__ bool wait_ready(const int32_t* f, int32_t need, int32_t limit) {
  for (int it = 0; it < limit; ++it) {
    const int32_t v = *reinterpret_cast<const volatile int32_t*>(f);
    if (v >= need) {
      __threadfence();
      return v < kAbortFlag;
    }
    if (it > 64) __nanosleep(128);
  }
  return false;
}

// Entries (i, c) of the kTile x kTile block at (t0, j0) that thread `tid`
// stages: e = tid + kSolveThreads * k, i = e / kTile, c = e % kTile.
__device__ __forceinline__ void load_block(const double* __restrict__ LU, int m, int t0, int w, int j0, int jw,
                                           int tid, double (&v)[kTLoads]) {
#pragma unroll
  for (int k = 0; k < kTLoads; ++k) {
    const int e = tid + kSolveThreads * k;
    const int i = e / kTile, c = e - i * kTile;
    v[k] = (i < w && c < jw) ? __ldg(LU + static_cast<size_t>(t0 + i) * m + j0 + c) : 0.0;
  }
}

template <bool kFwd, int kRC>
__global__ void __launch_bounds__(kSolveThreads, 2) k_trsv_tiles(DevPlan dp, const int32_t* __restrict__ units,
                                                              const int32_t* __restrict__ tile0, int32_t count,
                                                              int32_t* ticket, int32_t* ready,
                                                              const double* __restrict__ rhs, int32_t ldr,
                                                              double* __restrict__ xp,
                                                              const int32_t* __restrict__ nrhs_p) {
  const int32_t nrhs = *nrhs_p;
  extern __shared__ double tsm_d[];
  double* Ts = tsm_d;                  // factor block; also the partial-sum exchange
  double* xs = Ts + kTile * kTS;       // this tile's unknowns [i * kRC + c]
  double* xj = xs + kTile * kRC;       // finished tile's unknowns
  __shared__ int s_tk, s_ok;
  __shared__ double rdg[kTile];        // backward sweep: reciprocals of the diagonal block's pivots
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tk = atomicAdd(ticket, 1);
  __syncthreads();
  const int tk = s_tk;
  const int base0 = tile0[0];
  int q = 0;
  while (q + 1 < count && tile0[q + 1] - base0 <= tk) ++q;
  const int u = units[q];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int n = dp.n;
  const int nt = (m + kTile - 1) / kTile;
  const int kidx = tk - (tile0[q] - base0);
  const int I = kFwd ? kidx : nt - 1 - kidx;
  int32_t* rdy = ready + tile0[q];
  const int t0 = I * kTile, w = min(kTile, m - t0);
  const double* LU = dp.lu + dp.lu_off[u];
  const int r = tid & (kTile - 1), g = tid / kTile;  // row of the tile, 16-column group
  constexpr int kGroups = kSolveThreads / kTile;
  constexpr int kGCols = kTile / kGroups;
  constexpr int kWarps = kSolveThreads / 32;
  for (int c0 = 0; c0 < nrhs; c0 += kRC) {
    const int nc = min(kRC, nrhs - c0);
    const int32_t need = c0 / kRC + 1;
    if (kFwd) {
      for (int i = warp; i < w; i += kWarps) {
        const int rr = s + dp.lperm[s + t0 + i];
        const int p0 = dp.cpl_ptr[rr], p1 = dp.cpl_ptr[rr + 1];
        for (int c = 0; c < nc; ++c) {
          const double* xc = xp + static_cast<size_t>(c0 + c) * n;
          double acc = 0.0;
          for (int qq = p0 + lane; qq < p1; qq += 32) acc = fma(dp.cpl_val[qq], xc[dp.cpl_col[qq]], acc);
          acc = warp_sum(acc);
          if (lane == 0) xs[i * kRC + c] = rhs[dp.P[rr] + static_cast<size_t>(c0 + c) * ldr] - acc;
        }
      }
    } else {
      for (int e = tid; e < w * nc; e += kSolveThreads) {
        const int i = e / nc, c = e - i * nc;
        xs[i * kRC + c] = __ldcg(xp + static_cast<size_t>(c0 + c) * n + s + t0 + i);
      }
    }
    double acc[kRC];
#pragma unroll
    for (int c = 0; c < kRC; ++c) acc[c] = 0.0;
    const int jn = kFwd ? I : nt - 1 - I;
    bool ok = true;
    // The next block is loaded into registers while the current one is
    // used, so the loads overlap the arithmetic and the flag wait.
    // nxt: the next coupling block, and after the last one the diagonal
    // block, so the triangle's operands are in flight before they are needed.
    double nxt[kTLoads];
    if (jn > 0) {
      const int J = kFwd ? 0 : nt - 1;
      load_block(LU, m, t0, w, J * kTile, min(kTile, m - J * kTile), tid, nxt);
    } else {
      load_block(LU, m, t0, w, t0, w, tid, nxt);
    }
    for (int jk = 0; jk < jn; ++jk) {
      const int J = kFwd ? jk : nt - 1 - jk;
      const int j0 = J * kTile, jw = min(kTile, m - j0);
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kTLoads; ++k) {
        const int e = tid + kSolveThreads * k;
        const int i = e / kTile, c = e - i * kTile;
        Ts[i * kTS + c] = nxt[k];
      }
      if (jk + 1 < jn) {
        const int J2 = kFwd ? jk + 1 : nt - 2 - jk;
        load_block(LU, m, t0, w, J2 * kTile, min(kTile, m - J2 * kTile), tid, nxt);
      } else {
        load_block(LU, m, t0, w, t0, w, tid, nxt);
      }
      if (tid == 0) s_ok = wait_ready(rdy + J, need, dp.wait_limit) ? 1 : 0;
      __syncthreads();
      if (!s_ok) {
        ok = false;
        break;
      }
#pragma unroll
      for (int k = 0; k < kTile * kRC / kSolveThreads; ++k) {
        const int e = tid + kSolveThreads * k;
        const int jj = e / kRC, c = e - jj * kRC;
        xj[e] = (jj < jw && c < nc) ? __ldcg(xp + static_cast<size_t>(c0 + c) * n + s + j0 + jj) : 0.0;
      }
      __syncthreads();
#pragma unroll 1
      for (int k = 0; k < kGCols; ++k) {
        const int cc = g * kGCols + k;
        const double t = Ts[r * kTS + cc];
        const double2* xv = reinterpret_cast<const double2*>(xj + cc * kRC);
#pragma unroll
        for (int c2 = 0; c2 < kRC / 2; ++c2) {
          const double2 x2 = xv[c2];
          acc[2 * c2] = fma(t, x2.x, acc[2 * c2]);
          acc[2 * c2 + 1] = fma(t, x2.y, acc[2 * c2 + 1]);
        }
      }
    }
    if (!ok) {
      if (tid == 0) {
        atomicCAS(dp.status, 0, kFailSync);
        atomicExch(rdy + I, kAbortFlag);
      }
      return;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kRC; ++c) Ts[(g * kTile + r) * kRC + c] = acc[c];
    __syncthreads();
    for (int e = tid; e < w * nc; e += kSolveThreads) {
      const int i = e / nc, c = e - i * nc;
      double sum = 0.0;
#pragma unroll
      for (int gg = 0; gg < kGroups; ++gg) sum += Ts[(gg * kTile + i) * kRC + c];
      xs[i * kRC + c] -= sum;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kTLoads; ++k) {
      const int e = tid + kSolveThreads * k;
      const int i = e / kTile, c = e - i * kTile;
      Ts[i * kTS + c] = nxt[k];
      // The backward sweep multiplies by the pivots' reciprocals, formed
      // here in parallel: no division on its dependent chain.
      if (!kFwd && i == c) rdg[i] = 1.0 / nxt[k];
    }
    __syncthreads();
    // Each warp sweeps right-hand side `warp` and, when more than kWarps are
    // in this pass, also warp + kWarps alongside (their chains overlap).
    if (warp < nc) {
      const int ca = warp, cb = warp + kWarps;
      const bool two = kRC > kWarps && cb < nc;
      double a0 = (lane < w) ? xs[lane * kRC + ca] : 0.0;
      double b0 = (lane + 32 < w) ? xs[(lane + 32) * kRC + ca] : 0.0;
      double a1 = (two && lane < w) ? xs[lane * kRC + cb] : 0.0;
      double b1 = (two && lane + 32 < w) ? xs[(lane + 32) * kRC + cb] : 0.0;
      if (two) {
        if (kFwd) {
          for (int rr = 0; rr < w; ++rr) {
            const double x0 = __shfl_sync(0xffffffffu, rr < 32 ? a0 : b0, rr & 31);
            const double x1 = __shfl_sync(0xffffffffu, rr < 32 ? a1 : b1, rr & 31);
            if (lane > rr && lane < w) {
              const double t = Ts[lane * kTS + rr];
              a0 = fma(-t, x0, a0);
              a1 = fma(-t, x1, a1);
            }
            if (lane + 32 > rr && lane + 32 < w) {
              const double t = Ts[(lane + 32) * kTS + rr];
              b0 = fma(-t, x0, b0);
              b1 = fma(-t, x1, b1);
            }
          }
        } else {
          for (int rr = w - 1; rr >= 0; --rr) {
            const double rd = rdg[rr];
            const double x0 = __shfl_sync(0xffffffffu, rr < 32 ? a0 : b0, rr & 31) * rd;
            const double x1 = __shfl_sync(0xffffffffu, rr < 32 ? a1 : b1, rr & 31) * rd;
            if (lane == rr) {
              a0 = x0;
              a1 = x1;
            }
            if (lane + 32 == rr) {
              b0 = x0;
              b1 = x1;
            }
            if (lane < rr) {
              const double t = Ts[lane * kTS + rr];
              a0 = fma(-t, x0, a0);
              a1 = fma(-t, x1, a1);
            }
            if (lane + 32 < rr) {
              const double t = Ts[(lane + 32) * kTS + rr];
              b0 = fma(-t, x0, b0);
              b1 = fma(-t, x1, b1);
            }
          }
        }
      } else if (kFwd) {
        for (int rr = 0; rr < w; ++rr) {
          const double x0 = __shfl_sync(0xffffffffu, rr < 32 ? a0 : b0, rr & 31);
          if (lane > rr && lane < w) a0 = fma(-Ts[lane * kTS + rr], x0, a0);
          if (lane + 32 > rr && lane + 32 < w) b0 = fma(-Ts[(lane + 32) * kTS + rr], x0, b0);
        }
      } else {
        for (int rr = w - 1; rr >= 0; --rr) {
          const double x0 = __shfl_sync(0xffffffffu, rr < 32 ? a0 : b0, rr & 31) * rdg[rr];
          if (lane == rr) a0 = x0;
          if (lane + 32 == rr) b0 = x0;
          if (lane < rr) a0 = fma(-Ts[lane * kTS + rr], x0, a0);
          if (lane + 32 < rr) b0 = fma(-Ts[(lane + 32) * kTS + rr], x0, b0);
        }
      }
      double* xo = xp + static_cast<size_t>(c0 + ca) * n + s + t0;
      if (lane < w) xo[lane] = a0;
      if (lane + 32 < w) xo[lane + 32] = b0;
      if (two) {
        double* xo1 = xp + static_cast<size_t>(c0 + cb) * n + s + t0;
        if (lane < w) xo1[lane] = a1;
        if (lane + 32 < w) xo1[lane + 32] = b1;
      }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(rdy + I, need);
  }
}

// ---------------------------------------------------------------------------
// Value-only refactor of large units with the stored pivot order: steps of
// kRPanel (64) columns.  Per step:
//   k_rpanel  L21 = A21 U11^{-1} (row chunks) and U12 = L11^{-1} A12 (column
//             chunks); every CTA first factors the 64 x 64 diagonal block
//             without pivot search (diag_lu: rows in registers, one barrier
//             per column), then solves its strip by substitution (four
//             threads per line, entries in registers, no barriers).  A zero
//             or non-finite pivot flags the unit for full pivoting.
//   k_rgemm   A22 -= L21 U12, K = 64, 128 x 64 tiles, 4 x 8 accumulators per
//             thread, two CTAs per SM.  Part "a" updates tile row 0 and tile
//             column 0, which hold the next step's strips, and places the
//             factored diagonal block; part "b" updates the rest.
// Part b of step k runs on a second stream beside the next step's k_rpanel
// and part a (depth-1 lookahead); the regions are disjoint: the next step
// reads and writes rows/columns [base, base + 64) only, part b writes rows
// >= base + 128 and columns >= base + 64.
constexpr int kRP = kRPanel;
constexpr int kRS = kRP + 1;
constexpr int kRThreads = 256;
constexpr int kPadRow = 72;    // padded 64-entry row: quarter q at offset 18q (16-byte loads, no conflicts)
constexpr int kRAS = kRP + 1;  // As row stride in k_rgemm
constexpr size_t kRGemmSmem = (static_cast<size_t>(kRTileM) * kRAS + static_cast<size_t>(kRP) * kRTileN) * sizeof(double);

// Reciprocal of a pivot.  A plain FP64 division: on this part it has about
// 80 cycles of latency, less than Newton's iteration from the single-
// precision reciprocal (about 200), and it is correctly rounded.
__device__ __forceinline__ double pivot_rcp(double d) { return 1.0 / d; }

// LU without pivot search of the kRP x kRP diagonal block at (k0, k0) of a
// row-major m x m unit into shared memory D (stride kRS; rows/columns past nb
// padded with the identity).  Thread t keeps 16 entries of row i = t / 4 in
// registers (columns (t % 4) + 4q); the pivot row and its reciprocal go
// through a double-buffered shared row, one barrier per column; the row's
// multiplier comes from the lane that holds column j by shuffle.  The owner
// of the next pivot row publishes it right after its own update, so the
// dependent chain per column is barrier, shuffle, multiply, update, store.
// RowsLU<JQ> handles columns 4JQ .. 4JQ+3 (register indices compile-time).
template <int JQ>
struct RowsLU {
  static __device__ __forceinline__ void run(double (&v)[16], double (*prow)[kRP], double* rinv, int i, int sub,
                                             int lane) {
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
      const int j = 4 * JQ + s;
      __syncthreads();
      const double* pr = prow[j & 1];
      const double r = rinv[j & 1];
      const double a = __shfl_sync(0xffffffffu, v[JQ], (lane & ~3) | s);
      if (i > j) {
        const double l = a * r;
        if (sub == s) v[JQ] = l;
        if (sub > s) v[JQ] = fma(-l, pr[sub + 4 * JQ], v[JQ]);
#pragma unroll
        for (int q = JQ + 1; q < 16; ++q) v[q] = fma(-l, pr[sub + 4 * q], v[q]);
      }
      if (i == j + 1) {
        // Row j + 1 is final: publish it and its pivot's reciprocal (the
        // pivot is column j + 1: register JQ, or JQ + 1 after s = 3).
#pragma unroll
        for (int q = JQ; q < 16; ++q) prow[(j + 1) & 1][sub + 4 * q] = v[q];
        if (sub == ((j + 1) & 3)) rinv[(j + 1) & 1] = pivot_rcp(s == 3 ? v[JQ < 15 ? JQ + 1 : 15] : v[JQ]);
      }
    }
    RowsLU<JQ + 1>::run(v, prow, rinv, i, sub, lane);
  }
};
template <>
struct RowsLU<16> {
  static __device__ __forceinline__ void run(double (&)[16], double (*)[kRP], double*, int, int, int) {}
};
static_assert(kRP == 64 && kRThreads == 256, "diag_lu: four threads per row, 16 entries each");

__device__ void diag_lu(double* D, const double* A, int m, int k0, int nb) {
  __shared__ double prow[2][kRP];
  __shared__ double rinv[2];
  const int tid = threadIdx.x, lane = tid & 31;
  const int i = tid >> 2, sub = tid & 3;
  double v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int c = sub + 4 * q;
    v[q] = (i < nb && c < nb) ? __ldcg(A + static_cast<size_t>(k0 + i) * m + k0 + c) : (i == c ? 1.0 : 0.0);
  }
  if (i == 0) {
#pragma unroll
    for (int q = 0; q < 16; ++q) prow[0][sub + 4 * q] = v[q];
    if (sub == 0) rinv[0] = pivot_rcp(v[0]);
  }
  RowsLU<0>::run(v, prow, rinv, i, sub, lane);
#pragma unroll
  for (int q = 0; q < 16; ++q) D[i * kRS + sub + 4 * q] = v[q];
  __syncthreads();
}

// Strip entries of one thread: line = tid / 4 of the strip at o0 (a row of
// L21 for a row strip, a column of U12 for a column strip), entries
// 16qq .. 16qq+15 with qq = tid % 4; zero past nb or past the strip's w lines.
__device__ __forceinline__ void strip_load(const double* A, int m, int k0, int nb, int o0, int w, bool rowc,
                                           double (&x)[16]) {
  const int tid = threadIdx.x, line = tid >> 2, qq = tid & 3;
  const bool live = line < w;
#pragma unroll
  for (int t = 0; t < 16; ++t) {
    const int q = 16 * qq + t;
    double v = 0.0;
    if (live && q < nb)
      v = rowc ? __ldcg(A + static_cast<size_t>(o0 + line) * m + k0 + q)
               : __ldcg(A + static_cast<size_t>(k0 + q) * m + o0 + line);
    x[t] = v;
  }
}

// Solves one strip against the factored diagonal block D (stride kRS,
// identity past nb) and stores it: row strips x U11 = a, column strips
// L11 x = b.  Thread (line, quarter qq) holds its 16 entries in x; the
// factor's row j of U (column j of L) is staged padded in shared memory T
// (kRP x kPadRow), the pivot reciprocals in rd.
__device__ __forceinline__ void strip_solve(const double* D, double* T, double* rd, double* A, int m, int k0,
                                            int nb, int o0, int w, bool rowc, double (&x)[16]) {
  const int tid = threadIdx.x, lane = tid & 31;
  const int line = tid >> 2, qq = tid & 3;
  // T[j][18q + t]: rows: U[j][16q + t]; columns: L[16q + t][j].
  for (int e = tid; e < kRP * kRP; e += kRThreads) {
    const int j = e / kRP, c = e - j * kRP;
    T[j * kPadRow + 18 * (c >> 4) + (c & 15)] = rowc ? D[j * kRS + c] : D[c * kRS + j];
  }
  if (rowc && tid < kRP) rd[tid] = 1.0 / D[tid * kRS + tid];
  __syncthreads();
  const int src = (lane & ~3);
  for (int jq = 0; jq < 4; ++jq) {
#pragma unroll
    for (int jt = 0; jt < 16; ++jt) {
      const int j = 16 * jq + jt;
      if (rowc && qq == jq) x[jt] *= rd[j];
      const double xj = __shfl_sync(0xffffffffu, x[jt], src | jq);
      const double2* tv = reinterpret_cast<const double2*>(T + j * kPadRow + 18 * qq);
#pragma unroll
      for (int t2 = 0; t2 < 8; ++t2) {
        const double2 f = tv[t2];
        if (qq > jq || (qq == jq && 2 * t2 > jt)) x[2 * t2] = fma(-xj, f.x, x[2 * t2]);
        if (qq > jq || (qq == jq && 2 * t2 + 1 > jt)) x[2 * t2 + 1] = fma(-xj, f.y, x[2 * t2 + 1]);
      }
    }
  }
  if (line < w) {
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int q = 16 * qq + t;
      if (q < nb) {
        if (rowc) A[static_cast<size_t>(o0 + line) * m + k0 + q] = x[t];
        else A[static_cast<size_t>(k0 + q) * m + o0 + line] = x[t];
      }
    }
  }
}

// Panel of one step, fused: every CTA of a unit factors the diagonal block
// itself (diag_lu, redundantly: the CTAs run side by side, so the
// factorisation adds no time to the step's dependent chain), then solves its
// strip (strip_solve).  Row chunks: rows o0 .. o0+w of L21; column chunks:
// columns o0 .. o0+w of U12.  Chunk 0 checks the pivots and leaves the
// factored block in dp.dscratch (slot = the unit's index in the step); the
// step's update (part a) copies it into the arena once every CTA here has
// read the unfactored block.  A unit with nothing left to solve gets one CTA
// for that.
constexpr size_t kRPanelSmem =
    (static_cast<size_t>(kRP) * kRS + static_cast<size_t>(kRP) * kPadRow + kRP) * sizeof(double);

__global__ void __launch_bounds__(kRThreads) k_rpanel(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact) {
  extern __shared__ double psm[];
  double* D = psm;                    // kRP x kRS
  double* T = D + kRP * kRS;          // kRP x kPadRow (16-byte aligned: kRP * kRS is even)
  double* rd = T + kRP * kPadRow;     // kRP
  int a = 0;
  while (a + 1 < nact && dp.rstep_strip_pref[ubase + a + 1] <= static_cast<int>(blockIdx.x)) ++a;
  const int u = dp.rstep_unit[ubase + a];
  const int ch = blockIdx.x - dp.rstep_strip_pref[ubase + a];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kRP, m - k0);
  const int base = k0 + nb;
  const int chunks = (m - base + kRP - 1) / kRP;
  const bool rowc = ch < chunks;
  const int o0 = base + (rowc ? ch : ch - chunks) * kRP;
  const int w = max(0, min(kRP, m - o0));
  double* A = dp.lu + dp.lu_off[u];
  const int tid = threadIdx.x;
  // The strip's entries go to registers first (their loads overlap the LU).
  double x[16];
  strip_load(A, m, k0, nb, o0, w, rowc, x);
  diag_lu(D, A, m, k0, nb);
  __syncthreads();
  if (ch == 0) {
    if (tid < nb) {
      const double d = D[tid * kRS + tid];
      if (!(fabs(d) > 0.0) || !isfinite(d)) {
        if (atomicCAS(dp.status, 0, kFailReusedPivot) == 0) dp.status[1] = u;
      }
    }
    double* out = dp.dscratch + static_cast<size_t>(a) * kRP * kRP;
#pragma unroll 4
    for (int e = tid; e < kRP * kRP; e += kRThreads) out[e] = D[(e / kRP) * kRS + (e % kRP)];
  }
  strip_solve(D, T, rd, A, m, k0, nb, o0, w, rowc, x);
}

// Copies the factored diagonal block of step k0 (left by k_rpanel in
// dp.dscratch slot a) into the arena; run by the first part-a CTA of a unit.
__device__ __forceinline__ void place_diag(const DevPlan& dp, double* A, int m, int k0, int nb, int a) {
  const double* src = dp.dscratch + static_cast<size_t>(a) * kRP * kRP;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, c = e - i * nb;
    A[static_cast<size_t>(k0 + i) * m + k0 + c] = src[i * kRP + c];
  }
}

// C -= L U for the kRTileM x kRTileN tile at (i0, j0) of a row-major m x m
// unit: L = columns k0 .. k0+nb of rows i0.., U = rows k0 .. k0+nb of
// columns j0.. (rows and columns past m skipped).  rsm: kRGemmSmem bytes.
// Thread (ty, tx) accumulates rows i0 + 4ty + i, columns j0 + 8b + tx.
__device__ __forceinline__ void rgemm_tile(double* rsm, double* A, int m, int k0, int nb, int i0, int j0) {
  double* As = rsm;                      // kRTileM x kRAS
  double* Bs = rsm + kRTileM * kRAS;     // kRP x kRTileN
  const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
#pragma unroll 8
  for (int e = tid; e < kRTileM * kRP; e += kRThreads) {
    const int r = e / kRP, q = e - r * kRP;
    As[r * kRAS + q] = (i0 + r < m && q < nb) ? __ldcg(A + static_cast<size_t>(i0 + r) * m + k0 + q) : 0.0;
  }
#pragma unroll 8
  for (int e = tid; e < kRP * kRTileN; e += kRThreads) {
    const int q = e / kRTileN, c = e - q * kRTileN;
    Bs[e] = (q < nb && j0 + c < m) ? __ldcg(A + static_cast<size_t>(k0 + q) * m + j0 + c) : 0.0;
  }
  __syncthreads();
  double acc[4][8];
  const bool cin = j0 + 7 * 8 + tx < m;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = i0 + ty * 4 + i;
    const double* crow = A + static_cast<size_t>(r) * m + j0 + tx;
#pragma unroll
    for (int b = 0; b < 8; ++b)
      acc[i][b] = (r < m && (cin || j0 + b * 8 + tx < m)) ? __ldcg(crow + b * 8) : 0.0;
  }
#pragma unroll 2
  for (int k = 0; k < kRP; ++k) {
    double x[4], y[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) x[i] = As[(ty * 4 + i) * kRAS + k];
#pragma unroll
    for (int b = 0; b < 8; ++b) y[b] = Bs[k * kRTileN + b * 8 + tx];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int b = 0; b < 8; ++b) acc[i][b] = fma(-x[i], y[b], acc[i][b]);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = i0 + ty * 4 + i;
    double* crow = A + static_cast<size_t>(r) * m + j0 + tx;
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (r < m && (cin || j0 + b * 8 + tx < m)) crow[b * 8] = acc[i][b];
  }
}

__global__ void __launch_bounds__(kRThreads, 2) k_rgemm(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact,
                                                        int32_t part) {
  extern __shared__ double rsm[];
  const int32_t* pref = part ? dp.rstep_gb_pref : dp.rstep_ga_pref;
  int a = 0;
  while (a + 1 < nact && pref[ubase + a + 1] <= static_cast<int>(blockIdx.x)) ++a;
  const int u = dp.rstep_unit[ubase + a];
  const int t = blockIdx.x - pref[ubase + a];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kRP, m - k0);
  const int base = k0 + nb;
  const int rest = m - base;
  const int ntj = (rest + kRTileN - 1) / kRTileN;
  if (part == 0 && t == 0) {
    place_diag(dp, dp.lu + dp.lu_off[u], m, k0, nb, a);
    if (rest <= 0) return;
  }
  int ti, tj;
  if (part == 0) {
    if (t < ntj) {
      ti = 0;
      tj = t;
    } else {
      ti = t - ntj + 1;
      tj = 0;
    }
  } else {
    ti = 1 + t / (ntj - 1);
    tj = 1 + t % (ntj - 1);
  }
  rgemm_tile(rsm, dp.lu + dp.lu_off[u], m, k0, nb, base + ti * kRTileM, base + tj * kRTileN);
}

// ---------------------------------------------------------------------------
// Value-only refactor as one persistent kernel over the tile task graph of
// build_rtasks (plan.h): tiles kRP x kRP, tasks D(k), L(i, k), U(k, j) and
// G(i, j, k) (row tiles i, i + 1 of tile column j), in the list's order.
// A tile's version word counts the steps applied to it; a task waits for
//   D(k):       ver(k, k) >= k
//   L(i, k):    ver(k, k) >= k + 1 and ver(i, k) >= k
//   U(k, j):    ver(k, k) >= k + 1 and ver(k, j) >= k
//   G(i, j, k): ver(i, k), ver(i + 1, k), ver(k, j) >= k + 1 and
//               ver(i, j), ver(i + 1, j) >= k
// and sets its output tiles to k + 1.  CTAs take tasks by ticket (word 0 of
// the array, an atomic counter).  A task waits only for tasks earlier in the
// list, whose tickets running CTAs took, so the smallest unfinished ticket
// always progresses: nothing assumes that the CTAs are co-resident.  Waits
// are bounded (wait_ready); one that runs out records kFailRefactorSync and
// publishes kAbortFlag on the task's outputs, so that its dependents stop at
// once.  Matrix entries are read with ld.global.cg (from L2): a line that
// another SM rewrote is never served stale from this SM's L1.  The
// arithmetic per tile is that of k_rpanel / k_rgemm (diag_lu, strip_solve,
// rgemm_tile), so both schedules give bit-identical factors.
static_assert(kRTileM == 2 * kRP && kRTileN == kRP, "an update task covers two row tiles of one tile column");
constexpr size_t kRDagSmem = kRGemmSmem > kRPanelSmem ? kRGemmSmem : kRPanelSmem;

__device__ __forceinline__ void rdag_publish(int32_t* f, int32_t v) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicExch(f, v);
}

__global__ void __launch_bounds__(kRThreads, 2) k_rdag(DevPlan dp, const int4* __restrict__ tasks, int32_t ntasks,
                                                       int32_t* __restrict__ words) {
  extern __shared__ double gsm[];
  __shared__ int s_tk, s_ok;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_tk = atomicAdd(words, 1);
    __syncthreads();
    const int tk = s_tk;
    if (tk >= ntasks) break;
    const int4 tsk = __ldg(tasks + tk);
    const int u = tsk.x, k = tsk.y, i = tsk.z >> 16, j = tsk.z & 0xffff;
    int32_t* ver = words + tsk.w;
    const int s = dp.ustart[u];
    const int m = dp.ustart[u + 1] - s;
    const int nt = (m + kRP - 1) / kRP;
    double* A = dp.lu + dp.lu_off[u];
    const int k0 = k * kRP, nb = min(kRP, m - k0);
    int32_t* kk = ver + k * nt + k;
    if (i == k && j == k) {
      // D(k): factor tile (k, k) in place.
      if (tid == 0) s_ok = wait_ready(kk, k, dp.wait_limit);
      __syncthreads();
      if (s_ok) {
        double* D = gsm;
        diag_lu(D, A, m, k0, nb);
        if (tid < nb) {
          const double d = D[tid * kRS + tid];
          if (!(fabs(d) > 0.0) || !isfinite(d)) {
            if (atomicCAS(dp.status, 0, kFailReusedPivot) == 0) dp.status[1] = u;
          }
        }
        for (int e = tid; e < nb * nb; e += kRThreads) {
          const int r = e / nb, c = e - r * nb;
          A[static_cast<size_t>(k0 + r) * m + k0 + c] = D[r * kRS + c];
        }
        rdag_publish(kk, k + 1);
      } else if (tid == 0) {
        atomicCAS(dp.status, 0, kFailRefactorSync);
        atomicExch(kk, kAbortFlag);
      }
    } else if (i == k || j == k) {
      // L(i, k) (row strip) or U(k, j) (column strip).
      const bool rowc = j == k;
      const int o = rowc ? i : j;
      int32_t* out = rowc ? ver + i * nt + k : ver + k * nt + j;
      if (tid == 0) s_ok = wait_ready(kk, k + 1, dp.wait_limit) && wait_ready(out, k, dp.wait_limit);
      __syncthreads();
      if (s_ok) {
        double* D = gsm;                   // kRP x kRS
        double* T = D + kRP * kRS;         // kRP x kPadRow
        double* rd = T + kRP * kPadRow;    // kRP
        const int o0 = o * kRP, w = min(kRP, m - o0);
        double x[16];
        strip_load(A, m, k0, nb, o0, w, rowc, x);
        for (int e = tid; e < kRP * kRP; e += kRThreads) {
          const int r = e / kRP, c = e - r * kRP;
          D[r * kRS + c] = (r < nb && c < nb) ? __ldcg(A + static_cast<size_t>(k0 + r) * m + k0 + c)
                                              : (r == c ? 1.0 : 0.0);
        }
        __syncthreads();
        strip_solve(D, T, rd, A, m, k0, nb, o0, w, rowc, x);
        rdag_publish(out, k + 1);
      } else if (tid == 0) {
        atomicCAS(dp.status, 0, kFailRefactorSync);
        atomicExch(out, kAbortFlag);
      }
    } else {
      // G(i, j, k): row tiles i, i + 1 of tile column j.
      const bool two = i + 1 < nt;
      int32_t* c0 = ver + i * nt + j;
      int32_t* c1 = two ? c0 + nt : c0;
      if (tid == 0) {
        const int32_t lim = dp.wait_limit;
        bool ok = wait_ready(ver + i * nt + k, k + 1, lim) && wait_ready(ver + k * nt + j, k + 1, lim) &&
                  wait_ready(c0, k, lim);
        if (two) ok = ok && wait_ready(ver + (i + 1) * nt + k, k + 1, lim) && wait_ready(c1, k, lim);
        s_ok = ok;
      }
      __syncthreads();
      if (s_ok) {
        rgemm_tile(gsm, A, m, k0, nb, i * kRP, j * kRP);
        __threadfence();
        __syncthreads();
        if (tid == 0) {
          atomicExch(c0, k + 1);
          if (two) atomicExch(c1, k + 1);
        }
      } else if (tid == 0) {
        atomicCAS(dp.status, 0, kFailRefactorSync);
        atomicExch(c0, kAbortFlag);
        if (two) atomicExch(c1, kAbortFlag);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Tensor-core trailing updates for the mixed-precision route (tc_update.cuh):
// tcgen05.mma kind::tf32 with the accumulator in tensor memory, operands
// rounded to TF32 from the FP64 storage while staged in shared memory.  With
// split3 each operand is split a = hi + lo (both TF32, lo = tf32(a - hi)) and
// C -= hi hi + hi lo + lo hi ("3xTF32", a published way to reach about FP32
// accuracy on TF32 units).  Panels, pivot search and storage stay FP64; FP64
// iterative refinement recovers the accuracy.  A CTA allocates its
// accumulator columns only once it knows it has a tile, and frees them on
// every path out.
__device__ __forceinline__ uint8_t* tc_align(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~static_cast<uintptr_t>(1023));
}

constexpr size_t kRTcSmem = tc_smem_bytes<kRP, kRTileN>();
constexpr size_t kGTcSmem = tc_smem_bytes<kPanel, kGT>();
static_assert(kRTileM == kTcM && kGT == kTcM && kRThreads == kTcThreads, "tile shapes of the tensor-core update");

// Value-only refactor update (k_rgemm's 128 x 64 tiles, K = 64).
__global__ void __launch_bounds__(kTcThreads) k_rgemm_tc(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact,
                                                         int32_t part, int32_t split3) {
  extern __shared__ uint8_t tc_dyn_r[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  const int32_t* pref = part ? dp.rstep_gb_pref : dp.rstep_ga_pref;
  int a = 0;
  while (a + 1 < nact && pref[ubase + a + 1] <= static_cast<int>(blockIdx.x)) ++a;
  const int u = dp.rstep_unit[ubase + a];
  const int t = blockIdx.x - pref[ubase + a];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int nb = min(kRP, m - k0);
  const int base = k0 + nb;
  const int rest = m - base;
  const int ntj = (rest + kRTileN - 1) / kRTileN;
  if (part == 0 && t == 0) {
    place_diag(dp, dp.lu + dp.lu_off[u], m, k0, nb, a);
    if (rest <= 0) return;  // no tile: nothing allocated yet
  }
  int ti, tj;
  if (part == 0) {
    if (t < ntj) {
      ti = 0;
      tj = t;
    } else {
      ti = t - ntj + 1;
      tj = 0;
    }
  } else {
    ti = 1 + t / (ntj - 1);
    tj = 1 + t % (ntj - 1);
  }
  const uint32_t tmem = tc_tmem_alloc<kRTileN>(&s_tmem, &s_bar);
  uint32_t parity = 0;
  const bool ok = tile_update_tc<kRP, kRTileN>(dp.lu + dp.lu_off[u], m, base + ti * kRTileM, base + tj * kRTileN, k0,
                                               nb, split3 != 0, tc_align(tc_dyn_r), tmem, &s_bar, parity);
  if (!ok && threadIdx.x == 0) atomicCAS(dp.status, 0, kFailTensorSync);
  tc_tmem_free<kRTileN>(tmem);
}

// First-factor update (k_gemm_rm's 128 x 128 tiles, K = kPanel).
__global__ void __launch_bounds__(kTcThreads, 3) k_gemm_rm_tc(DevPlan dp, int32_t k0, int32_t ubase, int32_t nact,
                                                           int32_t split3) {
  extern __shared__ uint8_t tc_dyn_g[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
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
  const uint32_t tmem = tc_tmem_alloc<kGT>(&s_tmem, &s_bar);
  uint32_t parity = 0;
  const bool ok = tile_update_tc<kPanel, kGT>(dp.lu + dp.lu_off[u], m, base + ti * kGT, base + tj * kGT, k0, nb,
                                              split3 != 0, tc_align(tc_dyn_g), tmem, &s_bar, parity);
  if (!ok && threadIdx.x == 0) atomicCAS(dp.status, 0, kFailTensorSync);
  tc_tmem_free<kGT>(tmem);
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
    err = cudaFuncSetAttribute(k_gemm_rm, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kGemmSmem));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_rgemm, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kRGemmSmem));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_rpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kRPanelSmem));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_rdag, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kRDagSmem));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_trsv_tiles<true, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(trsv_smem<16>()));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_trsv_tiles<false, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(trsv_smem<16>()));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_trsv_tiles<true, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(trsv_smem<8>()));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_trsv_tiles<false, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(trsv_smem<8>()));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_rgemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kRTcSmem));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_gemm_rm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kGTcSmem));
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(k_large_perm, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 4 * 1024);
  });
  return err;
}

cudaError_t large_factor(const DevPlan& dp, const Plan& p, const int32_t* d_large_units, cudaStream_t stream,
                         int32_t* launches, int32_t prec) {
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
      (void)chunk;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(static_cast<unsigned>(na * csize));
      cfg.blockDim = dim3(kPanelThreads);
      cfg.dynamicSmemBytes = 0;
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
      if (prec > 0)
        k_gemm_rm_tc<<<p.step_gemm_total[static_cast<size_t>(st)], kTcThreads, kGTcSmem, stream>>>(dp, k0, ub, na,
                                                                                                  prec == 2);
      else
        k_gemm_rm<<<p.step_gemm_total[static_cast<size_t>(st)], kGThreads, kGemmSmem, stream>>>(dp, k0, ub, na);
      ++*launches;
    }
  }
  const int nl = static_cast<int>(p.large_units.size());
  if (nl > 0) {
    int32_t mmax = 0;
    for (int32_t u : p.large_units) mmax = std::max(mmax, p.ustart[static_cast<size_t>(u) + 1] - p.ustart[static_cast<size_t>(u)]);
    k_large_perm<<<nl, 256, static_cast<size_t>(mmax) * sizeof(int32_t), stream>>>(dp, d_large_units);
    ++*launches;
  }
  return cudaGetLastError();
}

cudaError_t large_scatter_reuse(const DevPlan& dp, const Plan& p, const double* d_vals, const int32_t* d_large_units,
                                cudaStream_t stream) {
  if (p.large_units.empty()) return cudaSuccess;
  k_scatter_large_perm<<<dim3(64, static_cast<unsigned>(p.large_units.size())), 256, 0, stream>>>(dp, d_vals, d_large_units);
  return cudaGetLastError();
}

cudaError_t large_refactor(const DevPlan& dp, const Plan& p, cudaStream_t sa, cudaStream_t sb, cudaEvent_t ev_a,
                           cudaEvent_t ev_b, int32_t* launches, int32_t prec) {
  cudaError_t e = large_setup();
  if (e != cudaSuccess) return e;
  // Fork: stream b starts after everything already queued on stream a.
  if ((e = cudaEventRecord(ev_a, sa)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(sb, ev_a, 0)) != cudaSuccess) return e;
  for (int32_t st = 0; st < p.rsteps; ++st) {
    const int32_t ub = p.rstep_ptr[static_cast<size_t>(st)];
    const int32_t na = p.rstep_ptr[static_cast<size_t>(st) + 1] - ub;
    if (na <= 0) continue;
    const int32_t k0 = st * kRPanel;
    const int32_t ns = p.rstep_strip_total[static_cast<size_t>(st)];
    k_rpanel<<<ns, kRThreads, kRPanelSmem, sa>>>(dp, k0, ub, na);
    ++*launches;
    // Part a of this step follows part b of the previous one (stream b so
    // far); part b of this step follows this step's strips (stream a so far).
    if ((e = cudaEventRecord(ev_b, sb)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(sa, ev_b, 0)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev_a, sa)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(sb, ev_a, 0)) != cudaSuccess) return e;
    const int32_t gb = p.rstep_gb_total[static_cast<size_t>(st)];
    if (gb > 0) {
      if (prec > 0) k_rgemm_tc<<<gb, kTcThreads, kRTcSmem, sb>>>(dp, k0, ub, na, 1, prec == 2);
      else k_rgemm<<<gb, kRThreads, kRGemmSmem, sb>>>(dp, k0, ub, na, 1);
      ++*launches;
    }
    const int32_t ga = p.rstep_ga_total[static_cast<size_t>(st)];
    if (ga > 0) {
      if (prec > 0) k_rgemm_tc<<<ga, kTcThreads, kRTcSmem, sa>>>(dp, k0, ub, na, 0, prec == 2);
      else k_rgemm<<<ga, kRThreads, kRGemmSmem, sa>>>(dp, k0, ub, na, 0);
      ++*launches;
    }
  }
  // Join.
  if ((e = cudaEventRecord(ev_b, sb)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(sa, ev_b, 0)) != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t large_refactor_dag(const DevPlan& dp, const Plan& p, const int32_t* d_tasks, int32_t* d_words,
                               cudaStream_t stream, int32_t* launches) {
  cudaError_t e = large_setup();
  if (e != cudaSuccess) return e;
  if (p.rtasks <= 0) return cudaErrorInvalidValue;
  static int grid_max = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rdag, kRThreads, kRDagSmem);
    grid_max = std::max(1, nsm * std::max(1, per_sm));
  });
  if ((e = cudaMemsetAsync(d_words, 0, static_cast<size_t>(p.rt_words) * sizeof(int32_t), stream)) != cudaSuccess)
    return e;
  const int grid = std::min(grid_max, p.rtasks);
  k_rdag<<<grid, kRThreads, kRDagSmem, stream>>>(dp, reinterpret_cast<const int4*>(d_tasks), p.rtasks, d_words);
  ++*launches;
  return cudaGetLastError();
}

cudaError_t large_solve_level(const DevPlan& dp, const Plan& p, int32_t level, const int32_t* d_units,
                              const int32_t* d_tile0, int32_t* d_sync, const double* rhs, int32_t ldr, double* xp,
                              const int32_t* nrhs, bool wide, cudaStream_t stream, int32_t* launches) {
  const int32_t g0 = p.lvl_large_ptr[static_cast<size_t>(level)];
  const int32_t g1 = p.lvl_large_ptr[static_cast<size_t>(level) + 1];
  if (g1 <= g0) return cudaSuccess;
  const int32_t tiles = p.lvl_large_tile0[static_cast<size_t>(g1)] - p.lvl_large_tile0[static_cast<size_t>(g0)];
  const int32_t nl = p.umax_level + 1;
  int32_t* tickets = d_sync + 2 * level;
  int32_t* ready_fwd = d_sync + 2 * nl;
  int32_t* ready_bwd = ready_fwd + p.large_tiles;
  if (wide) {
    k_trsv_tiles<true, 16><<<tiles, kSolveThreads, trsv_smem<16>(), stream>>>(
        dp, d_units + g0, d_tile0 + g0, g1 - g0, tickets, ready_fwd, rhs, ldr, xp, nrhs);
    k_trsv_tiles<false, 16><<<tiles, kSolveThreads, trsv_smem<16>(), stream>>>(
        dp, d_units + g0, d_tile0 + g0, g1 - g0, tickets + 1, ready_bwd, rhs, ldr, xp, nrhs);
  } else {
    k_trsv_tiles<true, 8><<<tiles, kSolveThreads, trsv_smem<8>(), stream>>>(
        dp, d_units + g0, d_tile0 + g0, g1 - g0, tickets, ready_fwd, rhs, ldr, xp, nrhs);
    k_trsv_tiles<false, 8><<<tiles, kSolveThreads, trsv_smem<8>(), stream>>>(
        dp, d_units + g0, d_tile0 + g0, g1 - g0, tickets + 1, ready_bwd, rhs, ldr, xp, nrhs);
  }
  *launches += 2;
  return cudaGetLastError();
}

int32_t large_sync_words(const Plan& p) { return 2 * (p.umax_level + 1) + 2 * p.large_tiles; }

}  // namespace bdlu
