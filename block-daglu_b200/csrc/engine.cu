// sm_100a kernels and device memory management for the numeric factor and
// solve.  Units are raw BTF blocks (plan.h).  Kernels:
//   k_gather          coupling values + scalar-unit diagonals from the
//                     canonical value array (value-only refactor is a gather)
//   k_lu_small        one CTA per dense unit, the unit in shared memory, fused
//                     value scatter; unblocked partial-pivoting LU that
//                     performs exactly the reference micro-kernel's operations
//                     (ubtf_block_solver.cpp:1450-1498): same pivot choice,
//                     same per-element operation order, no FMA contraction,
//                     so factors are bit-identical
//   k_scatter_large   value scatter into the arena slots of large units (the
//                     blocked LU and large-unit solves are in large.cu)
//   k_solve_level     one solve level's scalar rows and small dense units
//                     level-scheduled block back-substitution with the
//                     off-diagonal update fused in (ubtf_block_solver.cpp:
//                     2260-2401): rhs = b - A_cpl x, then the unit's L/U solve
//   k_unpermute       x[Q[i]] (+)= xperm[i]
//   k_residual        r = b - A x over the canonical CSR, with inf-norms
#include "engine.h"

#include "device_util.cuh"
#include "gp_dev.h"
#include "tc_update.cuh"
#include "tuner.h"
#include "large.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <utility>

namespace bdlu {

namespace {

constexpr int kThreads = 256;
// Rows of the largest small unit any kernel here takes (the shared-memory
// limit, small_unit_max(), is 169 on a 227 KB part), rounded up to a warp.
constexpr int kLuRowsMax = 192;
constexpr int32_t kWorkRhs = 16;
// ---------------------------------------------------------------------------
// Value gather for coupling entries and scalar units.
// ---------------------------------------------------------------------------
__global__ void k_gather(DevPlan dp, const double* __restrict__ vals, int64_t ncpl) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < ncpl; q += stride)
    dp.cpl_val[q] = vals[dp.cpl_src[q]];
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < dp.n; r += stride) {
    const int32_t src = dp.sdiag_src[r];
    if (src == -1) continue;  // row of a dense unit
    const double v = (src >= 0) ? vals[src] : 0.0;
    dp.sdiag[r] = v;
    if (v == 0.0) report_failure(dp.status, static_cast<int32_t>(r));
  }
}

__global__ void k_set_i32(int32_t* p, int32_t v) { *p = v; }

// Start of a solve: the right-hand-side count for the captured sweep, and a
// solve-wait failure left by the previous solve cleared (factor failures
// stay until the next factor).
__global__ void k_solve_begin(int32_t* nrhs_word, int32_t nrhs, int32_t* status) {
  *nrhs_word = nrhs;
  if (status[0] == kFailSync) {
    status[0] = 0;
    status[1] = 0;
  }
}

// ---------------------------------------------------------------------------
// Dense LU of one unit in shared memory (column-major, leading dimension m).
// ---------------------------------------------------------------------------
// Warp-level pivot candidate: the largest |v| (ties to the smallest row,
// rows with i == none taking no part) and the signed value of that entry.
__device__ __forceinline__ void warp_pivot_signed(double v, int i, int none, double& best, int& bi, double& sv) {
  double a = (i == none) ? 0.0 : fabs(v);
  int idx = i;
  warp_pivot_reduce(a, idx, none);
  const unsigned who = __ballot_sync(0xffffffffu, i != none && i == idx);
  sv = __shfl_sync(0xffffffffu, v, who ? __ffs(who) - 1 : 0);
  best = a;
  bi = idx;
}

// One unit factored by the whole CTA (kT threads, kT >= m): A is the CTA's
// m*m shared-memory slot.  A failed unit reports and returns (CTA-uniform).
template <int kT>
__device__ __forceinline__ void lu_cta_unit(const DevPlan& dp, const double* __restrict__ vals, int u, double* A,
                                            double* s_best, double* s_val, int* s_bi) {
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < m * m; i += kT) A[i] = 0.0;
  __syncthreads();
  for (int64_t e = dp.dent_ptr[u] + tid; e < dp.dent_ptr[u + 1]; e += kT) A[dp.dent_pos[e]] = vals[dp.dent_src[e]];
  __syncthreads();
  int32_t* piv = dp.piv + s;
  // Two barriers per column.  Pivot candidates of column k (first strict
  // maximum of |a|, with the signed value) come from the update of step k-1
  // (column 0: scanned first); after the barrier every thread combines the
  // per-warp candidates itself.  The row swap and the multipliers of column k
  // then run in one phase (the multipliers read the pivot row before the
  // swap: a'_pk = a_kk); the update of step k also collects column k+1's
  // candidates.  The arithmetic is the reference micro-kernel's, operation
  // for operation.  A lane keeps the first strict maximum of its rows.
  {
    const int i = (tid < m) ? tid : m;
    double best, sv;
    int bi;
    warp_pivot_signed(i < m ? A[i] : 0.0, i, m, best, bi, sv);
    if (lane == 0) {
      s_best[warp] = best;
      s_bi[warp] = bi;
      s_val[warp] = sv;
    }
  }
  __syncthreads();
  for (int k = 0; k < m; ++k) {
    double best = s_best[0], pv = s_val[0];
    int p = s_bi[0];
#pragma unroll
    for (int w = 1; w < kT / 32; ++w) {
      const double ob = s_best[w];
      const int oi = s_bi[w];
      if (oi != m && (p == m || ob > best || (ob == best && oi < p))) {
        best = ob;
        p = oi;
        pv = s_val[w];
      }
    }
    if (p == m || best == 0.0) {
      if (tid == 0) report_failure(dp.status, u);
      return;
    }
    double* colk = A + static_cast<size_t>(k) * m;
    if (tid == 0) piv[k] = p;
    const double akk = colk[k];
    if (p != k) {
      for (int j = tid; j < m; j += kT) {
        if (j == k) continue;
        double* c = A + static_cast<size_t>(j) * m;
        const double t = c[k];
        c[k] = c[p];
        c[p] = t;
      }
    }
    for (int i = k + 1 + tid; i < m; i += kT) colk[i] = __ddiv_rn(i == p ? akk : colk[i], pv);
    __syncthreads();
    if (tid == 0) colk[k] = pv;
    // Update of the active (m-k-1) x (m-k-1) block, spread evenly over the
    // CTA: element e = tid + kT q is row k+1 + e % nr of column k+1 + e / nr
    // (column-major, so a warp's loads and stores are consecutive), the row
    // and column advanced incrementally.  Every issued update is a real one.
    // Column k+1's entries (e < nr) also yield the next pivot candidates.
    double cb = 0.0, cv = 0.0;
    int ci = m;
    const int nr = m - k - 1;
    if (nr > 0) {
      const int ne = nr * nr;
      const int sr = kT % nr, sc = kT / nr;
      int ii = tid % nr, jj = tid / nr;
      for (int e = tid; e < ne; e += kT) {
        const int i = k + 1 + ii;
        double* c = A + static_cast<size_t>(k + 1 + jj) * m;
        const double v = __dsub_rn(c[i], __dmul_rn(colk[i], c[k]));
        c[i] = v;
        if (jj == 0 && (ci == m || fabs(v) > cb)) {
          cb = fabs(v);
          cv = v;
          ci = i;
        }
        ii += sr;
        jj += sc;
        if (ii >= nr) {
          ii -= nr;
          ++jj;
        }
      }
    }
    double nb, nsv;
    int nbi;
    warp_pivot_signed(cv, ci, m, nb, nbi, nsv);
    if (lane == 0) {
      s_best[warp] = nb;
      s_bi[warp] = nbi;
      s_val[warp] = nsv;
    }
    __syncthreads();
  }
  double* out = dp.lu + dp.lu_off[u];
  for (int i = tid; i < m * m; i += kT) out[i] = A[i];
  // Final row order (row k of the factor is local row lperm[k]) for the solve.
  __syncthreads();
  int32_t* ord = reinterpret_cast<int32_t*>(A);
  for (int k = tid; k < m; k += kT) ord[k] = k;
  __syncthreads();
  if (tid == 0) {
    for (int k = 0; k < m; ++k) {
      const int p = piv[k];
      if (p != k) {
        const int32_t t = ord[k];
        ord[k] = ord[p];
        ord[p] = t;
      }
    }
  }
  __syncthreads();
  for (int k = tid; k < m; k += kT) dp.lperm[s + k] = ord[k];
}

template <int kT>
__global__ void __launch_bounds__(kT) k_lu_small(DevPlan dp, const double* __restrict__ vals,
                                                  const int32_t* __restrict__ units) {
  extern __shared__ double A[];
  __shared__ double s_best[kT / 32], s_val[kT / 32];
  __shared__ int s_bi[kT / 32];
  lu_cta_unit<kT>(dp, vals, units[blockIdx.x], A, s_best, s_val, s_bi);
}

// ---------------------------------------------------------------------------
// Column-warp LU: one warp per unit of up to 32*R rows (the C2 "column-warp"
// path), several units per CTA, no CTA barriers.  Lane l holds rows l,
// l + 32, ... of the unit in registers (all columns, statically indexed: the
// column loop is unrolled), row swaps are logical (each held row carries its
// current position; a swap exchanges two positions), the pivot row is
// broadcast by shuffles.  Per element the arithmetic is the micro-kernel's:
// first strict maximum of |a| (ties to the smallest position), multipliers by
// division, a - l*u as multiply then subtract; so the factors, pivots and row
// order are bit-identical to k_lu_small's.
// One unit of up to 32*R rows factored by one warp; S is the warp's
// (32R)^2-double shared-memory staging slot.  A failed unit reports and
// returns (warp-uniform).
template <int R>
__device__ __forceinline__ void lu_warp_unit(const DevPlan& dp, const double* __restrict__ vals, int u, double* S) {
  constexpr int M = 32 * R;
  constexpr int kNone = 1 << 20;  // position of rows outside the unit
  const int lane = threadIdx.x & 31;
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  for (int i = lane; i < m * m; i += 32) S[i] = 0.0;
  __syncwarp();
  for (int64_t e = dp.dent_ptr[u] + lane; e < dp.dent_ptr[u + 1]; e += 32) S[dp.dent_pos[e]] = vals[dp.dent_src[e]];
  __syncwarp();
  double a[R][M];
  int pos[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int row = lane + 32 * r;
    pos[r] = row < m ? row : kNone;
#pragma unroll
    for (int j = 0; j < M; ++j) a[r][j] = (row < m && j < m) ? S[j * m + row] : 0.0;
  }
  int32_t* piv = dp.piv + s;
#pragma unroll
  for (int k = 0; k < M; ++k) {
    if (k >= m) break;
    // Pivot: this lane's best row (largest |a|, smallest position), then the
    // warp's.
    double best = 0.0;
    int bpos = kNone;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double v = fabs(a[r][k]);
      if (pos[r] >= k && pos[r] != kNone && (bpos == kNone || v > best || (v == best && pos[r] < bpos))) {
        best = v;
        bpos = pos[r];
      }
    }
    warp_pivot_reduce(best, bpos, kNone);
    if (bpos == kNone || best == 0.0) {
      if (lane == 0) report_failure(dp.status, u);
      return;
    }
    const int p = bpos;
    // Owner lane and row slot of the pivot row.
    int oslot = -1;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (pos[r] == p) oslot = r;
    const unsigned who = __ballot_sync(0xffffffffu, oslot >= 0);
    const int olane = __ffs(who) - 1;
    const int orow = __shfl_sync(0xffffffffu, oslot, olane);
    if (lane == 0) piv[k] = p;
    // Logical swap of positions k and p.
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (pos[r] == k) pos[r] = p;
      else if (pos[r] == p) pos[r] = k;
    }
    const double pv = __shfl_sync(0xffffffffu, orow == 0 ? a[0][k] : a[R - 1][k], olane);
    double l[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      l[r] = 0.0;
      if (pos[r] > k && pos[r] != kNone) {
        l[r] = __ddiv_rn(a[r][k], pv);
        a[r][k] = l[r];
      }
    }
#pragma unroll
    for (int j = k + 1; j < M; ++j) {
      if (j >= m) break;
      const double uj = __shfl_sync(0xffffffffu, orow == 0 ? a[0][j] : a[R - 1][j], olane);
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (pos[r] > k && pos[r] != kNone) a[r][j] = __dsub_rn(a[r][j], __dmul_rn(l[r], uj));
    }
  }
  double* out = dp.lu + dp.lu_off[u];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int row = lane + 32 * r;
    if (row < m) {
#pragma unroll
      for (int j = 0; j < M; ++j)
        if (j < m) out[static_cast<size_t>(j) * m + pos[r]] = a[r][j];
      dp.lperm[s + pos[r]] = row;
    }
  }
}

// Row-per-thread LU: one CTA of M threads per unit of up to M rows (M = 64
// or 96).  Thread t holds row t of the unit in registers; row swaps are
// logical as in lu_warp_unit (a row's position is final once it has been the
// pivot row).  The column loop runs at run time over a compact body: the
// update walks the row in chunks of kRC columns with constant register
// indices and skips, by a warp-uniform branch, every chunk left of the
// current column; multipliers go to the shared staging buffer (column-major,
// as the factor is written out), so no register is indexed by the column.
// Per column: warp candidates (first strict maximum of |a| over the rows not
// yet pivoted), combined by every thread from shared memory; the pivot row's
// owner publishes its remaining entries; each row below forms its multiplier
// and updates itself.  Two barriers of M threads per column.  Arithmetic per
// element is the micro-kernel's, so the factors, pivots and row order are
// bit-identical to k_lu_small's.
constexpr int kRC = 8;  // columns per register chunk of k_lu_rows
template <int M>
__global__ void __launch_bounds__(M) k_lu_rows(DevPlan dp, const double* __restrict__ vals,
                                               const int32_t* __restrict__ units) {
  static_assert(M % 32 == 0 && M % kRC == 0 && M <= 96, "rows per unit");
  constexpr int kW = M / 32, kChunks = M / kRC;
  constexpr int kNone = 1 << 20;
  extern __shared__ double S[];  // m x m: the unit's entries, then the multipliers
  __shared__ __align__(16) double s_u[M];  // the pivot row of the current column
  __shared__ double s_best[kW];
  __shared__ int s_pos[kW];
  const int u = units[blockIdx.x];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int i = t; i < m * m; i += M) S[i] = 0.0;
  __syncthreads();
  for (int64_t e = dp.dent_ptr[u] + t; e < dp.dent_ptr[u + 1]; e += M) S[dp.dent_pos[e]] = vals[dp.dent_src[e]];
  __syncthreads();
  double a[M];
#pragma unroll
  for (int j = 0; j < M; ++j) a[j] = (t < m && j < m) ? S[j * m + t] : 0.0;
  __syncthreads();  // S now takes the multipliers
  int pos = t < m ? t : kNone;
  double ak = a[0];  // this row's entry in the current column
  int32_t* piv = dp.piv + s;
  for (int k = 0; k < m; ++k) {
    const bool cand = pos >= k && pos != kNone;
    double best = cand ? fabs(ak) : 0.0;
    int bpos = cand ? pos : kNone;
    warp_pivot_reduce(best, bpos, kNone);
    if (lane == 0) {
      s_best[warp] = best;
      s_pos[warp] = bpos;
    }
    __syncthreads();
    best = s_best[0];
    bpos = s_pos[0];
#pragma unroll
    for (int w = 1; w < kW; ++w) pivot_combine(best, bpos, s_best[w], s_pos[w], kNone);
    if (bpos == kNone || best == 0.0) {  // CTA-uniform
      if (t == 0) report_failure(dp.status, u);
      return;
    }
    const int p = bpos;
    if (pos == p) {
      s_u[k] = ak;
#pragma unroll
      for (int c = 0; c < kChunks; ++c) {
        if (kRC * c + kRC - 1 <= k) continue;  // uniform
#pragma unroll
        for (int e = 0; e < kRC; ++e) {
          const int j = kRC * c + e;
          if (j > k && j < m) s_u[j] = a[j];
        }
      }
    }
    if (t == 0) piv[k] = p;
    if (pos == k) pos = p;
    else if (pos == p) pos = k;
    __syncthreads();
    double nk = 0.0;
    if (pos > k && pos != kNone) {
      const double l = __ddiv_rn(ak, s_u[k]);
      S[k * m + t] = l;
#pragma unroll
      for (int c = 0; c < kChunks; ++c) {
        if (kRC * c + kRC - 1 <= k || kRC * c >= m) continue;  // uniform
        if (kRC * c > k && kRC * c + kRC <= m) {
          // The chunk of the pivot row first (16-byte loads), then the
          // arithmetic: the loads overlap instead of each update waiting.
          double uc[kRC];
#pragma unroll
          for (int e = 0; e < kRC; e += 2) {
            const double2 v = *reinterpret_cast<const double2*>(s_u + kRC * c + e);
            uc[e] = v.x;
            uc[e + 1] = v.y;
          }
#pragma unroll
          for (int e = 0; e < kRC; ++e) {
            const int j = kRC * c + e;
            a[j] = __dsub_rn(a[j], __dmul_rn(l, uc[e]));
            if (j == k + 1) nk = a[j];
          }
        } else {
#pragma unroll
          for (int e = 0; e < kRC; ++e) {
            const int j = kRC * c + e;
            if (j > k && j < m) {
              a[j] = __dsub_rn(a[j], __dmul_rn(l, s_u[j]));
              if (j == k + 1) nk = a[j];
            }
          }
        }
      }
    }
    ak = nk;
  }
  // Row t sits at position `pos`, the step at which it was the pivot row:
  // its multipliers (columns before pos) are in S, its row of U in registers.
  if (t < m) {
    double* out = dp.lu + dp.lu_off[u];
    for (int j = 0; j < pos; ++j) out[static_cast<size_t>(j) * m + pos] = S[j * m + t];
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (j >= pos && j < m) out[static_cast<size_t>(j) * m + pos] = a[j];
    dp.lperm[s + pos] = t;
  }
}

template <int R, int W>
__global__ void __launch_bounds__(32 * W) k_lu_warp(DevPlan dp, const double* __restrict__ vals,
                                                    const int32_t* __restrict__ units, int32_t count) {
  extern __shared__ double wsm[];
  const int wib = threadIdx.x >> 5;
  const int slot = blockIdx.x * W + wib;
  if (slot >= count) return;  // warp-uniform
  lu_warp_unit<R>(dp, vals, units[slot], wsm + static_cast<size_t>(wib) * (32 * R) * (32 * R));
}

// Every small unit of the pattern in one persistent launch: each CTA takes
// tasks from a device queue (atomic ticket) until it is empty.  A task is one
// unit for the whole CTA (more than 32 rows) or a pack of up to eight units of
// at most 32 rows, one per warp (column-warp path).  Tasks come largest first
// (host-built list: first unit, unit count; count > 0 marks a pack).  Shared
// memory: the largest task's need.
constexpr int kQueueThreads = 256;
__global__ void __launch_bounds__(kQueueThreads) k_lu_queue(DevPlan dp, const double* __restrict__ vals,
                                                            const int32_t* __restrict__ units,
                                                            const int2* __restrict__ tasks, int32_t ntasks,
                                                            int32_t* __restrict__ ticket) {
  extern __shared__ double qsm[];
  __shared__ double s_best[kQueueThreads / 32], s_val[kQueueThreads / 32];
  __shared__ int s_bi[kQueueThreads / 32];
  __shared__ int s_t;
  const int warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_t = atomicAdd(ticket, 1);
    __syncthreads();
    const int t = s_t;
    __syncthreads();
    if (t >= ntasks) break;
    const int2 task = tasks[t];
    if (task.y == 0) {
      lu_cta_unit<kQueueThreads>(dp, vals, units[task.x], qsm, s_best, s_val, s_bi);
    } else if (warp < task.y) {
      lu_warp_unit<1>(dp, vals, units[task.x + warp], qsm + static_cast<size_t>(warp) * 32 * 32);
    }
    __syncthreads();
  }
}

constexpr int kWarpLuW1 = 4;  // units (warps) per CTA, up to 32 rows
constexpr int kWarpLuW2 = 2;  // up to 64 rows

// ---------------------------------------------------------------------------
// Large units: value scatter into their (row-major) arena slots.
// ---------------------------------------------------------------------------
__global__ void k_scatter_large(DevPlan dp, const double* __restrict__ vals, const int32_t* __restrict__ units) {
  const int u = units[blockIdx.y];
  double* A = dp.lu + dp.lu_off[u];
  for (int64_t e = dp.dent_ptr[u] + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < dp.dent_ptr[u + 1];
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    A[dp.dent_pos[e]] = vals[dp.dent_src[e]];
}

// ---------------------------------------------------------------------------
// Solve.  xp holds the solution in permuted order (n x nrhs, ld n).
// ---------------------------------------------------------------------------
// Small dense units (column-major LU, final row order in dp.lperm).  The
// unit's m x m factor is copied to shared memory as it lies in the arena;
// each warp then takes one right-hand side: it forms the pivoted rhs of its
// rows directly in registers (kSlots rows per lane, b - A_cpl x gathered
// through the row order), sweeps L and U with the column's values kept in
// registers and each finished unknown broadcast by a shuffle, and writes x.
// The backward sweep multiplies by the reciprocal of the pivot, which keeps
// the division off the dependent chain.
// kS rows per lane, chosen per launch from the level's largest unit: units
// up to 32 kS rows; at most kSlots (192 rows).
constexpr int kSlots = 6;
static_assert(32 * kSlots >= kLuRowsMax, "register slots must cover the small-unit limit");

// Programmatic dependent launch: the next kernel of the stream may start
// its prologue once every CTA of this one has started; griddepcontrol.wait
// blocks until the kernels this one depends on have completed and their
// writes are visible (it returns at once when the launch had no
// programmatic dependency).
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// One solve level's scalar rows and small dense units in one launch: CTAs
// below scal_ctas take the scalar rows (a warp per row: rhs - A_cpl x over
// the coupling row, divided by the diagonal); the others take one dense unit
// each.  From the second level on the kernel is launched as a programmatic
// dependent of the previous one: a dense CTA issues the bulk copy of its
// factor slot and computes its row order before it waits for the previous
// level, so the copy and the launch overlap the previous level's tail.
template <int kS>
__global__ void __launch_bounds__(kThreads, 4) k_solve_level(DevPlan dp, const int32_t* __restrict__ srows,
                                                           int32_t nsrows, int32_t scal_ctas,
                                                           const int32_t* __restrict__ units,
                                                           const double* __restrict__ rhs, int32_t ldr,
                                                           double* __restrict__ xp,
                                                           const int32_t* __restrict__ nrhs_p) {
  pdl_launch_dependents();
  const int32_t nrhs = *nrhs_p;
  if (static_cast<int32_t>(blockIdx.x) < scal_ctas) {
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int n = dp.n;
    constexpr int kW = kThreads / 32;
    for (int w = blockIdx.x * kW + (threadIdx.x >> 5); w < nsrows; w += scal_ctas * kW) {
      const int r = srows[w];
      const int p0 = dp.cpl_ptr[r], p1 = dp.cpl_ptr[r + 1];
      const double d = dp.sdiag[r];
      const int src = dp.P[r];
      for (int k = 0; k < nrhs; ++k) {
        double acc = 0.0;
        for (int q = p0 + lane; q < p1; q += 32) acc = fma(dp.cpl_val[q], xp[dp.cpl_col[q] + static_cast<size_t>(k) * n], acc);
        acc = warp_sum(acc);
        if (lane == 0) xp[r + static_cast<size_t>(k) * n] = (rhs[src + static_cast<size_t>(k) * ldr] - acc) / d;
      }
    }
    return;
  }
  extern __shared__ __align__(16) double T[];
  const int u = units[blockIdx.x - scal_ctas];
  const int s = dp.ustart[u];
  const int m = dp.ustart[u + 1] - s;
  const int n = dp.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = kThreads / 32;
  const int nmine = (nrhs - warp + kWarps - 1) / kWarps;  // right-hand sides of this warp
  double a[kS];
  int rows[kS];
#pragma unroll
  for (int k = 0; k < kS; ++k) {
    const int i = lane + 32 * k;
    rows[k] = (i < m) ? s + dp.lperm[s + i] : -1;
  }
  auto form = [&](int c) {
#pragma unroll
    for (int k = 0; k < kS; ++k) {
      a[k] = 0.0;
      const int r = rows[k];
      if (r >= 0) {
        const double* xk = xp + static_cast<size_t>(c) * n;
        double acc = 0.0;
        const int p1 = dp.cpl_ptr[r + 1];
#pragma unroll 4
        for (int q = dp.cpl_ptr[r]; q < p1; ++q) acc = fma(__ldg(dp.cpl_val + q), xk[__ldg(dp.cpl_col + q)], acc);
        a[k] = rhs[dp.P[r] + static_cast<size_t>(c) * ldr] - acc;
      }
    }
  };
  // The unit's factor slot is contiguous and 256-byte aligned: one bulk
  // copy (TMA) stages it while the warps form their right-hand sides.
  __shared__ __align__(8) uint64_t mbar;
  const double* LU = dp.lu + dp.lu_off[u];
  const uint32_t bytes = static_cast<uint32_t>((m * m + 1) / 2) * 16u;  // slots are padded to 32 doubles
  const uint32_t mbar_s = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar));
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_s));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar_s), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            static_cast<uint32_t>(__cvta_generic_to_shared(T))),
        "l"(LU), "r"(bytes), "r"(mbar_s)
        : "memory");
  }
  // Everything above reads only the factors; the right-hand sides read the
  // unknowns of earlier levels.
  pdl_wait();
  if (nmine > 0) form(warp);
  // Bounded wait for the copy (phase 0); on a timeout the unit reports a
  // synchronisation failure, waits once more for the copy in flight, and
  // skips its sweeps.
  bool staged = false;
  for (int pass = 0; pass < 2 && !staged; ++pass) {
    for (int it = 0; it < (1 << 22); ++it) {
      uint32_t done = 0;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
          : "=r"(done)
          : "r"(mbar_s)
          : "memory");
      if (done) {
        staged = true;
        break;
      }
    }
    if (!staged && pass == 0 && tid == 0) atomicCAS(dp.status, 0, kFailSync);
  }
  if (!__syncthreads_and(staged)) {
    if (tid == 0) atomicCAS(dp.status, 0, kFailSync);
    return;
  }
  // Reciprocals of the pivots, formed in parallel: the backward sweep
  // multiplies, with no division on its dependent chain.
  __shared__ double rdiag[32 * kS];
  for (int i = tid; i < m; i += kThreads) rdiag[i] = 1.0 / T[i * m + i];
  __syncthreads();
  for (int t = 0; t < nmine; ++t) {
    const int c = warp + t * kWarps;
    if (t > 0) form(c);
    // L: unit lower triangle, columns j = 0 .. m-2.
#pragma unroll
    for (int kk = 0; kk < kS; ++kk) {
      const int jend = min(32, m - 1 - 32 * kk);
      for (int jj = 0; jj < jend; ++jj) {
        const int j = 32 * kk + jj;
        const double xr = __shfl_sync(0xffffffffu, a[kk], jj);
        const double* col = T + j * m;
#pragma unroll
        for (int k = kk; k < kS; ++k) {
          const int i = lane + 32 * k;
          if (i > j && i < m) a[k] = fma(-col[i], xr, a[k]);
        }
      }
    }
    // U with its diagonal, columns j = m-1 .. 0.
#pragma unroll
    for (int kk = kS - 1; kk >= 0; --kk) {
      const int jtop = min(31, m - 1 - 32 * kk);
      for (int jj = jtop; jj >= 0; --jj) {
        const int j = 32 * kk + jj;
        const double* col = T + j * m;
        const double xr = __shfl_sync(0xffffffffu, a[kk], jj) * rdiag[j];
        if (lane == jj) a[kk] = xr;
#pragma unroll
        for (int k = 0; k <= kk; ++k) {
          const int i = lane + 32 * k;
          if (i < j) a[k] = fma(-col[i], xr, a[k]);
        }
      }
    }
    double* xo = xp + static_cast<size_t>(c) * n + s;
#pragma unroll
    for (int k = 0; k < kS; ++k) {
      const int i = lane + 32 * k;
      if (i < m) xo[i] = a[k];
    }
  }
}

__global__ void k_unpermute(const int32_t* __restrict__ Q, int32_t n, const double* __restrict__ xp,
                            double* __restrict__ X, int32_t ldx, int32_t nrhs, int add) {
  const int64_t total = static_cast<int64_t>(n) * nrhs;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = t / n;
    const int64_t i = t - k * n;
    double* dst = X + Q[i] + k * ldx;
    if (add) *dst += xp[t];
    else *dst = xp[t];
  }
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  atomicMax(a, static_cast<unsigned long long>(__double_as_longlong(v)));
}

// R = B - A X (original coordinates); norms[4k..4k+3] gather |r|_inf, |b|_inf,
// |x|_inf, |A|_inf for column k.  Four lanes per row (rows hold a few
// entries), grid-stride over rows, right-hand sides in chunks of kResRhs so
// each pass reads the matrix once for the chunk; each thread keeps running
// maxima, reduced per warp and per CTA, so a CTA issues four atomics per
// column instead of one per row.
constexpr int kResLanes = 4;
constexpr int kResRhs = 8;
__global__ void __launch_bounds__(kThreads) k_residual(DevPlan dp, const double* __restrict__ vals,
                                                        const double* __restrict__ X, int32_t ldx,
                                                        const double* __restrict__ B, int32_t ldb,
                                                        double* __restrict__ R, int32_t nrhs,
                                                        unsigned long long* norms) {
  __shared__ double red[kThreads / 32][4 * kResRhs];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = threadIdx.x & (kResLanes - 1);
  // The loop runs over the warp's first row so that every lane takes the
  // same iterations (the shuffles below need the whole warp).
  const int64_t wbase = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x - lane) / kResLanes;
  const int64_t groups = static_cast<int64_t>(gridDim.x) * blockDim.x / kResLanes;
  for (int k0 = 0; k0 < nrhs; k0 += kResRhs) {
    const int nc = min(kResRhs, nrhs - k0);
    double mr[kResRhs], mb[kResRhs], mx[kResRhs], ma = 0.0;
#pragma unroll
    for (int c = 0; c < kResRhs; ++c) mr[c] = mb[c] = mx[c] = 0.0;
    for (int64_t base = wbase; base < dp.n; base += groups) {
      const int64_t r = base + lane / kResLanes;
      const bool valid = r < dp.n;
      const int p0 = valid ? dp.csr_ptr[r] : 0, p1 = valid ? dp.csr_ptr[r + 1] : 0;
      double acc[kResRhs], arow = 0.0;
#pragma unroll
      for (int c = 0; c < kResRhs; ++c) acc[c] = 0.0;
      for (int q = p0 + sub; q < p1; q += kResLanes) {
        const double v = vals[q];
        const int col = dp.csr_col[q];
        arow += fabs(v);
#pragma unroll
        for (int c = 0; c < kResRhs; ++c)
          if (c < nc) acc[c] = fma(v, X[col + static_cast<size_t>(k0 + c) * ldx], acc[c]);
      }
#pragma unroll
      for (int off = kResLanes / 2; off > 0; off >>= 1) {
        arow += __shfl_xor_sync(0xffffffffu, arow, off, kResLanes);
#pragma unroll
        for (int c = 0; c < kResRhs; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off, kResLanes);
      }
      if (valid && sub == 0) {
        ma = fmax(ma, arow);
#pragma unroll
        for (int c = 0; c < kResRhs; ++c) {
          if (c >= nc) continue;
          const double bv = B[r + static_cast<size_t>(k0 + c) * ldb];
          const double res = bv - acc[c];
          if (R) R[r + static_cast<size_t>(k0 + c) * dp.n] = res;
          mr[c] = fmax(mr[c], fabs(res));
          mb[c] = fmax(mb[c], fabs(bv));
          mx[c] = fmax(mx[c], fabs(X[r + static_cast<size_t>(k0 + c) * ldx]));
        }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, off));
#pragma unroll
      for (int c = 0; c < kResRhs; ++c) {
        mr[c] = fmax(mr[c], __shfl_xor_sync(0xffffffffu, mr[c], off));
        mb[c] = fmax(mb[c], __shfl_xor_sync(0xffffffffu, mb[c], off));
        mx[c] = fmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], off));
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < kResRhs; ++c) {
        red[warp][4 * c + 0] = mr[c];
        red[warp][4 * c + 1] = mb[c];
        red[warp][4 * c + 2] = mx[c];
        red[warp][4 * c + 3] = ma;
      }
    }
    __syncthreads();
    if (threadIdx.x < 4 * nc) {
      double m = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) m = fmax(m, red[w][threadIdx.x]);
      atomic_max_nonneg(norms + 4 * k0 + threadIdx.x, m);
    }
    __syncthreads();
  }
}

int grid_for(int64_t work, int threads, int cap) {
  const int64_t g = (work + threads - 1) / threads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(g, cap)));
}

}  // namespace

int32_t small_unit_max() {
  int dev = 0;
  cudaGetDevice(&dev);
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || optin <= 0)
    optin = 227 * 1024;
  // m*m doubles plus the kernel's static shared memory (~1 KB).
  const int64_t budget = optin - 2048;
  int32_t m = 1;
  while (static_cast<int64_t>(m + 1) * (m + 1) * 8 <= budget) ++m;
  return std::min<int32_t>(m, kLuRowsMax);  // the kernels' row registers cover kLuRowsMax
}

Engine::Engine() {
  // The refactor graph's dependent chain is captured on the highest-priority
  // stream and its lookahead branch on the lowest, so waiting chain CTAs are
  // scheduled ahead of the branch's (the graph keeps node priorities).
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  cudaStreamCreateWithPriority(&cap_stream_, cudaStreamNonBlocking, prio_high);
  cudaStreamCreateWithPriority(&cap_stream2_, cudaStreamNonBlocking, prio_low);
  for (auto& a : aux_) cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking);
  for (auto& e : aux_ev_) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto& e : fork_ev_) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto& e : ev_) cudaEventCreate(&e);
  for (auto& e : pev_) cudaEventCreate(&e);
  cudaStreamCreateWithFlags(&gp_stream_, cudaStreamNonBlocking);
  for (auto& e : gp_ev_) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  if (cudaMallocHost(reinterpret_cast<void**>(&readback_), kReadbackBytes) != cudaSuccess) {
    readback_ = new char[kReadbackBytes];  // pageable: correct, only slower
    readback_pinned_ = false;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev);
}

Engine::~Engine() {
  release();
  if (wait_ev_) cudaEventDestroy(wait_ev_);
  if (readback_pinned_) cudaFreeHost(readback_);
  else delete[] readback_;
  if (cap_stream_) cudaStreamDestroy(cap_stream_);
  if (cap_stream2_) cudaStreamDestroy(cap_stream2_);
  for (auto& a : aux_)
    if (a) cudaStreamDestroy(a);
  for (auto& e : aux_ev_)
    if (e) cudaEventDestroy(e);
  for (auto& e : fork_ev_)
    if (e) cudaEventDestroy(e);
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  for (auto& e : pev_)
    if (e) cudaEventDestroy(e);
  if (gp_stream_) cudaStreamDestroy(gp_stream_);
  for (auto& e : gp_ev_)
    if (e) cudaEventDestroy(e);
}

void Engine::drop_graphs() {
  for (auto& ge : solve_exec_)
    if (ge) cudaGraphExecDestroy(ge);
  if (reuse_exec_) cudaGraphExecDestroy(reuse_exec_);
  solve_exec_[0] = solve_exec_[1] = nullptr;
  reuse_exec_ = nullptr;
  solve_exec_b0_ = nullptr;
}

void Engine::release() {
  drop_graphs();
  for (auto& a : allocs_) cudaFree(a.first);
  allocs_.clear();
  d_vals_ = nullptr;
  d_status_ = nullptr;
  d_b0_ = d_xp_ = d_r_ = d_rhs_ = nullptr;
  d_norms_ = nullptr;
  d_rtask_ = nullptr;
  d_rwords_ = nullptr;
  d_vals_stage_ = nullptr;
  d_qunits_ = d_qtasks_ = nullptr;
  d_qticket_ = nullptr;
  queue_tasks_ = 0;
  work_nrhs_ = 0;
  dp_ = DevPlan{};
  const GpDev keep = gp_;
  gp_ = GpDev{};
  gp_.diag_tol = keep.diag_tol;
  gp_.pivot_tol = keep.pivot_tol;
  gp_.min_abs_diag = keep.min_abs_diag;
  lvl_sparse_ = nullptr;
}

#define BDLU_CUDA(call)                                                      \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      return false;                                                          \
    }                                                                        \
  } while (0)

template <class T>
static bool upload_vec(std::vector<std::pair<void*, size_t>>& allocs, const std::vector<T>& v, const T** out, std::string& err) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
  BDLU_CUDA(cudaMalloc(&p, bytes));
  allocs.emplace_back(p, bytes);
  if (!v.empty()) BDLU_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = static_cast<const T*>(p);
  return true;
}

template <class T>
static bool alloc_dev(std::vector<std::pair<void*, size_t>>& allocs, size_t count, T** out, std::string& err) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  BDLU_CUDA(cudaMalloc(&p, bytes));
  allocs.emplace_back(p, bytes);
  *out = static_cast<T*>(p);
  return true;
}

bool Engine::upload(const Plan& plan, const Decomposition& dec, const CanonicalCoo& a, std::string& err) {
  release();
  have_pivots_ = false;
  last_reuse_ = false;
  plan_ = plan;
  DevPlan d{};
  d.n = plan.n;
  d.nunits = plan.nunits;
  d.nnz = plan.nnz;
  d.wait_limit = kWaitLimitDefault;
  if (!upload_vec(allocs_, dec.P, &d.P, err)) return false;
  if (!upload_vec(allocs_, dec.Q, &d.Q, err)) return false;
  if (!upload_vec(allocs_, plan.ustart, &d.ustart, err)) return false;
  if (!upload_vec(allocs_, plan.lu_off, &d.lu_off, err)) return false;
  if (!upload_vec(allocs_, plan.dent_ptr, &d.dent_ptr, err)) return false;
  if (!upload_vec(allocs_, plan.dent_pos, &d.dent_pos, err)) return false;
  if (!upload_vec(allocs_, plan.dent_src, &d.dent_src, err)) return false;
  if (!upload_vec(allocs_, plan.sdiag_src, &d.sdiag_src, err)) return false;
  if (!upload_vec(allocs_, plan.cpl_ptr, &d.cpl_ptr, err)) return false;
  if (!upload_vec(allocs_, plan.cpl_col, &d.cpl_col, err)) return false;
  if (!upload_vec(allocs_, plan.cpl_src, &d.cpl_src, err)) return false;
  if (!upload_vec(allocs_, plan.csr_ptr, &d.csr_ptr, err)) return false;
  if (!upload_vec(allocs_, a.col, &d.csr_col, err)) return false;
  if (!upload_vec(allocs_, plan.step_unit, &d.step_unit, err)) return false;
  if (!upload_vec(allocs_, plan.step_trsm_pref, &d.step_trsm_pref, err)) return false;
  if (!upload_vec(allocs_, plan.step_gemm_pref, &d.step_gemm_pref, err)) return false;
  if (!upload_vec(allocs_, plan.rstep_unit, &d.rstep_unit, err)) return false;
  if (!upload_vec(allocs_, plan.rstep_strip_pref, &d.rstep_strip_pref, err)) return false;
  if (!upload_vec(allocs_, plan.rstep_ga_pref, &d.rstep_ga_pref, err)) return false;
  if (!upload_vec(allocs_, plan.rstep_gb_pref, &d.rstep_gb_pref, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.rmax_active) * kRPanel * kRPanel, &d.dscratch, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.lu_size), &d.lu, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.n), &d.piv, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.n), &d.lperm, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.n), &d.liperm, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.n), &d.sdiag, err)) return false;
  if (!alloc_dev(allocs_, plan.cpl_col.size(), &d.cpl_val, err)) return false;
  if (!alloc_dev(allocs_, 2, &d.status, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(plan.nnz), &d_vals_, err)) return false;
  d_status_ = d.status;
  BDLU_CUDA(cudaMemset(d.status, 0, 2 * sizeof(int32_t)));
  BDLU_CUDA(cudaMemset(d.piv, 0, static_cast<size_t>(plan.n) * sizeof(int32_t)));
  dp_ = d;
  {
    // The dynamic shared-memory limit is a per-function process-wide
    // attribute; raise it once to the device maximum so handles of different
    // sizes never lower each other's limit.
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
      int dev = 0, optin = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      const int dyn = optin - 2048;
      attr_err = cudaFuncSetAttribute(k_lu_small<kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_lu_small<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_lu_small<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_solve_level<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_solve_level<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_solve_level<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_solve_level<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_solve_level<kSlots>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_lu_warp<2, kWarpLuW2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kWarpLuW2 * 64 * 64 * static_cast<int>(sizeof(double)));
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_lu_queue, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_lu_rows<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 64 * 8);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_lu_rows<96>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 96 * 8);
    });
    BDLU_CUDA(attr_err);
  }
  // Kernel attributes are set before any stream capture can start.
  BDLU_CUDA(large_setup());
  // Kernel work lists.
  const int32_t* small_list = nullptr;
  const int32_t* large_list = nullptr;
  const int32_t* lvl_scalar = nullptr;
  const int32_t* lvl_dense = nullptr;
  if (!upload_vec(allocs_, plan.small_units, &small_list, err)) return false;
  if (!upload_vec(allocs_, plan.large_units, &large_list, err)) return false;
  if (!upload_vec(allocs_, plan.lvl_scalar, &lvl_scalar, err)) return false;
  if (!upload_vec(allocs_, plan.lvl_dense, &lvl_dense, err)) return false;
  const int32_t* lvl_large = nullptr;
  if (!upload_vec(allocs_, plan.lvl_large, &lvl_large, err)) return false;
  lvl_large_ = lvl_large;
  const int32_t* tile0 = nullptr;
  if (!upload_vec(allocs_, plan.lvl_large_tile0, &tile0, err)) return false;
  lvl_large_tile0_ = tile0;
  sync_words_ = large_sync_words(plan);
  if (!alloc_dev(allocs_, static_cast<size_t>(sync_words_), &d_sync_, err)) return false;
  if (!alloc_dev(allocs_, 1, &d_nrhs_, err)) return false;
  if (plan.rtasks > 0) {
    if (!upload_vec(allocs_, plan.rtask, &d_rtask_, err)) return false;
    if (!alloc_dev(allocs_, static_cast<size_t>(plan.rt_words), &d_rwords_, err)) return false;
  }
  small_list_ = small_list;
  large_list_ = large_list;
  // Task queue of the one-launch small-unit LU: units largest first; units of
  // more than 32 rows one task each, smaller ones in packs of eight.
  queue_tasks_ = 0;
  if (!plan.small_units.empty()) {
    std::vector<int32_t> qunits(plan.small_units.rbegin(), plan.small_units.rend());
    std::vector<int32_t> qtasks;
    int64_t smem = 0;
    size_t i = 0;
    while (i < qunits.size()) {
      const int32_t u = qunits[i];
      const int32_t m = plan.ustart[static_cast<size_t>(u) + 1] - plan.ustart[static_cast<size_t>(u)];
      if (m > 32) {
        qtasks.push_back(static_cast<int32_t>(i));
        qtasks.push_back(0);
        smem = std::max<int64_t>(smem, static_cast<int64_t>(m) * m * 8);
        ++i;
      } else {
        const size_t cnt = std::min<size_t>(8, qunits.size() - i);
        qtasks.push_back(static_cast<int32_t>(i));
        qtasks.push_back(static_cast<int32_t>(cnt));
        smem = std::max<int64_t>(smem, 8 * 32 * 32 * 8);
        i += cnt;
      }
    }
    const int32_t* qu = nullptr;
    const int32_t* qt = nullptr;
    if (!upload_vec(allocs_, qunits, &qu, err)) return false;
    if (!upload_vec(allocs_, qtasks, &qt, err)) return false;
    if (!alloc_dev(allocs_, 1, &d_qticket_, err)) return false;
    d_qunits_ = qu;
    d_qtasks_ = qt;
    queue_tasks_ = static_cast<int32_t>(qtasks.size() / 2);
    queue_smem_ = static_cast<size_t>(smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_queue, kQueueThreads, queue_smem_);
    queue_grid_ = std::max(1, std::min(queue_tasks_, num_sms_ * std::max(1, per_sm)));
  }
  lvl_scalar_ = lvl_scalar;
  lvl_dense_ = lvl_dense;
  if (!plan.sparse_units.empty()) {
    BDLU_CUDA(gp_setup());
    GpDev& g = gp_;
    if (!upload_vec(allocs_, plan.sparse_units, &g.units, err)) return false;
    if (!upload_vec(allocs_, plan.gp_col0, &g.col0, err)) return false;
    if (!upload_vec(allocs_, plan.gp_cptr, &g.cptr, err)) return false;
    if (!upload_vec(allocs_, plan.gp_row, &g.row, err)) return false;
    if (!upload_vec(allocs_, plan.gp_dpos, &g.dpos, err)) return false;
    if (!upload_vec(allocs_, plan.gp_aptr, &g.aptr, err)) return false;
    if (!upload_vec(allocs_, plan.gp_arow, &g.arow, err)) return false;
    if (!upload_vec(allocs_, plan.gp_asrc, &g.asrc, err)) return false;
    if (!upload_vec(allocs_, plan.gp_lrp, &g.lrp, err)) return false;
    if (!upload_vec(allocs_, plan.gp_lci, &g.lci, err)) return false;
    if (!upload_vec(allocs_, plan.gp_lpos, &g.lpos, err)) return false;
    if (!upload_vec(allocs_, plan.gp_urp, &g.urp, err)) return false;
    if (!upload_vec(allocs_, plan.gp_uci, &g.uci, err)) return false;
    if (!upload_vec(allocs_, plan.gp_upos, &g.upos, err)) return false;
    if (!alloc_dev(allocs_, static_cast<size_t>(std::max<int64_t>(plan.gp_nnz, 1)), &g.val, err)) return false;
    if (!alloc_dev(allocs_, plan.sparse_units.size(), &g.gstat, err)) return false;
    g.maxm = plan.gp_maxm;
    g.wait_limit = dp_.wait_limit;
    if (!upload_vec(allocs_, plan.lvl_sparse, &lvl_sparse_, err)) return false;
  }
  return true;
}

void Engine::launch_lu_small(int threads, int32_t units, int32_t mb, cudaStream_t st, const double* d_vals,
                             const int32_t* list) {
  const size_t smem = static_cast<size_t>(mb) * mb * sizeof(double);
  if (threads == 32 && mb <= 32) {
    k_lu_warp<1, kWarpLuW1><<<(units + kWarpLuW1 - 1) / kWarpLuW1, 32 * kWarpLuW1, kWarpLuW1 * 32 * 32 * sizeof(double),
                              st>>>(dp_, d_vals, list, units);
    return;
  }
  if (threads == 32 && mb <= 64) {
    k_lu_warp<2, kWarpLuW2><<<(units + kWarpLuW2 - 1) / kWarpLuW2, 32 * kWarpLuW2, kWarpLuW2 * 64 * 64 * sizeof(double),
                              st>>>(dp_, d_vals, list, units);
    return;
  }
  if (threads == kLuRowsWidth && mb <= 64) {
    k_lu_rows<64><<<units, 64, smem, st>>>(dp_, d_vals, list);
    return;
  }
  if (threads == kLuRowsWidth && mb <= 96) {
    k_lu_rows<96><<<units, 96, smem, st>>>(dp_, d_vals, list);
    return;
  }
  if (threads == 64) k_lu_small<64><<<units, 64, smem, st>>>(dp_, d_vals, list);
  else if (threads == 128) k_lu_small<128><<<units, 128, smem, st>>>(dp_, d_vals, list);
  else k_lu_small<kThreads><<<units, kThreads, smem, st>>>(dp_, d_vals, list);
}

// The autotuner keeps one width per size class (the bucket cuts of the plan
// and the shared-memory limit), so buckets whose largest unit differs by a
// row share a choice.  Widths are still checked against the bucket's own mb.
static int32_t lu_bucket_class(int32_t mb) {
  static const int32_t kClass[] = {8, 16, 24, 32, 48, 64, 80, 96, 128};
  static const int32_t kMax = small_unit_max();
  for (int32_t c : kClass)
    if (mb <= c) return c;
  return kMax;
}

// Admissible widths of a bucket of units up to mb rows: 32 (one warp per
// unit, up to 64 rows), kLuRowsWidth (one thread per row, rows in registers,
// up to 96 rows), and CTA widths with one thread per row at least.
static bool lu_width_ok(int t, int32_t mb) {
  if (t == 32) return mb <= 64;
  if (t == kLuRowsWidth) return mb <= 96;
  return (t == 64 || t == 128 || t == kThreads) && t >= mb;
}

int Engine::lu_small_width(int32_t mb) const {
  // A width forced for this engine, the tuned choice, else the default rule:
  // narrow CTAs for small units (more units per SM, cheaper per-column
  // barriers).
  if (forced_lu_width_ != 0 && lu_width_ok(forced_lu_width_, mb)) return forced_lu_width_;
  const int t = Tuner::get().enabled() ? Tuner::get().lu_small_threads(lu_bucket_class(mb)) : 0;
  if (lu_width_ok(t, mb)) return t;
  return mb <= 32 ? 64 : (mb <= 64 ? 128 : kThreads);
}

// Times every admissible CTA width of each size bucket this GPU has no
// choice for yet, on the bucket's own units (one untimed and one timed
// launch each; the launches write the same factors the real one writes).
cudaError_t Engine::tune_lu_small(const double* d_vals, cudaStream_t stream) {
  const Plan& p = plan_;
  Tuner& tu = Tuner::get();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaSuccess;
  for (size_t bkt = 0; bkt < p.small_bucket_m.size() && e == cudaSuccess; ++bkt) {
    const int32_t mb = p.small_bucket_m[bkt];
    if (tu.lu_small_threads(lu_bucket_class(mb)) != 0) continue;
    if (!e0 && ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess)) break;
    const int32_t q0 = p.small_bucket_ptr[bkt], q1 = p.small_bucket_ptr[bkt + 1];
    int widths[5], count = 0;
    for (int t : {32, kLuRowsWidth, 64, 128, kThreads})
      if (lu_width_ok(t, mb)) widths[count++] = t;
    float ms[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    int best = widths[count - 1];
    float best_ms = 1e30f;
    for (int c = 0; c < count && e == cudaSuccess; ++c) {
      launch_lu_small(widths[c], q1 - q0, mb, stream, d_vals, small_list_ + q0);
      cudaEventRecord(e0, stream);
      launch_lu_small(widths[c], q1 - q0, mb, stream, d_vals, small_list_ + q0);
      cudaEventRecord(e1, stream);
      if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
      cudaEventElapsedTime(&ms[c], e0, e1);
      if (ms[c] < best_ms) {
        best_ms = ms[c];
        best = widths[c];
      }
    }
    if (e == cudaSuccess) tu.set_lu_small_threads(lu_bucket_class(mb), best, ms, widths, count);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

// The shared-memory LU of every small unit as one launch per size bucket
// (shared memory sized to the bucket), the buckets side by side on the
// auxiliary streams (forked from and joined back into `stream`), largest
// units first.
cudaError_t Engine::launch_small_buckets(const double* d_vals, cudaStream_t stream) {
  const Plan& p = plan_;
  cudaError_t e = cudaEventRecord(fork_ev_[0], stream);
  const size_t nbk = p.small_bucket_m.size();
  for (size_t q = 0; q < nbk && e == cudaSuccess; ++q) {
    const size_t bkt = nbk - 1 - q;
    cudaStream_t sb = aux_[q % kAux];
    if (q < static_cast<size_t>(kAux)) e = cudaStreamWaitEvent(sb, fork_ev_[0], 0);
    const int32_t q0 = p.small_bucket_ptr[bkt], q1 = p.small_bucket_ptr[bkt + 1];
    const int32_t mb = p.small_bucket_m[bkt];
    launch_lu_small(lu_small_width(mb), q1 - q0, mb, sb, d_vals, small_list_ + q0);
  }
  for (int q = 0; q < kAux && q < static_cast<int>(nbk) && e == cudaSuccess; ++q) {
    e = cudaEventRecord(aux_ev_[q], aux_[q]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, aux_ev_[q], 0);
  }
  return e == cudaSuccess ? cudaGetLastError() : e;
}

// The same factors in one persistent launch over the task queue (k_lu_queue).
cudaError_t Engine::launch_small_queue(const double* d_vals, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(d_qticket_, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return e;
  k_lu_queue<<<queue_grid_, kQueueThreads, queue_smem_, stream>>>(dp_, d_vals, d_qunits_,
                                                                 reinterpret_cast<const int2*>(d_qtasks_),
                                                                 queue_tasks_, d_qticket_);
  return cudaGetLastError();
}

// 0: per-bucket launches, 1: one persistent launch; forced for this engine,
// tuned for its pattern, else per-bucket.
int Engine::small_mode() const {
  if (queue_tasks_ <= 0) return 0;
  if (forced_small_mode_ >= 0) return forced_small_mode_;
  const int t = Tuner::get().enabled() ? Tuner::get().small_mode(pattern_key_) : -1;
  return t == 1 ? 1 : 0;
}

// Times both ways of launching the small units on this pattern (after the
// widths are tuned) once per pattern signature; both write the same factors.
cudaError_t Engine::tune_small_mode(const double* d_vals, cudaStream_t stream) {
  Tuner& tu = Tuner::get();
  if (forced_small_mode_ >= 0 || queue_tasks_ <= 0 || tu.small_mode(pattern_key_) >= 0) return cudaSuccess;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float ms[2] = {0.0f, 0.0f};
  for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
      if (rep == 1) e = cudaEventRecord(e0, stream);
      if (e == cudaSuccess) e = mode == 0 ? launch_small_buckets(d_vals, stream) : launch_small_queue(d_vals, stream);
      if (rep == 1 && e == cudaSuccess) e = cudaEventRecord(e1, stream);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[mode], e0, e1);
  }
  if (e == cudaSuccess) tu.set_small_mode(pattern_key_, ms[1] < ms[0] ? 1 : 0, ms[0], ms[1]);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return e;
}

bool Engine::factor_async(const double* d_vals, cudaStream_t stream, std::string& err, bool reuse_pivots) {
  const Plan& p = plan_;
  const bool reuse = reuse_pivots && have_pivots_ && !p.large_units.empty();
  last_reuse_ = reuse;
  BDLU_CUDA(cudaMemsetAsync(d_status_, 0, 2 * sizeof(int32_t), stream));
  BDLU_CUDA(cudaEventRecord(ev_[0], stream));
  const int64_t ncpl = static_cast<int64_t>(p.cpl_col.size());
  launches_factor_ = 1 + static_cast<int32_t>(p.small_bucket_m.size());
  k_gather<<<grid_for(std::max<int64_t>(ncpl, p.n), kThreads, num_sms_ * 8), kThreads, 0, stream>>>(dp_, d_vals, ncpl);
  BDLU_CUDA(cudaEventRecord(pev_[0], stream));
  // Sparse units on their own stream beside the dense ones, joined below.
  const int32_t nsparse = static_cast<int32_t>(p.sparse_units.size());
  if (nsparse > 0) {
    BDLU_CUDA(cudaEventRecord(gp_ev_[0], stream));
    BDLU_CUDA(cudaStreamWaitEvent(gp_stream_, gp_ev_[0], 0));
    BDLU_CUDA(cudaMemsetAsync(gp_.gstat, 0, static_cast<size_t>(nsparse) * sizeof(int32_t), gp_stream_));
    BDLU_CUDA(gp_factor_launch(gp_, nsparse, d_vals, d_status_, gp_stream_));
    BDLU_CUDA(cudaEventRecord(gp_ev_[1], gp_stream_));
  }
  // One launch per size bucket, shared memory sized to the bucket; the
  // buckets run side by side on the auxiliary streams (forked from and
  // joined back into `stream`), largest units first.
  if (!p.small_bucket_m.empty() && Tuner::get().enabled()) {
    // Tuning waits for its timing events: never inside a caller's capture.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BDLU_CUDA(cudaStreamIsCapturing(stream, &cap));
    if (cap == cudaStreamCaptureStatusNone) {
      BDLU_CUDA(tune_lu_small(d_vals, stream));
      BDLU_CUDA(tune_small_mode(d_vals, stream));
    }
  }
  if (!p.small_bucket_m.empty()) {
    if (small_mode() == 1) {
      BDLU_CUDA(launch_small_queue(d_vals, stream));
      launches_factor_ = 2;
    } else {
      BDLU_CUDA(launch_small_buckets(d_vals, stream));
    }
  }
  BDLU_CUDA(cudaEventRecord(pev_[1], stream));
  if (!p.large_units.empty() && reuse) {
    if (reuse_exec_ && (reuse_prec_ != prec_ || reuse_schedule_ != schedule_)) {
      cudaGraphExecDestroy(reuse_exec_);
      reuse_exec_ = nullptr;
    }
    if (!reuse_exec_ || d_vals != d_vals_) {
      if (d_vals != d_vals_) {
        err = "refactor with the stored pivot order reads the engine's value buffer";
        return false;
      }
      BDLU_CUDA(cudaStreamBeginCapture(cap_stream_, cudaStreamCaptureModeThreadLocal));
      int32_t n_launch = 0;
      cudaMemsetAsync(dp_.lu + p.lu_large_begin, 0,
                      static_cast<size_t>(p.lu_large_end - p.lu_large_begin) * sizeof(double), cap_stream_);
      cudaError_t ce = large_scatter_reuse(dp_, p, d_vals, large_list_, cap_stream_);
      if (ce == cudaSuccess) {
        if (prec_ == 0 && schedule_ == 1 && p.rtasks > 0)
          ce = large_refactor_dag(dp_, p, d_rtask_, d_rwords_, cap_stream_, &n_launch);
        else
          ce = large_refactor(dp_, p, cap_stream_, cap_stream2_, fork_ev_[0], fork_ev_[1], &n_launch, prec_);
      }
      cudaGraph_t g = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(cap_stream_, &g);
      BDLU_CUDA(ce);
      BDLU_CUDA(ee);
      const cudaError_t ie = cudaGraphInstantiate(&reuse_exec_, g, cudaGraphInstantiateFlagUseNodePriority);
      cudaGraphDestroy(g);
      BDLU_CUDA(ie);
      reuse_launches_ = n_launch + 1;
      reuse_prec_ = prec_;
      reuse_schedule_ = schedule_;
    }
    BDLU_CUDA(cudaGraphLaunch(reuse_exec_, stream));
    launches_factor_ += reuse_launches_;
  } else if (!p.large_units.empty()) {
    BDLU_CUDA(cudaMemsetAsync(dp_.lu + p.lu_large_begin, 0,
                              static_cast<size_t>(p.lu_large_end - p.lu_large_begin) * sizeof(double), stream));
    k_scatter_large<<<dim3(64, static_cast<unsigned>(p.large_units.size())), kThreads, 0, stream>>>(dp_, d_vals,
                                                                                                 large_list_);
    ++launches_factor_;
    BDLU_CUDA(large_factor(dp_, p, large_list_, stream, &launches_factor_, prec_));
  }
  if (nsparse > 0) {
    BDLU_CUDA(cudaStreamWaitEvent(stream, gp_ev_[1], 0));
    ++launches_factor_;  // the sparse factor
  }
  BDLU_CUDA(cudaGetLastError());
  BDLU_CUDA(cudaEventRecord(ev_[1], stream));
  factor_timed_ = true;
  return true;
}

cudaError_t Engine::wait(cudaStream_t stream) {
  if (!blocking_sync_) return cudaStreamSynchronize(stream);
  // Record an event created with cudaEventBlockingSync and wait on it: the
  // calling thread sleeps instead of spinning on a core.
  if (!wait_ev_) {
    const cudaError_t e = cudaEventCreateWithFlags(&wait_ev_, cudaEventBlockingSync | cudaEventDisableTiming);
    if (e != cudaSuccess) {
      wait_ev_ = nullptr;
      return e;
    }
  }
  const cudaError_t e = cudaEventRecord(wait_ev_, stream);
  return e == cudaSuccess ? cudaEventSynchronize(wait_ev_) : e;
}

int Engine::factor_status(cudaStream_t stream, std::string& err) {
  int32_t st[2] = {0, 0};
  // Read back through the engine's page-locked words: a pageable
  // destination would go through the driver's shared staging buffers, which
  // serialises the status reads of concurrent requests.
  cudaError_t e = cudaMemcpyAsync(readback_, d_status_, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = wait(stream);
  if (e != cudaSuccess) {
    err = std::string("factor status: ") + cudaGetErrorString(e);
    return -1;
  }
  std::memcpy(st, readback_, sizeof(st));
  if (st[0] == kFailZeroPivot) {
    err = "block factorization failed: zero pivot in diagonal block " + std::to_string(st[1]);
    return 1;
  }
  if (st[0] == kFailReusedPivot) {
    err = "reused pivot order met a zero pivot in diagonal block " + std::to_string(st[1]);
    return 2;
  }
  if (st[0] == kFailSparseSync) {
    err = "sparse LU: a bounded wait between columns ran out";
    return -1;
  }
  if (st[0] == kFailSparseReject) {
    err = "sparse LU of diagonal block " + std::to_string(st[1]) + " failed its pivot test";
    return 3;
  }
  if (st[0] == kFailTensorSync) {
    err = "tensor-core update: a bounded wait for the tensor cores ran out";
    return -1;
  }
  if (st[0] == kFailRefactorSync) {
    // Only the tile-graph refactor (stored pivot order) sets this; the
    // caller redoes the factor with pivoting, which does not use it.
    err = "refactor task graph: a bounded wait between tiles ran out";
    return 2;
  }
  if (!last_reuse_) have_pivots_ = true;
  return 0;
}

bool Engine::sparse_rejections(std::vector<int32_t>& units, std::vector<int32_t>& reasons, std::string& err) {
  units.clear();
  reasons.clear();
  const size_t ns = plan_.sparse_units.size();
  if (ns == 0) return true;
  std::vector<int32_t> st(ns);
  BDLU_CUDA(cudaDeviceSynchronize());
  BDLU_CUDA(cudaMemcpy(st.data(), gp_.gstat, ns * sizeof(int32_t), cudaMemcpyDeviceToHost));
  for (size_t g = 0; g < ns; ++g)
    if (st[g] != 0) {
      units.push_back(plan_.sparse_units[g]);
      reasons.push_back(st[g]);
    }
  return true;
}

bool Engine::ensure_work(int32_t nrhs, std::string& err) {
  if (nrhs <= work_nrhs_) return true;
  // Work space grows to at least kWorkRhs columns at once: a reallocation
  // (cudaMalloc synchronises the device) and the graphs it invalidates are
  // paid once for the common right-hand-side counts.
  nrhs = std::max(nrhs, kWorkRhs);
  const size_t nn = static_cast<size_t>(plan_.n) * static_cast<size_t>(nrhs);
  for (void* q : {static_cast<void*>(d_b0_), static_cast<void*>(d_xp_), static_cast<void*>(d_r_),
                  static_cast<void*>(d_rhs_), static_cast<void*>(d_norms_)}) {
    if (!q) continue;
    cudaFree(q);
    allocs_.erase(std::remove_if(allocs_.begin(), allocs_.end(), [q](const std::pair<void*, size_t>& a) { return a.first == q; }),
                  allocs_.end());
  }
  if (!alloc_dev(allocs_, nn, &d_b0_, err)) return false;
  if (!alloc_dev(allocs_, nn, &d_xp_, err)) return false;
  if (!alloc_dev(allocs_, nn, &d_r_, err)) return false;
  if (!alloc_dev(allocs_, nn, &d_rhs_, err)) return false;
  if (!alloc_dev(allocs_, static_cast<size_t>(4 * nrhs), &d_norms_, err)) return false;
  work_nrhs_ = nrhs;
  return true;
}

size_t Engine::device_bytes() const {
  size_t b = 0;
  for (const auto& a : allocs_) b += a.second;
  return b;
}

double* Engine::value_staging(std::string& err) {
  if (!d_vals_stage_ && !alloc_dev(allocs_, static_cast<size_t>(std::max<int64_t>(plan_.nnz, 1)), &d_vals_stage_, err))
    return nullptr;
  return d_vals_stage_;
}

double* Engine::rhs_buffer(int32_t nrhs, std::string& err) {
  if (!ensure_work(nrhs, err)) return nullptr;
  return d_rhs_;
}

void Engine::solve_core(const double* rhs, int32_t ldr, double* xp, const int32_t* nrhs, bool wide,
                        cudaStream_t stream) {
  const Plan& p = plan_;
  const int32_t nl = p.umax_level + 1;
  if (p.large_tiles > 0) cudaMemsetAsync(d_sync_, 0, static_cast<size_t>(sync_words_) * sizeof(int32_t), stream);
  // Within a level the scalar rows and small dense units run as one launch
  // on `stream`; large units and sparse-LU units, when the level has any,
  // run on auxiliary streams forked from `stream` and joined back, so the
  // level costs about its slowest part instead of their sum.  From the
  // second level on the fused launch is a programmatic dependent of the
  // work before it (k_solve_level: its factor staging overlaps that work's
  // tail; it waits for all of it before reading any unknown).
  bool prev = false;  // a kernel of an earlier level precedes on `stream`
  for (int32_t l = 0; l < nl; ++l) {
    const int32_t s0 = p.lvl_scalar_ptr[static_cast<size_t>(l)], s1 = p.lvl_scalar_ptr[static_cast<size_t>(l) + 1];
    const int32_t d0 = p.lvl_dense_ptr[static_cast<size_t>(l)], d1 = p.lvl_dense_ptr[static_cast<size_t>(l) + 1];
    const int32_t g0 = p.lvl_large_ptr[static_cast<size_t>(l)], g1 = p.lvl_large_ptr[static_cast<size_t>(l) + 1];
    const int32_t q0 = p.lvl_sparse_ptr.empty() ? 0 : p.lvl_sparse_ptr[static_cast<size_t>(l)];
    const int32_t q1 = p.lvl_sparse_ptr.empty() ? 0 : p.lvl_sparse_ptr[static_cast<size_t>(l) + 1];
    const bool has_sd = s1 > s0 || d1 > d0, has_g = g1 > g0, has_p = q1 > q0;
    const int kinds = static_cast<int>(has_sd) + static_cast<int>(has_g) + static_cast<int>(has_p);
    cudaStream_t st_g = stream, st_p = stream;
    if (kinds > 1) {
      cudaEventRecord(fork_ev_[0], stream);
      int used = 0;
      if (has_g && has_sd) st_g = aux_[used++];
      if (has_p && (has_sd || has_g)) st_p = aux_[used++];
      for (int q = 0; q < used; ++q) cudaStreamWaitEvent(aux_[q], fork_ev_[0], 0);
    }
    if (has_p) {
      ++launches_solve_;
      gp_solve_launch(dp_, gp_, lvl_sparse_ + q0, q1 - q0, rhs, ldr, xp, nrhs, st_p);
    }
    if (has_sd) {
      ++launches_solve_;
      const size_t mm = static_cast<size_t>(p.lvl_dense_maxm[static_cast<size_t>(l)]);
      const size_t smem = mm * mm * sizeof(double) + 16;
      const int32_t nsr = s1 - s0, nu = d1 - d0;
      const int32_t scal_ctas =
          nsr > 0 ? std::min<int32_t>((nsr + kThreads / 32 - 1) / (kThreads / 32), 4 * num_sms_) : 0;
      cudaLaunchAttribute attr{};
      attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr.val.programmaticStreamSerializationAllowed = 1;
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(static_cast<unsigned>(scal_ctas + nu));
      cfg.blockDim = dim3(kThreads);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = stream;
      cfg.attrs = &attr;
      cfg.numAttrs = (prev && pdl_) ? 1 : 0;
      const int32_t* sl = lvl_scalar_ + s0;
      const int32_t* dl = lvl_dense_ + d0;
      switch ((mm + 31) / 32) {
        case 0:
        case 1: cudaLaunchKernelEx(&cfg, k_solve_level<1>, dp_, sl, nsr, scal_ctas, dl, rhs, ldr, xp, nrhs); break;
        case 2: cudaLaunchKernelEx(&cfg, k_solve_level<2>, dp_, sl, nsr, scal_ctas, dl, rhs, ldr, xp, nrhs); break;
        case 3: cudaLaunchKernelEx(&cfg, k_solve_level<3>, dp_, sl, nsr, scal_ctas, dl, rhs, ldr, xp, nrhs); break;
        case 4: cudaLaunchKernelEx(&cfg, k_solve_level<4>, dp_, sl, nsr, scal_ctas, dl, rhs, ldr, xp, nrhs); break;
        default:
          cudaLaunchKernelEx(&cfg, k_solve_level<kSlots>, dp_, sl, nsr, scal_ctas, dl, rhs, ldr, xp, nrhs);
          break;
      }
      prev = true;
    }
    large_solve_level(dp_, p, l, lvl_large_, lvl_large_tile0_, d_sync_, rhs, ldr, xp, nrhs, wide, st_g,
                      &launches_solve_);
    if (kinds > 1) {
      int q = 0;
      for (cudaStream_t sx : {st_g, st_p}) {
        if (sx == stream) continue;
        cudaEventRecord(aux_ev_[q], sx);
        cudaStreamWaitEvent(stream, aux_ev_[q], 0);
        ++q;
      }
    }
    if (has_g || has_p) prev = true;
  }
}

bool Engine::solve_async(double* d_B, int32_t ldb, int32_t nrhs, int32_t refine_iters, cudaStream_t stream,
                         std::string& err) {
  if (!ensure_work(nrhs, err)) return false;
  const int32_t n = plan_.n;
  BDLU_CUDA(cudaEventRecord(ev_[2], stream));
  launches_solve_ = 3 + 3 * refine_iters;  // unpermute + residual (+ per step residual, unpermute) below
  BDLU_CUDA(cudaMemcpy2DAsync(d_b0_, static_cast<size_t>(n) * sizeof(double), d_B,
                              static_cast<size_t>(ldb) * sizeof(double), static_cast<size_t>(n) * sizeof(double),
                              static_cast<size_t>(nrhs), cudaMemcpyDeviceToDevice, stream));
  // The sweep's kernels read the right-hand-side count from d_nrhs_, so one
  // graph per tile-kernel width (up to 8 and up to 16 right-hand sides per
  // pass), captured on the current work buffers, serves every count.
  k_solve_begin<<<1, 1, 0, stream>>>(d_nrhs_, nrhs, d_status_);
  const int wide = nrhs > 8 ? 1 : 0;
  if (solve_exec_b0_ != d_b0_) {
    for (auto& ge : solve_exec_)
      if (ge) cudaGraphExecDestroy(ge);
    solve_exec_[0] = solve_exec_[1] = nullptr;
    solve_exec_b0_ = d_b0_;
  }
  if (!solve_exec_[wide]) {
    const int32_t saved = launches_solve_;
    BDLU_CUDA(cudaStreamBeginCapture(cap_stream_, cudaStreamCaptureModeThreadLocal));
    solve_core(d_b0_, n, d_xp_, d_nrhs_, wide != 0, cap_stream_);
    cudaGraph_t g = nullptr;
    BDLU_CUDA(cudaStreamEndCapture(cap_stream_, &g));
    const cudaError_t ie = cudaGraphInstantiate(&solve_exec_[wide], g, 0);
    cudaGraphDestroy(g);
    BDLU_CUDA(ie);
    solve_exec_launches_[wide] = launches_solve_ - saved;
    launches_solve_ = saved;
  }
  BDLU_CUDA(cudaGraphLaunch(solve_exec_[wide], stream));
  launches_solve_ += solve_exec_launches_[wide] + 1;
  const int ug = grid_for(static_cast<int64_t>(n) * nrhs, kThreads, num_sms_ * 16);
  k_unpermute<<<ug, kThreads, 0, stream>>>(dp_.Q, n, d_xp_, d_B, ldb, nrhs, 0);
  BDLU_CUDA(cudaEventRecord(pev_[2], stream));
  const int rg = grid_for(static_cast<int64_t>(n) * kResLanes, kThreads, num_sms_ * 8);
  for (int32_t it = 0; it < refine_iters; ++it) refine_core(d_B, ldb, nrhs, stream);
  BDLU_CUDA(cudaMemsetAsync(d_norms_, 0, static_cast<size_t>(4 * nrhs) * sizeof(unsigned long long), stream));
  k_residual<<<rg, kThreads, 0, stream>>>(dp_, d_vals_, d_B, ldb, d_b0_, n, nullptr, nrhs, d_norms_);
  BDLU_CUDA(cudaGetLastError());
  BDLU_CUDA(cudaEventRecord(ev_[3], stream));
  last_nrhs_ = nrhs;
  solve_timed_ = true;
  return true;
}

void Engine::refine_core(double* d_B, int32_t ldb, int32_t nrhs, cudaStream_t stream) {
  const int32_t n = plan_.n;
  const int ug = grid_for(static_cast<int64_t>(n) * nrhs, kThreads, num_sms_ * 16);
  const int rg = grid_for(static_cast<int64_t>(n) * kResLanes, kThreads, num_sms_ * 8);
  cudaMemsetAsync(d_norms_, 0, static_cast<size_t>(4 * nrhs) * sizeof(unsigned long long), stream);
  k_residual<<<rg, kThreads, 0, stream>>>(dp_, d_vals_, d_B, ldb, d_b0_, n, d_r_, nrhs, d_norms_);
  solve_core(d_r_, n, d_xp_, d_nrhs_, nrhs > 8, stream);
  k_unpermute<<<ug, kThreads, 0, stream>>>(dp_.Q, n, d_xp_, d_B, ldb, nrhs, 1);
  launches_solve_ += 3;
}

bool Engine::refine_async(double* d_B, int32_t ldb, int32_t nrhs, cudaStream_t stream, std::string& err) {
  const int32_t n = plan_.n;
  const int rg = grid_for(static_cast<int64_t>(n) * kResLanes, kThreads, num_sms_ * 8);
  k_set_i32<<<1, 1, 0, stream>>>(d_nrhs_, nrhs);
  refine_core(d_B, ldb, nrhs, stream);
  BDLU_CUDA(cudaMemsetAsync(d_norms_, 0, static_cast<size_t>(4 * nrhs) * sizeof(unsigned long long), stream));
  k_residual<<<rg, kThreads, 0, stream>>>(dp_, d_vals_, d_B, ldb, d_b0_, n, nullptr, nrhs, d_norms_);
  BDLU_CUDA(cudaGetLastError());
  launches_solve_ += 2;
  last_nrhs_ = nrhs;
  return true;
}

bool Engine::last_residual(cudaStream_t stream, SolveResidual& out, std::string& err) {
  out = SolveResidual{0, 0, 0, 0};
  if (last_nrhs_ <= 0) return true;
  int32_t st[2] = {0, 0};
  // Status and norms through page-locked words (see factor_status); norms of
  // more right-hand sides than they hold go through a host vector.
  const size_t nn = static_cast<size_t>(4 * last_nrhs_);
  std::vector<unsigned long long> h;
  unsigned long long* hn = reinterpret_cast<unsigned long long*>(readback_ + 32);
  if (nn > kReadbackNorms) {
    h.resize(nn);
    hn = h.data();
  }
  BDLU_CUDA(cudaMemcpyAsync(readback_, d_status_, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
  BDLU_CUDA(cudaMemcpyAsync(hn, d_norms_, nn * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
  BDLU_CUDA(wait(stream));
  std::memcpy(st, readback_, sizeof(st));
  if (st[0] == kFailSync) {
    err = "solve failed: a bounded wait between solve tiles ran out";
    return false;
  }
  double worst = -1.0;
  for (int32_t k = 0; k < last_nrhs_; ++k) {
    double v[4];
    std::memcpy(v, hn + 4 * k, sizeof(v));
    const double denom = v[3] * v[2] + v[1];
    const double rel = denom > 0.0 ? v[0] / denom : v[0];
    if (rel > worst) {
      worst = rel;
      out = SolveResidual{v[0], v[1], v[2], v[3]};
    }
  }
  return true;
}

void Engine::phase_ms(float out[kPhases]) {
  for (int i = 0; i < kPhases; ++i) out[i] = 0.0f;
  if (factor_timed_ && cudaEventSynchronize(ev_[1]) == cudaSuccess) {
    cudaEventElapsedTime(&out[0], ev_[0], pev_[0]);
    cudaEventElapsedTime(&out[1], pev_[0], pev_[1]);
    cudaEventElapsedTime(&out[2], pev_[1], ev_[1]);
  }
  if (solve_timed_ && cudaEventSynchronize(ev_[3]) == cudaSuccess) {
    cudaEventElapsedTime(&out[3], ev_[2], pev_[2]);
    cudaEventElapsedTime(&out[4], pev_[2], ev_[3]);
  }
}

float Engine::last_factor_ms() {
  float ms = 0.0f;
  if (factor_timed_ && cudaEventSynchronize(ev_[1]) == cudaSuccess) cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
  return ms;
}

float Engine::last_solve_ms() {
  float ms = 0.0f;
  if (solve_timed_ && cudaEventSynchronize(ev_[3]) == cudaSuccess) cudaEventElapsedTime(&ms, ev_[2], ev_[3]);
  return ms;
}

bool Engine::download_unit(int32_t u, std::vector<double>& lu, std::vector<int32_t>& piv, double& scalar,
                           std::string& err) {
  if (u < 0 || u >= plan_.nunits) {
    err = "unit index out of range";
    return false;
  }
  const int32_t s = plan_.ustart[static_cast<size_t>(u)];
  const int32_t m = plan_.ustart[static_cast<size_t>(u) + 1] - s;
  BDLU_CUDA(cudaDeviceSynchronize());
  if (plan_.ukind[static_cast<size_t>(u)] == kUnitScalar) {
    BDLU_CUDA(cudaMemcpy(&scalar, dp_.sdiag + s, sizeof(double), cudaMemcpyDeviceToHost));
    lu.assign(1, scalar);
    piv.assign(1, 0);
    return true;
  }
  lu.resize(static_cast<size_t>(m) * m);
  piv.resize(static_cast<size_t>(m));
  if (plan_.ukind[static_cast<size_t>(u)] == kUnitSparse) {
    // Expand the column-compressed factor; no row was swapped.
    const int32_t g = plan_.gp_index[static_cast<size_t>(u)];
    const int32_t c0 = plan_.gp_col0[static_cast<size_t>(g)];
    const int32_t e0 = plan_.gp_cptr[static_cast<size_t>(c0)], e1 = plan_.gp_cptr[static_cast<size_t>(c0 + m)];
    std::vector<double> v(static_cast<size_t>(e1 - e0));
    BDLU_CUDA(cudaMemcpy(v.data(), gp_.val + e0, v.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::fill(lu.begin(), lu.end(), 0.0);
    for (int32_t j = 0; j < m; ++j)
      for (int32_t q = plan_.gp_cptr[static_cast<size_t>(c0 + j)]; q < plan_.gp_cptr[static_cast<size_t>(c0 + j) + 1]; ++q)
        lu[static_cast<size_t>(j) * m + plan_.gp_row[static_cast<size_t>(q)]] = v[static_cast<size_t>(q - e0)];
    for (int32_t k = 0; k < m; ++k) piv[static_cast<size_t>(k)] = k;
    return true;
  }
  BDLU_CUDA(cudaMemcpy(lu.data(), dp_.lu + plan_.lu_off[static_cast<size_t>(u)], lu.size() * sizeof(double),
                       cudaMemcpyDeviceToHost));
  if (plan_.ukind[static_cast<size_t>(u)] == kUnitLarge) {
    // Large units are stored row-major; hand out column-major like the rest.
    std::vector<double> t(lu.size());
    for (int32_t i = 0; i < m; ++i)
      for (int32_t j = 0; j < m; ++j) t[static_cast<size_t>(j) * m + i] = lu[static_cast<size_t>(i) * m + j];
    lu.swap(t);
  }
  BDLU_CUDA(cudaMemcpy(piv.data(), dp_.piv + s, piv.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return true;
}

}  // namespace bdlu
