// Batched dense factor + solve that allocates no memory.
//
// Who needs it: callers that may not allocate device memory at the point
// where they solve -- code running under an allocator or memory budget that
// is closed after start-up, real-time loops that cannot absorb cudaMalloc's
// latency or its implicit synchronisation, and libraries called back from
// inside another framework's step that must not grow the device footprint.
// The handle-based API (bdlu_create / bdlu_analyze / ...) allocates its
// per-pattern device structures; this entry point instead keeps its scratch
// (LU factors, pivots, per-matrix failure flags, a status word) in one file-scope static device array
// that is part of the library image: every GPU that loads the library holds
// it (about 8.5 MiB) until the process exits.
//
// It is a variant of the engine's dense-unit path: the factor kernel is the
// same partial-pivoting LU as k_lu_small in engine.cu (first strict maximum,
// full-row swaps, multiply then subtract), reading a caller's dense matrix
// instead of scattered coordinates and writing the factors to the static
// scratch; the solve kernel applies the pivots and the L and U sweeps as
// k_solve_level does.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "bdlu.h"

namespace {

constexpr int kNaMaxM = 128;                      // rows of one matrix
constexpr long long kNaLuDoubles = 1LL << 20;     // batch * m * m <= 1,048,576 (8 MiB)
constexpr long long kNaPivInts = 1LL << 16;       // batch * m <= 65,536
constexpr long long kNaFlagInts = kNaPivInts;      // one failure flag per matrix (batch <= batch * m)
constexpr long long kNaScratchDoubles = kNaLuDoubles + kNaPivInts / 2 + kNaFlagInts / 2 + 32;
constexpr int kNaThreads = 256;
constexpr int kNaMaxDevices = 64;

// The scratch: [0, kNaLuDoubles) factors, then pivots (int32), then one
// failure flag per matrix (int32), then two int32 status words.  Host code
// must not use this name as an address.
static __device__ __align__(256) double g_noalloc_scratch[kNaScratchDoubles];

std::mutex g_na_mu;
double* g_na_addr[kNaMaxDevices] = {};

__device__ __forceinline__ void na_pivot_combine(double& best, int& bi, double ob, int oi, int none) {
  if (oi == none) return;
  if (bi == none || ob > best || (ob == best && oi < bi)) {
    best = ob;
    bi = oi;
  }
}

__device__ __forceinline__ void na_warp_pivot(double& best, int& bi, int none) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
    na_pivot_combine(best, bi, ob, oi, none);
  }
}

// One CTA per matrix: the matrix in shared memory, factors to the scratch.
// Every matrix writes its failure flag (0 or 1), so the flags need no
// clearing between calls.
__global__ void __launch_bounds__(kNaThreads) k_noalloc_lu(const double* __restrict__ A, int m, double* lu,
                                                           int32_t* piv_all, int32_t* failed, int32_t* status) {
  extern __shared__ double S[];
  __shared__ double s_best[kNaThreads / 32];
  __shared__ int s_bi[kNaThreads / 32];
  __shared__ int s_piv;
  __shared__ double s_pbest;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long mm = static_cast<long long>(m) * m;
  const double* a = A + blockIdx.x * mm;
  int32_t* piv = piv_all + static_cast<long long>(blockIdx.x) * m;
  for (int i = tid; i < mm; i += kNaThreads) S[i] = a[i];
  __syncthreads();
  for (int k = 0; k < m; ++k) {
    double* colk = S + static_cast<size_t>(k) * m;
    double best = 0.0;
    int bi = m;
    for (int i = k + tid; i < m; i += kNaThreads) {
      const double v = fabs(colk[i]);
      if (bi == m || v > best) {
        best = v;
        bi = i;
      }
    }
    na_warp_pivot(best, bi, m);
    if (lane == 0) {
      s_best[warp] = best;
      s_bi[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      best = (lane < kNaThreads / 32) ? s_best[lane] : 0.0;
      bi = (lane < kNaThreads / 32) ? s_bi[lane] : m;
      na_warp_pivot(best, bi, m);
      if (lane == 0) {
        s_piv = bi;
        s_pbest = best;
      }
    }
    __syncthreads();
    const int p = s_piv;
    // A zero or NaN pivot magnitude fails the matrix.
    if (!(s_pbest > 0.0)) {
      if (tid == 0) {
        failed[blockIdx.x] = 1;
        if (atomicCAS(status, 0, 1) == 0) status[1] = blockIdx.x;
      }
      return;
    }
    if (tid == 0) piv[k] = p;
    if (p != k) {
      for (int j = tid; j < m; j += kNaThreads) {
        double* c = S + static_cast<size_t>(j) * m;
        const double t = c[k];
        c[k] = c[p];
        c[p] = t;
      }
    }
    __syncthreads();
    const double akk = colk[k];
    for (int i = k + 1 + tid; i < m; i += kNaThreads) colk[i] = __ddiv_rn(colk[i], akk);
    __syncthreads();
    const int r = m - k - 1;
    for (int t = tid; t < r * r; t += kNaThreads) {
      const int jj = t / r, ii = t - jj * r;
      double* c = S + static_cast<size_t>(k + 1 + jj) * m;
      c[k + 1 + ii] = __dsub_rn(c[k + 1 + ii], __dmul_rn(colk[k + 1 + ii], c[k]));
    }
    __syncthreads();
  }
  double* out = lu + blockIdx.x * mm;
  for (int i = tid; i < mm; i += kNaThreads) out[i] = S[i];
  if (tid == 0) failed[blockIdx.x] = 0;
}

// One CTA per (matrix, right-hand side).  B and X may be the same buffer.
// A matrix whose factorisation failed is skipped: its X block is not written.
__global__ void __launch_bounds__(kNaThreads) k_noalloc_solve(const double* __restrict__ lu_all,
                                                              const int32_t* __restrict__ piv_all,
                                                              const int32_t* __restrict__ failed, int m, int nrhs,
                                                              const double* B, double* X) {
  __shared__ double x[kNaMaxM];
  const int mat = blockIdx.x / nrhs, col = blockIdx.x - (blockIdx.x / nrhs) * nrhs;
  if (failed[mat] != 0) return;  // CTA-uniform
  const long long base = (static_cast<long long>(mat) * nrhs + col) * m;
  const double* LU = lu_all + static_cast<long long>(mat) * m * m;
  const int32_t* piv = piv_all + static_cast<long long>(mat) * m;
  const int tid = threadIdx.x;
  for (int i = tid; i < m; i += kNaThreads) x[i] = B[base + i];
  __syncthreads();
  if (tid == 0)
    for (int i = 0; i < m; ++i) {
      const int p = piv[i];
      if (p != i) {
        const double t = x[i];
        x[i] = x[p];
        x[p] = t;
      }
    }
  __syncthreads();
  for (int j = 0; j < m - 1; ++j) {
    const double xj = x[j];
    const double* lc = LU + static_cast<size_t>(j) * m;
    for (int i = j + 1 + tid; i < m; i += kNaThreads) x[i] = fma(-lc[i], xj, x[i]);
    __syncthreads();
  }
  for (int j = m - 1; j >= 0; --j) {
    const double* uc = LU + static_cast<size_t>(j) * m;
    const double xj = x[j] / uc[j];
    for (int i = tid; i < j; i += kNaThreads) x[i] = fma(-uc[i], xj, x[i]);
    __syncthreads();
    if (tid == 0) x[j] = xj;
    __syncthreads();
  }
  for (int i = tid; i < m; i += kNaThreads) X[base + i] = x[i];
}

int na_fail(int code, char* msg, int64_t len, const char* text) {
  if (msg && len > 0) {
    std::strncpy(msg, text, static_cast<size_t>(len - 1));
    msg[len - 1] = '\0';
  }
  return code;
}

}  // namespace

extern "C" int bdlu_dense_batch_solve_noalloc(const double* d_A, int32_t m, int32_t batch, const double* d_B,
                                              double* d_X, int32_t nrhs, void* stream, char* msg, int64_t msg_len) {
  if (msg && msg_len > 0) msg[0] = '\0';
  if (!d_A || !d_B || !d_X || m < 1 || batch < 1 || nrhs < 1)
    return na_fail(BDLU_INVALID_DIMENSION, msg, msg_len, "null buffer or non-positive m, batch or nrhs");
  if (m > kNaMaxM)
    return na_fail(BDLU_INVALID_DIMENSION, msg, msg_len, "m exceeds the no-allocation limit of 128 rows");
  if (static_cast<long long>(batch) * m * m > kNaLuDoubles)
    return na_fail(BDLU_INVALID_DIMENSION, msg, msg_len,
                   "batch * m * m exceeds the no-allocation limit of 1048576 factor entries");
  if (static_cast<long long>(batch) * m > kNaPivInts)
    return na_fail(BDLU_INVALID_DIMENSION, msg, msg_len, "batch * m exceeds the no-allocation limit of 65536 rows");
  if (static_cast<long long>(batch) * nrhs > 2147483647LL)
    return na_fail(BDLU_INVALID_DIMENSION, msg, msg_len, "batch * nrhs too large");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices)
    return na_fail(BDLU_BACKEND_UNAVAILABLE, msg, msg_len, "no usable current CUDA device");
  double* base = nullptr;
  {
    // First call on this device: resolve the scratch's device address (the
    // array's name is only a host-side stand-in) and raise the factor
    // kernel's shared-memory limit, with this device current.
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return na_fail(BDLU_BACKEND_UNAVAILABLE, msg, msg_len, buf);
      }
      e = cudaFuncSetAttribute(k_noalloc_lu, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kNaMaxM * kNaMaxM * static_cast<int>(sizeof(double)));
      if (e != cudaSuccess) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
        return na_fail(BDLU_BACKEND_UNAVAILABLE, msg, msg_len, buf);
      }
      g_na_addr[dev] = static_cast<double*>(p);
    }
    base = g_na_addr[dev];
  }
  auto* s = static_cast<cudaStream_t>(stream);
  double* lu = base;
  auto* piv = reinterpret_cast<int32_t*>(base + kNaLuDoubles);
  auto* failed = reinterpret_cast<int32_t*>(base + kNaLuDoubles + kNaPivInts / 2);
  auto* status = reinterpret_cast<int32_t*>(base + kNaLuDoubles + kNaPivInts / 2 + kNaFlagInts / 2);
  // The scratch keeps the previous call's contents; only the status words
  // must start at zero (factors, pivots and failure flags are rewritten for
  // every matrix of the call before the solve reads them).
  cudaError_t e = cudaMemsetAsync(status, 0, 2 * sizeof(int32_t), s);
  if (e == cudaSuccess) {
    k_noalloc_lu<<<batch, kNaThreads, static_cast<size_t>(m) * m * sizeof(double), s>>>(d_A, m, lu, piv, failed,
                                                                                         status);
    k_noalloc_solve<<<batch * nrhs, kNaThreads, 0, s>>>(lu, piv, failed, m, nrhs, d_B, d_X);
    e = cudaGetLastError();
  }
  int32_t h_status[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_status, status, sizeof(h_status), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "CUDA error: %s", cudaGetErrorString(e));
    return na_fail(BDLU_SOLVE_FAILED, msg, msg_len, buf);
  }
  if (h_status[0] != 0) {
    char buf[128];
    std::snprintf(buf, sizeof(buf), "zero pivot in matrix %d", h_status[1]);
    return na_fail(BDLU_FACTORIZATION_FAILED, msg, msg_len, buf);
  }
  return BDLU_OK;
}
