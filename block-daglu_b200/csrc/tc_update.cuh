// Trailing updates of the mixed-precision route on the 5th-generation tensor
// cores (tcgen05): C -= L U for one 128 x TN tile of a large unit's
// row-major FP64 slot, K <= 64 deep.
//
// Per tile:
//   1. every thread stages L (128 x K) and U^T (TN x K) from FP64 into shared
//      memory as TF32 words (round to nearest; with split3 also the low
//      parts lo = tf32(x - hi)), in the canonical K-major layout without
//      swizzle that the tensor core reads through a shared-memory
//      descriptor: 8-row x 16-byte core matrices, the two K-halves of an
//      8-deep K slice LBO = 128 bytes apart, consecutive 8-row groups
//      SBO = 256 bytes apart, one K slice after another;
//   2. one thread issues the K/8 tcgen05.mma (kind::tf32, M = 128, N = TN,
//      FP32 accumulator in tensor memory; 3K/8 with split3: hi*hi + hi*lo +
//      lo*hi) and commits them to an mbarrier;
//   3. all threads wait on the mbarrier (bounded), read the accumulator
//      (tcgen05.ld, warp w reads lanes 32(w%4).. of its sub-partition) and
//      subtract it from C with coalesced FP64 read-modify-writes.  Square
//      tiles (TN = 128) are computed transposed, D^T = U^T L^T, so a
//      tensor-memory lane is a column of C: each thread updates its column
//      straight from its registers, a warp touching 32 consecutive columns
//      of one row at a time, and the first C rows are loaded before the
//      wait.  Other tiles pass the accumulator through shared memory and
//      update C row by row.
// The accumulator's tensor-memory columns are allocated once per CTA
// (tc_tmem_alloc) and freed before the CTA exits (tc_tmem_free).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"

namespace bdlu {

constexpr int kFailTensorSync = 5;  // a bounded wait for tensor-core work ran out
constexpr int kTcM = 128;           // tile rows (one tensor-memory lane per row)
constexpr int kTcThreads = 256;     // 8 warps: two per tensor-memory sub-partition
constexpr int kTcSpin = 1 << 22;    // polls of the completion barrier (~ tens of ms)

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, M = 128, N.
template <int N>
__host__ __device__ constexpr uint32_t tc_idesc_tf32() {
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N of an M = 128 tcgen05.mma");
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(kTcM >> 4) << 24);
}

__device__ __forceinline__ uint32_t tc_to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// Allocates `cols` tensor-memory columns (warp 0) and initialises the
// completion barrier (thread 0); every thread returns the column base.
template <int kCols>
__device__ __forceinline__ uint32_t tc_tmem_alloc(uint32_t* s_tmem, uint64_t* s_bar) {
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(s_tmem)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(s_bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return *reinterpret_cast<volatile uint32_t*>(s_tmem);
}

template <int kCols>
__device__ __forceinline__ void tc_tmem_free(uint32_t tmem) {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
  }
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                            uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

// Bounded wait for the barrier phase `parity`; false if it ran out.
__device__ __forceinline__ bool tc_wait(uint64_t* s_bar, uint32_t parity) {
  const uint32_t addr = tc_smem_addr(s_bar);
  for (int it = 0; it < kTcSpin; ++it) {
    uint32_t done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// Shared memory of one tile update: staged operands (hi, and lo with split3);
// the accumulator pass-through of non-square tiles reuses the same bytes.
template <int K, int TN>
__host__ __device__ constexpr size_t tc_smem_bytes() {
  constexpr size_t ops = 2 * (static_cast<size_t>(kTcM) * K * 4 + static_cast<size_t>(TN) * K * 4);
  // (square tiles read the accumulator straight from tensor memory)
  constexpr size_t acc = TN == kTcM ? 0 : static_cast<size_t>(kTcM) * (TN + 1) * 4;
  return (ops > acc ? ops : acc) + 1024;  // + alignment slack of the dynamic base
}

// C = A[i0 : i0+128, j0 : j0+TN] -= A[i0 :, k0 : k0+kk] * A[k0 : k0+kk, j0 :]
// on a row-major m x m FP64 block (kk <= K; rows/columns past m are skipped).
// `smem` is 1024-byte aligned, tc_smem_bytes<K, TN>() long; `parity` is the
// barrier phase this call waits for (flipped on return).  Returns false if
// the tensor-core work did not complete within the bound (C is untouched).
template <int K, int TN>
__device__ bool tile_update_tc(double* A, int m, int i0, int j0, int k0, int kk, bool split3, uint8_t* smem,
                               uint32_t tmem, uint64_t* s_bar, uint32_t& parity) {
  static_assert(K % 8 == 0 && K <= 64, "K slices of 8");
  static_assert(TN == 64 || TN == 128, "tile width");
  constexpr uint32_t kAChunk = kTcM * 32;  // bytes of one 8-deep K slice of A
  constexpr uint32_t kBChunk = TN * 32;
  constexpr uint32_t kABytes = kTcM * K * 4;
  constexpr uint32_t kBBytes = TN * K * 4;
  uint8_t* Ah = smem;
  uint8_t* Bh = Ah + kABytes;
  uint8_t* Al = Bh + kBBytes;
  uint8_t* Bl = Al + kABytes;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = kTcThreads / 32;
  // Square tiles keep the accumulator transposed (lane = column of C), so
  // each thread owns one column and a warp's C accesses are whole rows.
  constexpr bool kColMajorAcc = TN == kTcM;
  // Stage: one warp per core matrix (8 rows x 4 K), lane = row%8 * 4 + k%4,
  // so a warp writes 128 contiguous bytes.  Each warp first issues the loads
  // of kBatch core matrices (read-only path: the panels do not change during
  // the launch), then converts and stores them, so the loads overlap.
  constexpr int kQG = K / 4;
  constexpr int kBatch = 8;
  constexpr int kBlocksA = (kTcM / 8) * kQG, kBlocksB = (TN / 8) * kQG;
  static_assert(kBlocksA % (kWarps * kBatch) == 0 && kBlocksB % (kWarps * kBatch) == 0, "staging batches");
  for (int b0 = warp; b0 < kBlocksA; b0 += kWarps * kBatch) {
    double v[kBatch];
#pragma unroll
    for (int t = 0; t < kBatch; ++t) {
      const int b = b0 + t * kWarps;
      const int rg = b / kQG, qg = b - rg * kQG;
      const int r = rg * 8 + (lane >> 2), q = qg * 4 + (lane & 3);
      v[t] = (i0 + r < m && q < kk) ? __ldg(A + static_cast<size_t>(i0 + r) * m + k0 + q) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < kBatch; ++t) {
      const int b = b0 + t * kWarps;
      const int rg = b / kQG, qg = b - rg * kQG;
      const int q = qg * 4 + (lane & 3);
      const float f = static_cast<float>(v[t]);
      const uint32_t h = tc_to_tf32(f);
      const uint32_t off = (q >> 3) * kAChunk + rg * 256 + ((q >> 2) & 1) * 128 + lane * 4;
      *reinterpret_cast<uint32_t*>(Ah + off) = h;
      if (split3) *reinterpret_cast<uint32_t*>(Al + off) = tc_to_tf32(f - __uint_as_float(h));
    }
  }
  for (int b0 = warp; b0 < kBlocksB; b0 += kWarps * kBatch) {
    double v[kBatch];
#pragma unroll
    for (int t = 0; t < kBatch; ++t) {
      const int b = b0 + t * kWarps;
      const int ng = b / kQG, qg = b - ng * kQG;
      const int n = ng * 8 + (lane >> 2), q = qg * 4 + (lane & 3);
      v[t] = (q < kk && j0 + n < m) ? __ldg(A + static_cast<size_t>(k0 + q) * m + j0 + n) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < kBatch; ++t) {
      const int b = b0 + t * kWarps;
      const int ng = b / kQG, qg = b - ng * kQG;
      const int q = qg * 4 + (lane & 3);
      const float f = static_cast<float>(v[t]);
      const uint32_t h = tc_to_tf32(f);
      const uint32_t off = (q >> 3) * kBChunk + ng * 256 + ((q >> 2) & 1) * 128 + lane * 4;
      *reinterpret_cast<uint32_t*>(Bh + off) = h;
      if (split3) *reinterpret_cast<uint32_t*>(Bl + off) = tc_to_tf32(f - __uint_as_float(h));
    }
  }
  // Generic-proxy writes become visible to the tensor core's async proxy.
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (tid == 0) {
    constexpr uint32_t idesc = tc_idesc_tf32<TN>();
    const uint32_t ah = tc_smem_addr(Ah), bh = tc_smem_addr(Bh), al = tc_smem_addr(Al), bl = tc_smem_addr(Bl);
    const int nk = (kk + 7) / 8;
    for (int kc = 0; kc < nk; ++kc) {
      const uint64_t dah = tc_desc(ah + kc * kAChunk, 128, 256);
      const uint64_t dbh = tc_desc(bh + kc * kBChunk, 128, 256);
      const uint64_t dal = tc_desc(al + kc * kAChunk, 128, 256);
      const uint64_t dbl = tc_desc(bl + kc * kBChunk, 128, 256);
      if constexpr (kColMajorAcc) {
        // D^T = U^T L^T: tensor-memory lane = column of C.
        tc_mma_tf32(tmem, dbh, dah, idesc, kc > 0 ? 1u : 0u);
        if (split3) {
          tc_mma_tf32(tmem, dbh, dal, idesc, 1u);
          tc_mma_tf32(tmem, dbl, dah, idesc, 1u);
        }
      } else {
        tc_mma_tf32(tmem, dah, dbh, idesc, kc > 0 ? 1u : 0u);
        if (split3) {
          tc_mma_tf32(tmem, dah, dbl, idesc, 1u);
          tc_mma_tf32(tmem, dal, dbh, idesc, 1u);
        }
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tc_smem_addr(s_bar))
                 : "memory");
  }
  if constexpr (kColMajorAcc) {
    // Thread (sub-partition s, lane l) owns column 32 s + l of the tile and
    // rows [64 h, 64 h + 64) (h = warp / 4), in chunks of kCh rows.  The first
    // chunk of C is loaded before the wait, so those loads overlap the MMAs.
    constexpr int kCh = 16, kNch = kTcM / 2 / kCh;
    const int sub = warp & 3, half = warp >> 2;
    const int jj = sub * 32 + lane;
    const bool colok = j0 + jj < m;
    double* colp = A + j0 + jj;
    const uint32_t tlane = tmem + (static_cast<uint32_t>(sub * 32) << 16);
    double cv[kCh];
    auto load_chunk = [&](int ch) {
      const int rb = i0 + half * (kTcM / 2) + ch * kCh;
#pragma unroll
      for (int t = 0; t < kCh; ++t)
        cv[t] = (colok && rb + t < m) ? colp[static_cast<size_t>(rb + t) * m] : 0.0;
    };
    load_chunk(0);
    bool ok = tc_wait(s_bar, parity);
    if (!ok) ok = tc_wait(s_bar, parity);
    parity ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!__syncthreads_and(ok)) return false;
#pragma unroll 1
    for (int ch = 0; ch < kNch; ++ch) {
      if (ch > 0) load_chunk(ch);
      const int r0 = half * (kTcM / 2) + ch * kCh;
      uint32_t v[kCh];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tlane + static_cast<uint32_t>(r0)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int rb = i0 + r0;
#pragma unroll
      for (int t = 0; t < kCh; ++t)
        if (colok && rb + t < m) colp[static_cast<size_t>(rb + t) * m] = cv[t] - static_cast<double>(__uint_as_float(v[t]));
    }
    // The next tile's MMAs overwrite the accumulator only after a barrier.
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    return true;
  }
  // Every thread waits; one that runs out waits once more (bounded) so no
  // tensor-core work is left reading shared memory, and the tile is skipped.
  bool ok = tc_wait(s_bar, parity);
  if (!ok) ok = tc_wait(s_bar, parity);
  parity ^= 1u;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!__syncthreads_and(ok)) return false;
  // Accumulator -> shared memory (row r = lane of the tensor memory).
  float* Cs = reinterpret_cast<float*>(smem);
  constexpr int kCS = TN + 1;
  const int sub = warp & 3, half = warp >> 2;
  const int r = sub * 32 + lane;
#pragma unroll
  for (int c0 = half * (TN / 2); c0 < (half + 1) * (TN / 2); c0 += 32) {
    uint32_t v[32];
    const uint32_t taddr = tmem + (static_cast<uint32_t>(sub * 32) << 16) + static_cast<uint32_t>(c0);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c = 0; c < 32; ++c) Cs[r * kCS + c0 + c] = __uint_as_float(v[c]);
  }
  // The next tile's MMAs overwrite the accumulator only after this barrier.
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  // C -= accumulator: warps along rows, lanes along a row (coalesced); each
  // warp loads the C entries of kRows rows before it subtracts and stores,
  // so those loads are in flight together.
  constexpr int kCols = TN / 32, kRows = 4;
  static_assert(kTcM % (kWarps * kRows) == 0, "epilogue row groups");
  for (int rr0 = warp; rr0 < kTcM; rr0 += kWarps * kRows) {
    double cv[kRows][kCols];
#pragma unroll
    for (int h = 0; h < kRows; ++h) {
      const int gi = i0 + rr0 + h * kWarps;
#pragma unroll
      for (int t = 0; t < kCols; ++t) {
        const int c = lane + 32 * t;
        cv[h][t] = (gi < m && j0 + c < m) ? A[static_cast<size_t>(gi) * m + j0 + c] : 0.0;
      }
    }
#pragma unroll
    for (int h = 0; h < kRows; ++h) {
      const int rr = rr0 + h * kWarps, gi = i0 + rr;
#pragma unroll
      for (int t = 0; t < kCols; ++t) {
        const int c = lane + 32 * t;
        if (gi < m && j0 + c < m)
          A[static_cast<size_t>(gi) * m + j0 + c] = cv[h][t] - static_cast<double>(Cs[rr * kCS + c]);
      }
    }
  }
  __syncthreads();  // Cs is the next tile's staging area
  return true;
}

}  // namespace bdlu
