// Large units: blocked LU and block-triangular solves (large.cu).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>

#include "engine.h"
#include "plan.h"

namespace bdlu {

cudaError_t large_setup();

// Enqueues the blocked LU of every large unit (slots already hold the unit
// values, row-major).  reuse = false: partial pivoting, then the final row
// orders (lperm/liperm).  reuse = true: the slots were filled by
// large_scatter_reuse in the stored row order and no pivot search is made; a
// zero or non-finite pivot sets status code 2.
// prec: 0 FP64 trailing updates; 1 TF32 tensor-core updates; 2 3xTF32.
cudaError_t large_factor(const DevPlan& dp, const Plan& p, const int32_t* d_large_units, cudaStream_t stream,
                         int32_t* launches, int32_t prec);

// Scatters the values of all large units into their (zeroed) slots with the
// rows in the stored pivot order.
cudaError_t large_scatter_reuse(const DevPlan& dp, const Plan& p, const double* d_vals, const int32_t* d_large_units,
                                cudaStream_t stream);

// Value-only refactor of all large units with the stored pivot order (rows
// already scattered in that order).  Work is queued on sa and sb (forked from
// and joined back into sa with the two events); zero or non-finite pivots set
// the reused-pivot status.
cudaError_t large_refactor(const DevPlan& dp, const Plan& p, cudaStream_t sa, cudaStream_t sb, cudaEvent_t ev_a,
                           cudaEvent_t ev_b, int32_t* launches, int32_t prec);

// The same refactor as one persistent kernel over the tile task graph of
// build_rtasks (p.rtask, uploaded to d_tasks; p.rtasks > 0).  d_words holds
// p.rt_words words (ticket and tile versions), zeroed here on the stream.
// Zero or non-finite pivots set the reused-pivot status; a wait that runs out
// sets kFailRefactorSync.
cudaError_t large_refactor_dag(const DevPlan& dp, const Plan& p, const int32_t* d_tasks, int32_t* d_words,
                               cudaStream_t stream, int32_t* launches);

// Forward and backward solves of the large units of one level (two
// launches).  d_sync holds large_sync_words(p) zeroed words per solve sweep;
// nrhs points to the right-hand-side count in device memory; wide selects the
// 16-per-pass kernels (for counts above 8).
cudaError_t large_solve_level(const DevPlan& dp, const Plan& p, int32_t level, const int32_t* d_units,
                              const int32_t* d_tile0, int32_t* d_sync, const double* rhs, int32_t ldr, double* xp,
                              const int32_t* nrhs, bool wide, cudaStream_t stream, int32_t* launches);

int32_t large_sync_words(const Plan& p);

}  // namespace bdlu
