// Device side of the sparse-LU route (gp.h): the device view of the plan's
// sparse-unit tables and the launches of the numeric factor and the solve.
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>

#include "engine.h"
#include "gp.h"

namespace bdlu {

// Kernel attributes (dynamic shared memory); once per process.
cudaError_t gp_setup();

// Numeric factor of all `count` sparse units from canonical values `vals`.
// A unit whose pivot test fails gets gstat[g] = reason (1 zero pivot, 2 the
// reference would swap rows, 3 tiny pivot, 4 below min_abs_diag) and
// status[0] = kFailSparseReject, status[1] = its unit id (first one wins); a
// bounded wait between columns that runs out records kGpReasonSync and
// kFailSparseSync instead.
cudaError_t gp_factor_launch(const GpDev& g, int32_t count, const double* vals, int32_t* status,
                             cudaStream_t stream);

// Solve of the sparse units glist[0 .. count) of one level: right-hand sides
// b - A_cpl x (coupling to later units), then the unit-lower and upper
// triangular sweeps.  A bounded wait that runs out records kFailSync in
// dp.status (the solve then fails like a large unit's tile solve).  Same conventions as the dense solves:
// rhs in original row order (ld ldr), xp in permuted order (ld n).
cudaError_t gp_solve_launch(const DevPlan& dp, const GpDev& g, const int32_t* glist, int32_t count,
                            const double* rhs, int32_t ldr, double* xp, const int32_t* nrhs, cudaStream_t stream);

}  // namespace bdlu
