// pmg.h -- multigrid preconditioner (p-levels + aggregation levels) for scalar DG Jacobians.
#pragma once
#include <cuda_runtime.h>

#include "bosss_b200.h"

namespace bosss {
// V-cycle hierarchy of the cell-block Jacobian A of the operator of h (scalar, whole grid)
int pmg_create(const bosss_handle* h, const bosss_bsr* A, bosss_pmg** out);
// x = M^-1 b (one V-cycle), device vectors, enqueued on s
int pmg_apply(bosss_pmg* M, const double* b, double* x, cudaStream_t s);
void pmg_destroy(bosss_pmg* M);
}  // namespace bosss
