// bsr.h -- device storage of a block-sparse matrix (BlockMsrMatrix counterpart).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bosss_b200.h"

struct bosss_bsr {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t nbr = 0, nbc = 0, nnzb = 0;
    int br = 0, bc = 0;
    int64_t* d_rowptr = nullptr;
    int32_t* d_colidx = nullptr;
    double* d_vals = nullptr;   // blocks stored column-major
    float* d_vals32 = nullptr;  // FP32 copy for the inner solves of the mixed-precision refinement
    double* dx = nullptr;
    double* dy = nullptr;
    // sliced-ELL copy for the SpMV (built on the first product, spmv.cu): `ell_w` block slots
    // per block row; ell_col[s * nbr + i] the block column of slot s of row i (padding: column
    // 0, zero block); values in slices of 32 scalar rows, per slice slot-major then column
    int ell_w = 0;
    int32_t* d_ell_col = nullptr;
    double* d_ell_vals = nullptr;
};

namespace bosss {
// y = beta y + alpha A x on `s` (device vectors)
int bsr_spmv(bosss_bsr* A, double alpha, const double* x, double beta, double* y, cudaStream_t s);
}  // namespace bosss
