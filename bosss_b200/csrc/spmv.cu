// spmv.cu -- block-sparse matrix-vector product y = beta y + alpha A x
// (BlockMsrMatrix.SpMV, BlockMsrMatrix.cs:2554-2990).
//
// The reference loops over block rows and calls dgemv per block (blocks >= 40 entries) or a
// scalar loop. Here the product is HBM-bound streaming of the block values: the matrix is
// copied once (at the first product) into a sliced-ELL layout with slices of 32 scalar rows
// (one warp): per slice, block slot s, block column c, the 32 rows' entries, so every load
// instruction of a warp reads 256 contiguous bytes and a warp walks its slice's values as one
// contiguous stream (a layout with one plane per (slot, column) over all rows makes each warp
// read 70 places 9 MB apart at the C3 k=2 pattern, which measured 15 % slower than the plain
// block-row kernel). One thread per scalar row; the threads of a block row read the same x
// entry (L1 broadcast), x itself is re-read from L2. Rows with fewer blocks than the widest
// row are padded with zero blocks (Cartesian DG patterns: boundary cells only). Matrices
// whose padding would exceed a quarter of the blocks keep the block-row kernel.
#include <algorithm>
#include <string>
#include <vector>

#include "bsr.h"

namespace bosss {

int fail(int code, const std::string& msg);

namespace {

constexpr int SLICE = 32;   // scalar rows per slice (one warp)

// BSR (column-major blocks) -> sliced ELL: ell_vals[((slice * w + s) * bc + c) * 32 + lane] =
// entry (r, c) of block slot s of the block row of scalar row slice * 32 + lane (0 past the
// last row or the row's last block); one thread per entry of the padded layout
__global__ void k_to_ell(long long nbr, int br, int bc, int w, const long long* __restrict__ rowptr,
                         const int* __restrict__ colidx, const double* __restrict__ vals, int* __restrict__ ell_col,
                         double* __restrict__ ell_vals) {
    const long long nrows = nbr * br, nsl = (nrows + SLICE - 1) / SLICE;
    const long long n = nsl * w * bc * SLICE;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int lane = (int)(t % SLICE);
        const long long q = t / SLICE;
        const int c = (int)(q % bc);
        const long long q2 = q / bc;
        const int s = (int)(q2 % w);
        const long long row = (q2 / w) * SLICE + lane;
        double v = 0.0;
        if (row < nrows) {
            const long long i = row / br;
            const int r = (int)(row - i * br);
            const long long b = rowptr[i] + s;
            const bool have = b < rowptr[i + 1];
            if (have) v = vals[b * br * bc + (long long)c * br + r];
            if (c == 0 && r == 0) ell_col[(long long)s * nbr + i] = have ? colidx[b] : 0;
        }
        ell_vals[t] = v;
    }
}

template <int BC>
__global__ void __launch_bounds__(256) k_ell_spmv(long long nbr, int br, int bc_rt, int w, const int* __restrict__ ell_col,
                                                  const double* __restrict__ ell_vals, const double* __restrict__ x,
                                                  double alpha, double beta, double* __restrict__ y) {
    const int bc = BC > 0 ? BC : bc_rt;
    const long long nrows = nbr * br;
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < nrows;
         row += (long long)gridDim.x * blockDim.x) {
        const long long i = row / br;
        const double* v = ell_vals + (row / SLICE) * w * bc * SLICE + (row % SLICE);
        double acc = 0.0;
        for (int s = 0; s < w; ++s) {
            const double* xb = x + (long long)ell_col[(long long)s * nbr + i] * bc;
            const double* vs = v + (long long)s * bc * SLICE;
            if (BC > 0) {
#pragma unroll
                for (int c = 0; c < BC; ++c) acc += __ldcs(vs + c * SLICE) * __ldg(xb + c);
            } else {
                for (int c = 0; c < bc; ++c) acc += __ldcs(vs + c * SLICE) * __ldg(xb + c);
            }
        }
        y[row] = (beta == 0.0) ? alpha * acc : beta * y[row] + alpha * acc;
    }
}

// block-row kernel for matrices whose ELL padding does not pay: one thread per scalar row
__global__ void k_bsr_spmv(long long nbr, int br, int bc, const long long* __restrict__ rowptr,
                           const int* __restrict__ colidx, const double* __restrict__ vals, const double* __restrict__ x,
                           double alpha, double beta, double* __restrict__ y) {
    const long long nrows = nbr * br;
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < nrows;
         row += (long long)gridDim.x * blockDim.x) {
        const long long i = row / br;
        const int r = (int)(row - i * br);
        double acc = 0.0;
        for (long long b = rowptr[i]; b < rowptr[i + 1]; ++b) {
            const double* blk = vals + b * (long long)br * bc;
            const double* xb = x + (long long)colidx[b] * bc;
            for (int c = 0; c < bc; ++c) acc += blk[(long long)c * br + r] * __ldg(xb + c);
        }
        y[row] = (beta == 0.0) ? alpha * acc : beta * y[row] + alpha * acc;
    }
}

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32)); }

// builds the ELL copy on the first product; ell_w = -1 marks "block-row kernel"
int ensure_ell(bosss_bsr* A, cudaStream_t s) {
    if (A->ell_w != 0) return 0;
    std::vector<int64_t> rp(A->nbr + 1);
    cudaError_t e = cudaMemcpyAsync(rp.data(), A->d_rowptr, sizeof(int64_t) * rp.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("SpMV setup: ") + cudaGetErrorString(e));
    int64_t w = 0;
    for (int64_t i = 0; i < A->nbr; ++i) w = std::max<int64_t>(w, rp[i + 1] - rp[i]);
    if (w == 0 || (double)w * A->nbr > 1.25 * (double)A->nnzb) {
        A->ell_w = -1;
        return 0;
    }
    const long long nrows = A->nbr * A->br;
    const size_t nv = (size_t)((nrows + SLICE - 1) / SLICE) * w * A->bc * SLICE;
    e = cudaMalloc(&A->d_ell_col, sizeof(int32_t) * (size_t)w * A->nbr);
    if (e == cudaSuccess) e = cudaMalloc(&A->d_ell_vals, sizeof(double) * nv);
    if (e != cudaSuccess) {
        cudaFree(A->d_ell_col);
        cudaFree(A->d_ell_vals);
        A->d_ell_col = nullptr;
        A->d_ell_vals = nullptr;
        cudaGetLastError();
        A->ell_w = -1;   // not enough memory for the copy: the block-row kernel
        return 0;
    }
    k_to_ell<<<grid_for((long long)nv), 256, 0, s>>>(A->nbr, A->br, A->bc, (int)w, (const long long*)A->d_rowptr,
                                                     A->d_colidx, A->d_vals, A->d_ell_col, A->d_ell_vals);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("SpMV setup: ") + cudaGetErrorString(e));
    A->ell_w = (int)w;
    return 0;
}

}  // namespace

int bsr_spmv(bosss_bsr* A, double alpha, const double* x, double beta, double* y, cudaStream_t s) {
    const long long nrows = A->nbr * A->br;
    if (nrows == 0) return 0;
    int rc = ensure_ell(A, s);
    if (rc) return rc;
    const int grid = grid_for(nrows);
    if (A->ell_w > 0) {
        switch (A->bc) {
            case 4: k_ell_spmv<4><<<grid, 256, 0, s>>>(A->nbr, A->br, A->bc, A->ell_w, A->d_ell_col, A->d_ell_vals, x, alpha, beta, y); break;
            case 10: k_ell_spmv<10><<<grid, 256, 0, s>>>(A->nbr, A->br, A->bc, A->ell_w, A->d_ell_col, A->d_ell_vals, x, alpha, beta, y); break;
            case 20: k_ell_spmv<20><<<grid, 256, 0, s>>>(A->nbr, A->br, A->bc, A->ell_w, A->d_ell_col, A->d_ell_vals, x, alpha, beta, y); break;
            case 35: k_ell_spmv<35><<<grid, 256, 0, s>>>(A->nbr, A->br, A->bc, A->ell_w, A->d_ell_col, A->d_ell_vals, x, alpha, beta, y); break;
            default: k_ell_spmv<0><<<grid, 256, 0, s>>>(A->nbr, A->br, A->bc, A->ell_w, A->d_ell_col, A->d_ell_vals, x, alpha, beta, y); break;
        }
    } else {
        k_bsr_spmv<<<grid, 256, 0, s>>>(A->nbr, A->br, A->bc, (const long long*)A->d_rowptr, A->d_colidx, A->d_vals,
                                        x, alpha, beta, y);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("SpMV: ") + cudaGetErrorString(e));
    return 0;
}

}  // namespace bosss
