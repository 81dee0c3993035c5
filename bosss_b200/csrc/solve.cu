// solve.cu -- Jacobian assembly, block-Jacobi preconditioner, matrix-free Newton-GMRES
// and mixed-precision (FP32 GMRES / FP64 refinement) block-sparse solves.
//
// Reference counterparts:
//  * bosss_b200_compute_jacobian: EvaluatorLinear.ComputeMatrix -> LEC quadrature ->
//    BlockMsrMatrix.AccBlock (DifferentialOperator.cs:1766-1838) / FDJacobianBuilder
//    (:2558-2858, cell colouring + repeated Evaluate). Here: exact JVP probes over a
//    distance-2 colouring of the cells, one probe per (colour, local column), scattered
//    into the cell-block pattern (self + face neighbours).
//  * bosss_b200_newton_solve: Newton with MatrixFreeGMRES (Newton.cs:1231-1440), the FD
//    directional derivative dirder (Newton.cs:1450-1495) replaced by the exact JVP.
//  * bosss_b200_bsr_solve: GMRES (SoftGMRES.cs) on a BlockMsrMatrix, here in FP32 inside
//    FP64 iterative refinement.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "bsr.h"
#include "handle.h"
#include "pmg.h"
#include "solver.cuh"

namespace bosss {

// ------------------------------------------------------------------ colouring
// Either a linear colouring, colour = (a_0 i + a_1 j + a_2 k) mod lin, or a product of per-
// direction moduli, colour = (i mod m_0, j mod m_1, k mod m_2).
struct Colouring {
    int m[3] = {1, 1, 1};
    int ncol = 1;
    int lin = 0;              // > 0: linear colouring modulo lin
    int a[3] = {0, 0, 0};
};

// Distance-2 colouring of the face-neighbour graph (no two cells of one colour share a cell
// of N(j) u {j}, so one probe per colour and local column recovers every block): the linear
// colouring (i + 2j + 3k) mod 7 in 3D, (i + 2j) mod 5 in 2D, whose 2D+1 colours give every
// cell and its face neighbours distinct colours -- valid when no periodic wrap breaks it
// (periodic directions with n a multiple of 2D+1); else per-direction moduli >= 3.
static Colouring make_colouring(const GridConst& g) {
    Colouring c;
    const int M = 2 * g.D + 1;
    bool lin_ok = g.D >= 2;
    for (int d = 0; d < g.D; ++d) lin_ok = lin_ok && (!g.periodic[d] || g.n[d] % M == 0);
    if (lin_ok) {
        c.lin = M;
        c.ncol = M;
        for (int d = 0; d < g.D; ++d) c.a[d] = d + 1;
        return c;
    }
    for (int d = 0; d < g.D; ++d) {
        const int n = g.n[d];
        if (!g.periodic[d]) {
            c.m[d] = std::min(3, n);
        } else {
            c.m[d] = n;
            for (int k = 3; k <= n; ++k)
                if (n % k == 0) {
                    c.m[d] = k;
                    break;
                }
        }
        c.ncol *= c.m[d];
    }
    return c;
}

__device__ __forceinline__ int cell_colour(const GridConst& g, long long j, const Colouring& cl) {
    int ijk[3];
    cell_ijk(g, j, ijk);
    if (cl.lin > 0) return (cl.a[0] * ijk[0] + cl.a[1] * ijk[1] + cl.a[2] * ijk[2]) % cl.lin;
    int c = ijk[0] % cl.m[0];
    if (g.D >= 2) c = c * cl.m[1] + ijk[1] % cl.m[1];
    if (g.D >= 3) c = c * cl.m[2] + ijk[2] % cl.m[2];
    return c;
}

// probe: V[j*Nd + i] = 1 for cells of colour `col` and local column `i0`, else 0
__global__ void k_probe(GridConst g, Colouring cl, int col, int Nd, int i0, double* V) {
    const long long n = (long long)g.J * Nd;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / Nd;
        const int i = (int)(t - j * Nd);
        V[t] = (i == i0 && cell_colour(g, j, cl) == col) ? 1.0 : 0.0;
    }
}

// scatter JV into column i0 of every block whose column cell has colour `col`
// (blocks column-major: vals[b*br*bc + i0*br + r])
__global__ void k_scatter(GridConst g, Colouring cl, int col, int i0, int br, int bc,
                          const long long* __restrict__ rowptr, const int* __restrict__ colidx,
                          const double* __restrict__ JV, double* __restrict__ vals) {
    const long long nrows = (long long)g.J * br;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrows; t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / br;
        const int r = (int)(t - j * br);
        for (long long b = rowptr[j]; b < rowptr[j + 1]; ++b)
            if (cell_colour(g, colidx[b], cl) == col) vals[b * (long long)br * bc + (long long)i0 * br + r] = JV[t];
    }
}

// cell-block pattern: self first, then the face neighbours (duplicates dropped)
static void block_pattern(const GridConst& g, std::vector<int64_t>& rowptr, std::vector<int32_t>& colidx) {
    rowptr.assign(1, 0);
    colidx.clear();
    for (long long j = 0; j < g.J; ++j) {
        int ijk[3] = {0, 0, 0};
        for (int d = 0; d < g.D; ++d) ijk[d] = (int)((j / g.stride[d]) % g.n[d]);
        std::vector<int32_t> cols{(int32_t)j};
        for (int d = 0; d < g.D; ++d)
            for (int s = 0; s < 2; ++s) {
                int i = ijk[d] + (s ? 1 : -1);
                if (i < 0 || i >= g.n[d]) {
                    if (!g.periodic[d]) continue;
                    i = (i + g.n[d]) % g.n[d];
                }
                long long nb = 0;
                for (int dd = 0; dd < g.D; ++dd) nb += (long long)((dd == d) ? i : ijk[dd]) * g.stride[dd];
                if (std::find(cols.begin(), cols.end(), (int32_t)nb) == cols.end()) cols.push_back((int32_t)nb);
            }
        colidx.insert(colidx.end(), cols.begin(), cols.end());
        rowptr.push_back((int64_t)colidx.size());
    }
}

static int grid_of(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

// host threads of bosss_b200_batch_solve (one stream and one set of work arrays each)
static constexpr int BATCH_SOLVE_THREADS = 4;

// A += sigma I on the self blocks (the first block of every row, block_pattern); blocks
// column-major, so entry (r, r) of block b sits at b*nb*nb + r*(nb+1)
__global__ void k_shift_diag(long long nbr, int nb, const long long* __restrict__ rowptr, double* __restrict__ vals,
                             double sigma) {
    const long long n = nbr * nb;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long i = t / nb;
        const int r = (int)(t - i * nb);
        vals[rowptr[i] * (long long)nb * nb + (long long)r * (nb + 1)] += sigma;
    }
}

// out = A^T for a structurally symmetric block pattern (the face-neighbour pattern of
// block_pattern): block (j, i) of the result is block (i, j) of A transposed. One warp per
// block row; a missing mirror block sets *bad
__global__ void k_transpose_sym(long long nbr, int nb, const long long* __restrict__ rowptr,
                                const int* __restrict__ colidx, const double* __restrict__ vals,
                                double* __restrict__ out, int* bad) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long bs = (long long)nb * nb;
    for (long long i = w0; i < nbr; i += nw) {
        for (long long b = rowptr[i]; b < rowptr[i + 1]; ++b) {
            const int j = colidx[b];
            long long q = -1;
            for (long long c = rowptr[j]; c < rowptr[j + 1]; ++c)
                if (colidx[c] == (int)i) q = c;
            if (q < 0) {
                if (lane == 0) atomicExch(bad, 1);
                continue;
            }
            for (long long e = lane; e < bs; e += 32) {
                const long long c = e / nb, r = e - c * nb;   // entry (r, c) of the result block
                out[q * bs + e] = vals[b * bs + r * nb + c];
            }
        }
    }
}

// assemble J(U_dev) into a new bosss_bsr (values on the device)
static int assemble(bosss_handle* h, const double* U_dev, double time, bosss_bsr** out) {
    const GridConst& g = h->base.g;
    const int Nd = (int)(h->ndom / g.J), Nc = (int)(h->ncod / g.J);
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    block_pattern(g, rp, ci);
    bosss_bsr* A = new bosss_bsr();
    A->device = h->device;
    A->nbr = A->nbc = g.J;
    A->nnzb = (int64_t)ci.size();
    A->br = Nc;
    A->bc = Nd;
    const size_t bs = (size_t)Nc * Nd;
    cudaStream_t s = h->stream;
    auto bail = [&](cudaError_t e) {
        bosss_b200_bsr_destroy(A);
        return fail(BOSSS_ERR_CUDA, std::string("Jacobian assembly: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&A->d_rowptr, sizeof(int64_t) * rp.size());
    if (e == cudaSuccess) e = cudaMalloc(&A->d_colidx, sizeof(int32_t) * ci.size());
    if (e == cudaSuccess) e = cudaMalloc(&A->d_vals, sizeof(double) * bs * ci.size());
    if (e == cudaSuccess) e = cudaMemcpy(A->d_rowptr, rp.data(), sizeof(int64_t) * rp.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(A->d_colidx, ci.data(), sizeof(int32_t) * ci.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(A->d_vals, 0, sizeof(double) * bs * ci.size(), s);
    double *V = nullptr, *JV = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&V, sizeof(double) * h->ndom);
    if (e == cudaSuccess) e = cudaMalloc(&JV, sizeof(double) * h->ncod);
    if (e != cudaSuccess) {
        cudaFree(V);
        cudaFree(JV);
        return bail(e);
    }
    const Colouring c = make_colouring(g);
    for (int col = 0; col < c.ncol && e == cudaSuccess; ++col)
        for (int i0 = 0; i0 < Nd && e == cudaSuccess; ++i0) {
            k_probe<<<grid_of(h->ndom), 256, 0, s>>>(g, c, col, Nd, i0, V);
            int rc = run_mode(h, MODE_JVP, 1.0, 0.0, U_dev, V, JV, time, s);
            if (rc) {
                cudaFree(V);
                cudaFree(JV);
                bosss_b200_bsr_destroy(A);
                return rc;
            }
            k_scatter<<<grid_of(h->ncod), 256, 0, s>>>(g, c, col, i0, Nc, Nd,
                                                       (const long long*)A->d_rowptr, A->d_colidx, JV, A->d_vals);
            e = cudaGetLastError();
        }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(V);
    cudaFree(JV);
    if (e != cudaSuccess) return bail(e);
    *out = A;
    return BOSSS_OK;
}

// ------------------------------------------------------------------ block-Jacobi
// y_j = Dinv_j x_j (blocks column-major), one thread per scalar row
template <class T>
__global__ void k_apply_blockdiag(long long ncell, int nb, const T* __restrict__ inv, const T* __restrict__ x,
                                  T* __restrict__ y) {
    const long long n = ncell * nb;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / nb;
        const int r = (int)(t - j * nb);
        const T* B = inv + j * (long long)nb * nb;
        const T* xj = x + j * nb;
        double acc = 0.0;
        for (int c = 0; c < nb; ++c) acc += (double)B[(long long)c * nb + r] * (double)xj[c];
        y[t] = (T)acc;
    }
}

template <class T>
static int block_jacobi(const bosss_bsr* A, T** inv, cudaStream_t s) {
    if (A->br != A->bc || A->nbr != A->nbc) return fail(BOSSS_ERR_BAD_ARG, "block-Jacobi needs square diagonal blocks");
    const int nb = A->br;
    if ((size_t)2 * nb * nb * 8 > 200 * 1024) return fail(BOSSS_ERR_BAD_ARG, "cell block too large for block-Jacobi");
    CUDA_TRY(cudaMalloc(inv, sizeof(T) * (size_t)nb * nb * A->nbr));
    int* sing = nullptr;
    CUDA_TRY(cudaMalloc(&sing, sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(sing, 0, sizeof(int), s));
    const size_t smem = (size_t)2 * nb * nb * 8;
    CUDA_TRY(cudaFuncSetAttribute(k_invert_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (A->nbr > 0) k_invert_diag<T><<<(unsigned)A->nbr, 128, smem, s>>>(nb, (const long long*)A->d_rowptr, A->d_vals, *inv, sing);
    CUDA_TRY(cudaGetLastError());
    int flag = 0;
    CUDA_TRY(cudaMemcpyAsync(&flag, sing, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(sing);
    if (flag) return fail(BOSSS_ERR_BAD_ARG, "singular diagonal block in block-Jacobi");
    return BOSSS_OK;
}

template <class T>
__global__ void bsr_spmv_t(long long nbr, int br, int bc, const long long* __restrict__ rowptr, const int* __restrict__ colidx,
                           const T* __restrict__ vals, const T* __restrict__ x, T* __restrict__ y) {
    const long long nrows = nbr * br;
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < nrows; row += (long long)gridDim.x * blockDim.x) {
        const long long i = row / br;
        const int r = (int)(row - i * br);
        T acc = T(0);
        for (long long b = rowptr[i]; b < rowptr[i + 1]; ++b) {
            const T* blk = vals + b * (long long)br * bc;
            const T* xb = x + (long long)colidx[b] * bc;
            for (int c = 0; c < bc; ++c) acc += blk[(long long)c * br + r] * xb[c];
        }
        y[row] = acc;
    }
}

static void fill_defaults(const bosss_solver_opts* o, bosss_solver_opts& r, double rtol, int outer) {
    std::memset(&r, 0, sizeof(r));
    r.rtol = rtol;
    r.atol = 0.0;
    r.max_outer = outer;
    r.restart = 50;
    r.max_krylov = 2000;
    r.precond = 1;
    r.inner_rtol = 1e-3;
    if (o) {
        if (o->rtol > 0) r.rtol = o->rtol;
        if (o->atol > 0) r.atol = o->atol;
        if (o->max_outer > 0) r.max_outer = o->max_outer;
        if (o->restart > 0) r.restart = std::min(o->restart, 200);
        if (o->max_krylov > 0) r.max_krylov = o->max_krylov;
        r.precond = o->precond;
        if (o->inner_rtol > 0) r.inner_rtol = o->inner_rtol;
        r.precond_update = o->precond_update;
    }
}

template <class T>
struct KrylovWork {
    T* V = nullptr;
    T* w = nullptr;
    T* z = nullptr;
    double* partials = nullptr;
    double* hbuf = nullptr;
    double* pinned = nullptr;   // host slots of the lagged residual checks
    ~KrylovWork() {
        cudaFree(V);
        cudaFree(w);
        cudaFree(z);
        cudaFree(partials);
        cudaFree(hbuf);
        if (pinned) cudaFreeHost(pinned);
    }
    cudaError_t alloc(long long n, int m) {
        cudaError_t e = cudaMalloc(&V, sizeof(T) * (size_t)(m + 1) * n);
        if (e == cudaSuccess) e = cudaMalloc(&w, sizeof(T) * n);
        if (e == cudaSuccess) e = cudaMalloc(&z, sizeof(T) * n);
        if (e == cudaSuccess) e = cudaMalloc(&partials, sizeof(double) * RED_BLOCKS * (m + 1));
        if (e == cudaSuccess) e = cudaMalloc(&hbuf, sizeof(double) * gmres_dev_doubles(m));
        if (e == cudaSuccess) e = cudaMallocHost(&pinned, sizeof(double) * 8);
        return e;
    }
};

static double norm2(const double* x, long long n, double* partials, cudaStream_t s) {
    k_dot_partials<double><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, x, x, partials);
    std::vector<double> hp(RED_BLOCKS);
    cudaMemcpyAsync(hp.data(), partials, sizeof(double) * RED_BLOCKS, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double acc = 0.0;
    for (double v : hp) acc += v;
    return std::sqrt(std::max(acc, 0.0));
}

// ------------------------------------------------------------------ per-instance batched solves
// distance-1 colouring (face neighbours differ): the parity (i + j + k) mod 2 when no periodic
// direction has an odd cell count; else per direction the smallest modulus m >= 2 with
// n mod m != 1 on periodic directions (so that cells n-1 and 0 differ too), 1 for one cell
static Colouring make_colouring1(const GridConst& g) {
    Colouring c;
    bool parity = true;
    for (int d = 0; d < g.D; ++d) parity = parity && (!g.periodic[d] || g.n[d] % 2 == 0);
    if (parity) {
        c.lin = 2;
        c.ncol = 2;
        for (int d = 0; d < g.D; ++d) c.a[d] = 1;
        return c;
    }
    for (int d = 0; d < g.D; ++d) {
        const int n = g.n[d];
        int m = 1;
        if (n > 1) {
            m = 2;
            while (g.periodic[d] && n % m == 1) ++m;
        }
        c.m[d] = m;
        c.ncol *= m;
    }
    return c;
}

// column i0 of the diagonal cell blocks of (I/dt + J) from the probe product JV (blocks
// column-major; the probe covered the cells of colour `col`)
__global__ void k_scatter_diag(GridConst g, Colouring cl, int col, int nb, int i0, double idt,
                               const double* __restrict__ JV, double* __restrict__ blocks) {
    const long long n = (long long)g.J * nb;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / nb;
        const int r = (int)(t - j * nb);
        if (cell_colour(g, j, cl) != col) continue;
        blocks[j * (long long)nb * nb + (long long)i0 * nb + r] = JV[t] + (r == i0 ? idt : 0.0);
    }
}

// in-place transpose of every nb x nb block
__global__ void k_transpose_blocks(long long nblk, int nb, double* __restrict__ blocks) {
    const long long n = nblk * nb * nb;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / ((long long)nb * nb);
        const int e = (int)(t - b * nb * nb), c = e / nb, r = e % nb;
        if (r < c) {
            double* B = blocks + b * (long long)nb * nb;
            const double v = B[c * nb + r];
            B[c * nb + r] = B[r * nb + c];
            B[r * nb + c] = v;
        }
    }
}

__global__ void k_iota(long long n, long long* __restrict__ p) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) p[t] = t;
}

}  // namespace bosss

using namespace bosss;

extern "C" {

int bosss_b200_compute_jacobian(bosss_handle* h, const double* U, double time, bosss_bsr** out) {
    if (!h || !U || !out) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    int rc = ensure_staging(h);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpyAsync(h->dU, U, sizeof(double) * h->ndom, cudaMemcpyHostToDevice, h->stream));
    return assemble(h, h->dU, time, out);
}

int bosss_b200_newton_solve(bosss_handle* h, double* U, double time, const bosss_solver_opts* opt,
                            bosss_solver_report* rep) {
    if (!h || !U) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (h->ndom != h->ncod) return fail(BOSSS_ERR_BAD_ARG, "Newton needs a square operator");
    bosss_solver_opts o;
    fill_defaults(opt, o, 1e-10, 20);
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t s = h->stream;
    const long long n = h->ndom;
    if (o.precond < 0 || o.precond > 2) return fail(BOSSS_ERR_BAD_ARG, "unknown preconditioner");
    double *dU = nullptr, *dR = nullptr, *dX = nullptr, *dT = nullptr, *dW = nullptr, *dinv = nullptr;
    bosss_pmg* mg = nullptr;
    KrylovWork<double> kw;
    auto cleanup = [&]() {
        pmg_destroy(mg);
        cudaFree(dU);
        cudaFree(dR);
        cudaFree(dX);
        cudaFree(dT);
        cudaFree(dW);
        cudaFree(dinv);
    };
    cudaError_t e = cudaMalloc(&dU, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dR, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dX, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dT, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dW, sizeof(double) * n);
    if (e == cudaSuccess) e = kw.alloc(n, o.restart);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dU, U, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        cleanup();
        return fail(BOSSS_ERR_CUDA, std::string("Newton work arrays: ") + cudaGetErrorString(e));
    }
    bosss_solver_report r{};
    int rc = 0;
    const int nb = (int)(n / h->base.g.J);
    double res = 0.0, res0 = 0.0;
    for (int it = 0; it <= o.max_outer; ++it) {
        rc = run_mode(h, MODE_RES, 1.0, 0.0, dU, nullptr, dR, time, s);
        if (rc) break;
        res = norm2(dR, n, kw.partials, s);
        if (it == 0) res0 = res;
        r.residual = res;
        if (!std::isfinite(res)) {
            rc = fail(BOSSS_ERR_NAN, "non-finite residual in Newton");
            break;
        }
        if (res <= std::max(o.rtol * res0, o.atol)) {
            r.converged = 1;
            break;
        }
        if (it == o.max_outer) break;
        r.outer_iters = it + 1;
        // right-preconditioned J M^-1 z = -R, dU_step = M^-1 z
        const int upd = std::max(o.precond_update, 1);
        if ((o.precond == 1 || o.precond == 2) && it % upd == 0) {
            cudaFree(dinv);
            dinv = nullptr;
            pmg_destroy(mg);
            mg = nullptr;
            bosss_bsr* A = nullptr;
            rc = assemble(h, dU, time, &A);
            if (rc) break;
            rc = (o.precond == 1) ? block_jacobi<double>(A, &dinv, s) : pmg_create(h, A, &mg);
            bosss_b200_bsr_destroy(A);
            if (rc) break;
        }
        k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, -1.0, dR, 0.0, dW);   // rhs = -R
        CUDA_TRY(cudaMemsetAsync(dX, 0, sizeof(double) * n, s));
        int inner_rc = 0;
        auto apply = [&](const double* x, double* y) -> cudaError_t {
            const double* xin = x;
            if (dinv) {
                k_apply_blockdiag<double><<<grid_of(n), 256, 0, s>>>(h->base.g.J, nb, dinv, x, dT);
                xin = dT;
            } else if (mg) {
                int rr = pmg_apply(mg, x, dT, s);
                if (rr) {
                    inner_rc = rr;
                    return cudaErrorUnknown;
                }
                xin = dT;
            }
            int rr = run_mode(h, MODE_JVP, 1.0, 0.0, dU, xin, y, time, s);
            if (rr) inner_rc = rr;
            return rr ? cudaErrorUnknown : cudaGetLastError();
        };
        GmresResult g = gmres<double>(n, apply, dW, dX, o.restart, o.max_krylov, o.inner_rtol, 0.0, kw.V, kw.w,
                                      kw.partials, kw.hbuf, s, kw.pinned);
        r.krylov_iters += g.iters;
        if (inner_rc) {
            rc = inner_rc;
            break;
        }
        if (g.error) {
            rc = fail(BOSSS_ERR_CUDA, "GMRES: " + std::string(cudaGetErrorString((cudaError_t)g.error)));
            break;
        }
        const double* step = dX;
        if (dinv) {
            k_apply_blockdiag<double><<<grid_of(n), 256, 0, s>>>(h->base.g.J, nb, dinv, dX, dT);
            step = dT;
        } else if (mg) {
            rc = pmg_apply(mg, dX, dT, s);
            if (rc) break;
            step = dT;
        }
        // backtracking on the residual norm
        CUDA_TRY(cudaMemcpyAsync(dW, dU, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        double lam = 1.0;
        for (int ls = 0; ls < 8; ++ls) {
            CUDA_TRY(cudaMemcpyAsync(dU, dW, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, lam, step, 1.0, dU);
            rc = run_mode(h, MODE_RES, 1.0, 0.0, dU, nullptr, dR, time, s);
            if (rc) break;
            const double rn = norm2(dR, n, kw.partials, s);
            if (std::isfinite(rn) && rn < res) break;
            lam *= 0.5;
        }
        if (rc) break;
    }
    if (!rc) {
        cudaError_t e2 = cudaMemcpyAsync(U, dU, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
        if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s);
        if (e2 != cudaSuccess) rc = fail(BOSSS_ERR_CUDA, cudaGetErrorString(e2));
    }
    r.residual0 = res0;
    if (rep) *rep = r;
    cleanup();
    return rc;
}

int bosss_b200_bsr_solve(bosss_bsr* A, const double* b, double* x, const bosss_solver_opts* opt,
                         bosss_solver_report* rep) {
    if (!A || !b || !x) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (A->nbr != A->nbc || A->br != A->bc) return fail(BOSSS_ERR_BAD_ARG, "bsr_solve needs a square matrix");
    bosss_solver_opts o;
    fill_defaults(opt, o, 1e-10, 30);
    CUDA_TRY(cudaSetDevice(A->device));
    cudaStream_t s = A->stream;
    const long long n = A->nbr * A->br;
    const size_t nv = (size_t)A->nnzb * A->br * A->bc;
    if (!A->d_vals32) {
        CUDA_TRY(cudaMalloc(&A->d_vals32, sizeof(float) * std::max<size_t>(nv, 1)));
        k_convert<double, float><<<grid_of((long long)nv), 256, 0, s>>>((long long)nv, A->d_vals, A->d_vals32);
        CUDA_TRY(cudaGetLastError());
    }
    double *db = nullptr, *dx = nullptr, *dr = nullptr;
    float *rf = nullptr, *cf = nullptr, *tf = nullptr, *inv = nullptr;
    KrylovWork<float> kw;
    auto cleanup = [&]() {
        cudaFree(db);
        cudaFree(dx);
        cudaFree(dr);
        cudaFree(rf);
        cudaFree(cf);
        cudaFree(tf);
        cudaFree(inv);
    };
    cudaError_t e = cudaMalloc(&db, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dx, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&rf, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&cf, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&tf, sizeof(float) * n);
    if (e == cudaSuccess) e = kw.alloc(n, o.restart);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        cleanup();
        return fail(BOSSS_ERR_CUDA, std::string("solver work arrays: ") + cudaGetErrorString(e));
    }
    int rc = 0;
    if (o.precond == 2) {
        cleanup();
        return fail(BOSSS_ERR_BAD_ARG, "bsr_solve: preconditioner 0 (none) or 1 (block-Jacobi)");
    }
    if (o.precond == 1) {
        rc = block_jacobi<float>(A, &inv, s);
        if (rc) {
            cleanup();
            return rc;
        }
    }
    const double bnorm = norm2(db, n, kw.partials, s);
    bosss_solver_report r{};
    const int nb = A->br;
    for (int it = 0; it <= o.max_outer; ++it) {
        // r = b - A x in FP64
        rc = bosss_b200_bsr_spmv_device(A, -1.0, dx, 0.0, dr, s);
        if (rc) break;
        k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, 1.0, db, 1.0, dr);
        const double res = norm2(dr, n, kw.partials, s);
        if (it == 0) r.residual0 = res;
        r.residual = res;
        if (!std::isfinite(res)) {
            rc = fail(BOSSS_ERR_NAN, "non-finite residual in refinement");
            break;
        }
        if (res <= std::max(o.rtol * bnorm, o.atol)) {
            r.converged = 1;
            break;
        }
        if (it == o.max_outer) break;
        r.outer_iters = it + 1;
        // FP32 correction: A c = r
        k_convert<double, float><<<grid_of(n), 256, 0, s>>>(n, dr, rf);
        CUDA_TRY(cudaMemsetAsync(cf, 0, sizeof(float) * n, s));
        auto apply = [&](const float* xx, float* yy) -> cudaError_t {
            const float* xin = xx;
            if (inv) {
                k_apply_blockdiag<float><<<grid_of(n), 256, 0, s>>>(A->nbr, nb, inv, xx, tf);
                xin = tf;
            }
            bsr_spmv_t<float><<<grid_of(n), 256, 0, s>>>(A->nbr, A->br, A->bc, (const long long*)A->d_rowptr,
                                                          A->d_colidx, A->d_vals32, xin, yy);
            return cudaGetLastError();
        };
        GmresResult g = gmres<float>(n, apply, rf, cf, o.restart, o.max_krylov, o.inner_rtol, 0.0, kw.V, kw.w,
                                     kw.partials, kw.hbuf, s, kw.pinned);
        r.krylov_iters += g.iters;
        if (g.error) {
            rc = fail(BOSSS_ERR_CUDA, "GMRES: " + std::string(cudaGetErrorString((cudaError_t)g.error)));
            break;
        }
        const float* corr = cf;
        if (inv) {
            k_apply_blockdiag<float><<<grid_of(n), 256, 0, s>>>(A->nbr, nb, inv, cf, tf);
            corr = tf;
        }
        // x += c (FP64 accumulation of the FP32 correction)
        k_convert<float, double><<<grid_of(n), 256, 0, s>>>(n, corr, dr);
        k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, 1.0, dr, 1.0, dx);
        CUDA_TRY(cudaGetLastError());
    }
    if (!rc) {
        cudaError_t e2 = cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
        if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s);
        if (e2 != cudaSuccess) rc = fail(BOSSS_ERR_CUDA, cudaGetErrorString(e2));
    }
    if (rep) *rep = r;
    cleanup();
    return rc;
}


int bosss_b200_batch_solve(bosss_batch* B, int32_t transpose, const double* dt, const double* U_dev,
                           const double* b_dev, double* x_dev, const bosss_solver_opts* opt,
                           bosss_solver_report* reports) {
    if (!B || !dt || !b_dev || !x_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (transpose != 0 && transpose != 1) return fail(BOSSS_ERR_BAD_ARG, "transpose: 0 or 1");
    for (int i = 0; i < B->n; ++i) {
        if (!(dt[i] > 0.0) || !std::isfinite(dt[i])) return fail(BOSSS_ERR_BAD_ARG, "dt must be positive");
        if (B->h[i]->ndom != B->h[i]->ncod) return fail(BOSSS_ERR_BAD_ARG, "batch solve needs square operators");
    }
    bosss_solver_opts o;
    fill_defaults(opt, o, 1e-10, 30);
    if (o.precond < 0 || o.precond > 2) return fail(BOSSS_ERR_BAD_ARG, "batch solve: preconditioner 0, 1 or 2");
    if (o.precond == 2)
        for (int i = 0; i < B->n; ++i)
            if (B->h[i]->ndom != (int64_t)B->h[i]->base.g.J * np_of(B->h[i]->D, B->h[i]->K))
                return fail(BOSSS_ERR_BAD_ARG, "batch solve: the multigrid preconditioner needs scalar operators");
    CUDA_TRY(cudaSetDevice(B->device));
    // instances largest first, taken by a few host threads with their own streams and work
    // arrays, so that the launch-bound solves of the small instances overlap the large ones
    std::vector<int> order(B->n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return B->h[a]->ndom > B->h[b]->ndom; });
    std::atomic<int> next{0};
    std::atomic<bool> abort_all{false};
    const int nworkers = std::max(1, std::min(B->n, BATCH_SOLVE_THREADS));
    std::vector<int> wrc(nworkers, 0);
    std::vector<std::string> wmsg(nworkers);
    auto worker = [&]() -> int {
    CUDA_TRY(cudaSetDevice(B->device));
    cudaStream_t s = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    long long nmax = 0, bmax = 0;
    for (int i = 0; i < B->n; ++i) {
        const bosss_handle* h = B->h[i];
        const long long nb = h->ndom / h->base.g.J;
        nmax = std::max<long long>(nmax, h->ndom);
        bmax = std::max<long long>(bmax, (long long)h->base.g.J * nb * nb);
    }
    double *r64 = nullptr, *t64 = nullptr, *y64 = nullptr, *z64 = nullptr, *u0 = nullptr, *blk = nullptr;
    bosss_pmg* mg = nullptr;
    float *r32 = nullptr, *c32 = nullptr, *t32 = nullptr, *inv = nullptr;
    long long* rp = nullptr;
    int* sing = nullptr;
    KrylovWork<float> kw;
    auto cleanup = [&]() {
        cudaFree(r64);
        cudaFree(t64);
        cudaFree(y64);
        cudaFree(z64);
        pmg_destroy(mg);
        mg = nullptr;
        cudaFree(u0);
        cudaFree(blk);
        cudaFree(r32);
        cudaFree(c32);
        cudaFree(t32);
        cudaFree(inv);
        cudaFree(rp);
        cudaFree(sing);
        cudaStreamDestroy(s);
    };
    cudaError_t e = cudaMalloc(&r64, sizeof(double) * nmax);
    if (e == cudaSuccess) e = cudaMalloc(&t64, sizeof(double) * nmax);
    if (e == cudaSuccess) e = cudaMalloc(&y64, sizeof(double) * nmax);
    if (e == cudaSuccess && !U_dev) e = cudaMalloc(&u0, sizeof(double) * nmax);
    if (e == cudaSuccess && o.precond == 2) e = cudaMalloc(&z64, sizeof(double) * nmax);
    if (e == cudaSuccess) e = cudaMalloc(&r32, sizeof(float) * nmax);
    if (e == cudaSuccess) e = cudaMalloc(&c32, sizeof(float) * nmax);
    if (e == cudaSuccess) e = cudaMalloc(&t32, sizeof(float) * nmax);
    if (e == cudaSuccess && o.precond == 1) e = cudaMalloc(&blk, sizeof(double) * bmax);
    if (e == cudaSuccess && o.precond == 1) e = cudaMalloc(&inv, sizeof(float) * bmax);
    if (e == cudaSuccess && o.precond == 1) e = cudaMalloc(&rp, sizeof(long long) * (nmax + 1));
    if (e == cudaSuccess) e = cudaMalloc(&sing, sizeof(int));
    if (e == cudaSuccess) e = kw.alloc(nmax, o.restart);
    if (e == cudaSuccess && u0) e = cudaMemsetAsync(u0, 0, sizeof(double) * nmax, s);
    if (e != cudaSuccess) {
        cleanup();
        return fail(BOSSS_ERR_CUDA, std::string("batch solve work arrays: ") + cudaGetErrorString(e));
    }
    int rc = 0;
    auto cu = [&](cudaError_t e2, const char* what) {
        if (e2 != cudaSuccess && !rc) rc = fail(BOSSS_ERR_CUDA, std::string("batch solve (") + what + "): " +
                                                                  cudaGetErrorString(e2));
        return rc == 0;
    };
    const int mode = transpose ? MODE_VJP : MODE_JVP;
    for (int it = next++; it < B->n && !rc && !abort_all; it = next++) {
        const int i = order[it];
        bosss_handle* h = B->h[i];
        const GridConst& g = h->base.g;
        const long long n = h->ndom, off = B->dom_off[i];
        const int nb = (int)(n / g.J);
        const double idt = 1.0 / dt[i];
        const double* U = U_dev ? U_dev + off : u0;
        const double* bi = b_dev + off;
        double* xi = x_dev + off;
        // y = x/dt + J x (transpose: + J^T x), FP64
        auto op64 = [&](const double* xin, double* yout) -> int {
            int r2 = run_mode(h, mode, 1.0, 0.0, U, xin, yout, 0.0, s);
            if (r2) return r2;
            k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, idt, xin, 1.0, yout);
            return cudaGetLastError() == cudaSuccess ? 0 : fail(BOSSS_ERR_CUDA, "batch solve: vector update");
        };
        bosss_solver_report r{};
        // block-Jacobi: the diagonal cell blocks of I/dt + J, probed over a distance-1 colouring
        if (o.precond == 1) {
            const Colouring c = make_colouring1(g);
            for (int col = 0; col < c.ncol && !rc; ++col)
                for (int i0 = 0; i0 < nb && !rc; ++i0) {
                    k_probe<<<grid_of(n), 256, 0, s>>>(g, c, col, nb, i0, t64);
                    rc = run_mode(h, MODE_JVP, 1.0, 0.0, U, t64, y64, 0.0, s);
                    if (!rc)
                        k_scatter_diag<<<grid_of(n), 256, 0, s>>>(g, c, col, nb, i0, idt, y64, blk);
                }
            if (rc) break;
            if (transpose) k_transpose_blocks<<<grid_of((long long)g.J * nb * nb), 256, 0, s>>>(g.J, nb, blk);
            k_iota<<<grid_of(g.J + 1), 256, 0, s>>>(g.J + 1, rp);
            const size_t smem = (size_t)2 * nb * nb * 8;
            if (!cu(cudaMemsetAsync(sing, 0, sizeof(int), s), "memset") ||
                !cu(cudaFuncSetAttribute(k_invert_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "attribute"))
                break;
            k_invert_diag<float><<<(unsigned)g.J, 128, smem, s>>>(nb, rp, blk, inv, sing);
            int flag = 0;
            if (!cu(cudaGetLastError(), "block inverse") ||
                !cu(cudaMemcpyAsync(&flag, sing, sizeof(int), cudaMemcpyDeviceToHost, s), "copy") ||
                !cu(cudaStreamSynchronize(s), "synchronize"))
                break;
            if (flag) {
                rc = fail(BOSSS_ERR_BAD_ARG, "batch solve: singular diagonal block");
                break;
            }
        }
        // multigrid: V-cycle on the assembled I/dt + J (transpose: its transpose)
        pmg_destroy(mg);
        mg = nullptr;
        if (o.precond == 2) {
            if (!cu(cudaStreamSynchronize(s), "synchronize")) break;
            bosss_bsr* A = nullptr;
            rc = assemble(h, U, 0.0, &A);
            if (rc) break;
            const long long bsz = (long long)nb * nb;
            k_shift_diag<<<grid_of((long long)g.J * nb), 256, 0, s>>>(g.J, nb, (const long long*)A->d_rowptr,
                                                                      A->d_vals, idt);
            bool ok = cu(cudaGetLastError(), "diagonal shift");
            if (ok && transpose) {
                double* tv = nullptr;
                ok = cu(cudaMalloc(&tv, sizeof(double) * bsz * A->nnzb), "transpose alloc") &&
                     cu(cudaMemsetAsync(sing, 0, sizeof(int), s), "memset");
                if (ok) {
                    k_transpose_sym<<<grid_of((long long)g.J * 32), 256, 0, s>>>(
                        g.J, nb, (const long long*)A->d_rowptr, A->d_colidx, A->d_vals, tv, sing);
                    int flag = 0;
                    ok = cu(cudaGetLastError(), "transpose") &&
                         cu(cudaMemcpyAsync(&flag, sing, sizeof(int), cudaMemcpyDeviceToHost, s), "copy") &&
                         cu(cudaStreamSynchronize(s), "synchronize");
                    if (ok && flag) {
                        rc = fail(BOSSS_ERR_BAD_ARG, "batch solve: block pattern is not symmetric");
                        ok = false;
                    }
                }
                if (ok) {
                    cudaFree(A->d_vals);
                    A->d_vals = tv;
                } else {
                    cudaFree(tv);
                }
            }
            if (ok) ok = cu(cudaStreamSynchronize(s), "synchronize");
            if (ok) rc = pmg_create(h, A, &mg);
            bosss_b200_bsr_destroy(A);
            if (!ok || rc) break;
        }
        const double bnorm = norm2(bi, n, kw.partials, s);
        for (int it = 0; it <= o.max_outer; ++it) {
            // r = b - (I/dt + J) x in FP64
            rc = op64(xi, r64);
            if (rc) break;
            k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, 1.0, bi, -1.0, r64);
            const double res = norm2(r64, n, kw.partials, s);
            if (it == 0) r.residual0 = res;
            r.residual = res;
            if (!std::isfinite(res)) {
                rc = fail(BOSSS_ERR_NAN, "non-finite residual in the batch solve");
                break;
            }
            if (res <= std::max(o.rtol * bnorm, o.atol)) {
                r.converged = 1;
                break;
            }
            if (it == o.max_outer) break;
            r.outer_iters = it + 1;
            // FP32 GMRES for the correction, right block-Jacobi, operator applied in FP64
            k_convert<double, float><<<grid_of(n), 256, 0, s>>>(n, r64, r32);
            if (!cu(cudaMemsetAsync(c32, 0, sizeof(float) * n, s), "memset")) break;
            int inner_rc = 0;
            auto apply = [&](const float* v, float* y) -> cudaError_t {
                const float* vin = v;
                if (mg) {
                    k_convert<float, double><<<grid_of(n), 256, 0, s>>>(n, v, t64);
                    int r2 = pmg_apply(mg, t64, z64, s);
                    if (!r2) r2 = op64(z64, y64);
                    if (r2) {
                        inner_rc = r2;
                        return cudaErrorUnknown;
                    }
                    k_convert<double, float><<<grid_of(n), 256, 0, s>>>(n, y64, y);
                    return cudaGetLastError();
                }
                if (inv) {
                    k_apply_blockdiag<float><<<grid_of(n), 256, 0, s>>>(g.J, nb, inv, v, t32);
                    vin = t32;
                }
                k_convert<float, double><<<grid_of(n), 256, 0, s>>>(n, vin, t64);
                int r2 = op64(t64, y64);
                if (r2) {
                    inner_rc = r2;
                    return cudaErrorUnknown;
                }
                k_convert<double, float><<<grid_of(n), 256, 0, s>>>(n, y64, y);
                return cudaGetLastError();
            };
            GmresResult gr = gmres<float>(n, apply, r32, c32, o.restart, o.max_krylov, o.inner_rtol, 0.0, kw.V, kw.w,
                                          kw.partials, kw.hbuf, s, kw.pinned);
            r.krylov_iters += gr.iters;
            if (inner_rc) {
                rc = inner_rc;
                break;
            }
            if (gr.error) {
                rc = fail(BOSSS_ERR_CUDA, "GMRES: " + std::string(cudaGetErrorString((cudaError_t)gr.error)));
                break;
            }
            const float* corr = c32;
            if (inv) {
                k_apply_blockdiag<float><<<grid_of(n), 256, 0, s>>>(g.J, nb, inv, c32, t32);
                corr = t32;
            }
            k_convert<float, double><<<grid_of(n), 256, 0, s>>>(n, corr, t64);
            if (mg) {
                rc = pmg_apply(mg, t64, z64, s);
                if (rc) break;
                k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, 1.0, z64, 1.0, xi);
            } else {
                k_axpby<double><<<grid_of(n), 256, 0, s>>>(n, 1.0, t64, 1.0, xi);
            }
            if (!cu(cudaGetLastError(), "update")) break;
        }
        if (reports) reports[i] = r;
    }
    if (!rc) {
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    }
    cleanup();
    return rc;
    };
    // errors are thread-local: each worker keeps its message for the calling thread
    auto run_worker = [&](int wid) {
        const int r = worker();
        if (r) {
            char buf[512];
            bosss_b200_last_error(buf, sizeof(buf));
            wrc[wid] = r;
            wmsg[wid] = buf;
            abort_all = true;
        }
    };
    std::vector<std::thread> threads;
    for (int w = 1; w < nworkers; ++w) threads.emplace_back(run_worker, w);
    run_worker(0);
    for (auto& t : threads) t.join();
    for (int w = 0; w < nworkers; ++w)
        if (wrc[w]) return fail(wrc[w], wmsg[w]);
    return BOSSS_OK;
}

}  // extern "C"
