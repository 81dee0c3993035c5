// pmg.cu -- multigrid preconditioner for the Jacobians of scalar DG operators on Cartesian
// grids: block-Jacobi smoothed p-levels (degree k, k-1, ..., 1 on the same cells), then the
// piecewise-constant level and its geometric aggregates of 2^D cells, one V-cycle per
// application, replayed from a CUDA graph.
//
// Reference counterparts:
//  * ClassicMultigrid.Solve (ClassicMultigrid.cs:335-420): pre-smoother, restriction of the
//    residual, coarse-level solve, prolongation of the correction, post-smoother;
//  * LevelPmg (LevelPmg.cs:561-600): coarsening in the polynomial degree on one grid level.
//    The basis is orthonormal and hierarchical (modes ordered by total degree), so the
//    restriction to degree k' keeps the first Np(k') coefficients of each cell, the
//    prolongation pads with zeros, and the Galerkin operator R A P is the leading
//    Np(k') x Np(k') sub-block of every cell block;
//  * BlockJacobi (BlockJacobi.cs:148-185, omega = 1, one sweep): the cell-block smoother;
//  * CoarseningAlgorithms.CreateSequence / Coarsen (CoarseningAlgorithms.cs:59-215):
//    aggregation grids; here the aggregates are the 2x2x2 boxes of the Cartesian grid and the
//    aggregate operator is the Galerkin sum of the piecewise-constant couplings.
//
// Levels and kernels:
//  p-level l (m = Np(k_l) modes per cell, blocks m x m column-major, the fine pattern):
//    x = Dinv b;  b' = first m' rows of (b - A x) per cell;  coarse solve;  x += P x';
//    r = b - A x;  x += Dinv r
//  structured level (one unknown per cell or aggregate, 7-point couplings):
//    nu damped Jacobi sweeps;  b' = aggregate sums of (b - A x);  coarse solve;
//    x += P x';  nu damped Jacobi sweeps
//  coarsest structured level (<= 100 unknowns): dense inverse (Gauss-Jordan at setup), or
//    damped Jacobi sweeps when it is singular (periodic pure diffusion: constants).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bsr.h"
#include "handle.h"
#include "pmg.h"
#include "solver.cuh"

namespace bosss {

namespace {

constexpr int NS = 7;            // structured stencil: diagonal, then (d, s) = (0,0),(0,1),(1,0),...
constexpr int COARSE_MAX = 100;  // largest dense coarsest level
constexpr double OMEGA = 0.7;    // damping of the Jacobi sweeps on the structured levels
constexpr int NU_H = 2;          // Jacobi sweeps before and after each structured coarse correction
constexpr int COARSE_SWEEPS = 40;

// structured level geometry (index = sum_d ijk[d] * stride[d], n[d] = 1 for d >= D)
struct SGeom {
    int n[3];
    int per[3];
    long long stride[3];
    long long N;
};

__host__ __device__ inline void s_ijk(const SGeom& g, long long i, int* ijk) {
    for (int d = 0; d < 3; ++d) ijk[d] = (int)((i / g.stride[d]) % g.n[d]);
}

// neighbour (d, s) of the cell ijk; -1 outside a non-periodic direction
__host__ __device__ inline long long s_nb(const SGeom& g, const int* ijk, int d, int s) {
    int i = ijk[d] + (s ? 1 : -1);
    if (i < 0 || i >= g.n[d]) {
        if (!g.per[d]) return -1;
        i = (i + g.n[d]) % g.n[d];
    }
    long long j = 0;
    for (int dd = 0; dd < 3; ++dd) j += (long long)((dd == d) ? i : ijk[dd]) * g.stride[dd];
    return j;
}

// y = A x for the structured stencil at cell i
__device__ inline double s_apply_row(const SGeom& g, const double* __restrict__ st, const double* __restrict__ x,
                                     long long i) {
    int ijk[3];
    s_ijk(g, i, ijk);
    double acc = st[i] * x[i];
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s) {
            const double c = st[(1 + 2 * d + s) * g.N + i];
            if (c != 0.0) acc += c * x[s_nb(g, ijk, d, s)];
        }
    return acc;
}

#define GRID_STRIDE(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// ---- setup kernels
// leading m x m sub-block of every m0 x m0 block (both column-major)
__global__ void k_sub_blocks(long long nnzb, int m0, int m, const double* __restrict__ v0, double* __restrict__ v) {
    const long long n = nnzb * m * m;
    GRID_STRIDE(t, n) {
        const long long b = t / (m * m);
        const int e = (int)(t - b * m * m), c = e / m, r = e % m;
        v[t] = v0[b * m0 * m0 + (long long)c * m0 + r];
    }
}

// piecewise-constant couplings of the finest structured level from the cell blocks'
// (0, 0) entries: the diagonal block to st[0], a face neighbour's block to its direction
__global__ void k_p0_extract(SGeom g, int m, const long long* __restrict__ rowptr, const int* __restrict__ colidx,
                             const double* __restrict__ vals, double* __restrict__ st) {
    GRID_STRIDE(i, g.N) {
        int ijk[3];
        s_ijk(g, i, ijk);
        double c[NS] = {0, 0, 0, 0, 0, 0, 0};
        for (long long b = rowptr[i]; b < rowptr[i + 1]; ++b) {
            const long long j = colidx[b];
            const double v = vals[b * (long long)m * m];
            if (j == i) {
                c[0] += v;
                continue;
            }
            for (int q = 0; q < 6; ++q)
                if (s_nb(g, ijk, q / 2, q % 2) == j) {
                    c[1 + q] += v;
                    break;
                }
        }
        for (int q = 0; q < NS; ++q) st[q * g.N + i] = c[q];
    }
}

// index of the aggregate of fine cell ijk on the coarse level
__device__ inline long long s_agg(const SGeom& gc, const int* ijk) {
    long long J = 0;
    for (int d = 0; d < 3; ++d) J += (long long)(ijk[d] / 2) * gc.stride[d];
    return J;
}

// Galerkin operator of the aggregates: sum of the couplings between their cells, one thread
// per aggregate (fixed summation order)
__global__ void k_agg_build(SGeom gf, SGeom gc, const double* __restrict__ stf, double* __restrict__ stc) {
    GRID_STRIDE(I, gc.N) {
        int IJK[3];
        s_ijk(gc, I, IJK);
        double c[NS] = {0, 0, 0, 0, 0, 0, 0};
        for (int a = 0; a < 8; ++a) {
            int ijk[3];
            bool ok = true;
            for (int d = 0; d < 3; ++d) {
                ijk[d] = 2 * IJK[d] + ((a >> d) & 1);
                ok = ok && ijk[d] < gf.n[d];
            }
            if (!ok) continue;
            long long i = 0;
            for (int d = 0; d < 3; ++d) i += (long long)ijk[d] * gf.stride[d];
            c[0] += stf[i];
            for (int q = 0; q < 6; ++q) {
                const double v = stf[(1 + q) * gf.N + i];
                if (v == 0.0) continue;
                const long long j = s_nb(gf, ijk, q / 2, q % 2);
                if (j < 0) continue;
                int jjk[3];
                s_ijk(gf, j, jjk);
                const long long J = s_agg(gc, jjk);
                if (J == I) {
                    c[0] += v;
                    continue;
                }
                for (int q2 = 0; q2 < 6; ++q2)
                    if (s_nb(gc, IJK, q2 / 2, q2 % 2) == J) {
                        c[1 + q2] += v;
                        break;
                    }
            }
        }
        for (int q = 0; q < NS; ++q) stc[q * gc.N + I] = c[q];
    }
}

// dense column-major matrix of a structured level (coarsest)
__global__ void k_dense(SGeom g, const double* __restrict__ st, double* __restrict__ M) {
    GRID_STRIDE(i, g.N) {
        int ijk[3];
        s_ijk(g, i, ijk);
        for (long long j = 0; j < g.N; ++j) M[j * g.N + i] = 0.0;
        M[i * g.N + i] += st[i];
        for (int q = 0; q < 6; ++q) {
            const double c = st[(1 + q) * g.N + i];
            if (c == 0.0) continue;
            const long long j = s_nb(g, ijk, q / 2, q % 2);
            if (j >= 0) M[j * g.N + i] += c;
        }
    }
}

// Gauss-Jordan inverse with partial pivoting of the dense coarsest matrix (column-major, one
// CTA, [A | I] in shared memory); a pivot below 1e-12 of the largest entry marks the matrix
// singular (the piecewise-constant operator of periodic problems without a reaction term
// has the constants in its kernel)
__global__ void k_dense_inverse(int N, const double* __restrict__ M, double* __restrict__ inv, int* __restrict__ singular) {
    extern __shared__ double sm[];
    double* A = sm;              // row-major
    double* I = sm + N * N;
    __shared__ int piv;
    __shared__ double amax;
    if (threadIdx.x == 0) amax = 0.0;
    __syncthreads();
    double loc = 0.0;
    for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
        const int r = t / N, c = t % N;
        A[t] = M[(long long)c * N + r];
        I[t] = (r == c) ? 1.0 : 0.0;
        loc = fmax(loc, fabs(A[t]));
    }
    for (int o = 16; o > 0; o >>= 1) loc = fmax(loc, __shfl_down_sync(0xffffffffu, loc, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)&amax, __double_as_longlong(loc));
    __syncthreads();
    const double tiny = 1e-12 * amax;
    for (int k = 0; k < N; ++k) {
        if (threadIdx.x == 0) {
            int p = k;
            double best = fabs(A[k * N + k]);
            for (int r = k + 1; r < N; ++r)
                if (fabs(A[r * N + k]) > best) {
                    best = fabs(A[r * N + k]);
                    p = r;
                }
            piv = p;
            if (!(best > tiny)) *singular = 1;
        }
        __syncthreads();
        const int p = piv;
        if (p != k)
            for (int c = threadIdx.x; c < N; c += blockDim.x) {
                double t0 = A[k * N + c];
                A[k * N + c] = A[p * N + c];
                A[p * N + c] = t0;
                t0 = I[k * N + c];
                I[k * N + c] = I[p * N + c];
                I[p * N + c] = t0;
            }
        __syncthreads();
        const double d = A[k * N + k];
        const double inv_d = (d != 0.0) ? 1.0 / d : 0.0;
        __syncthreads();
        for (int c = threadIdx.x; c < N; c += blockDim.x) {
            A[k * N + c] *= inv_d;
            I[k * N + c] *= inv_d;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
            const int r = t / N, c = t % N;
            if (r == k) continue;
            const double f = A[r * N + k];
            if (c != k) A[t] -= f * A[k * N + c];
            I[t] -= f * I[k * N + c];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < N; r += blockDim.x)
            if (r != k) A[r * N + k] = 0.0;
        __syncthreads();
    }
    for (int t = threadIdx.x; t < N * N; t += blockDim.x) {
        const int r = t / N, c = t % N;
        inv[(long long)c * N + r] = I[t];
    }
}

// ---- V-cycle kernels: p-levels (m modes per cell, pattern rowptr / colidx)
// out = Dinv in (add: out += Dinv in); one thread per scalar row
__global__ void k_bdiag(long long J, int m, const double* __restrict__ inv, const double* __restrict__ in,
                        double* __restrict__ out, int add) {
    GRID_STRIDE(t, J * m) {
        const long long j = t / m;
        const int r = (int)(t - j * m);
        const double* B = inv + j * (long long)m * m;
        const double* v = in + j * m;
        double acc = 0.0;
        for (int c = 0; c < m; ++c) acc += B[(long long)c * m + r] * v[c];
        out[t] = add ? out[t] + acc : acc;
    }
}

// rows r < mo of each cell of (b - A x) into out[j * mo + r] (mo = m: the full residual)
__global__ void k_resid(long long J, int m, int mo, const long long* __restrict__ rowptr, const int* __restrict__ colidx,
                        const double* __restrict__ vals, const double* __restrict__ x, const double* __restrict__ b,
                        double* __restrict__ out) {
    GRID_STRIDE(t, J * mo) {
        const long long j = t / mo;
        const int r = (int)(t - j * mo);
        double acc = b[j * m + r];
        for (long long bb = rowptr[j]; bb < rowptr[j + 1]; ++bb) {
            const double* blk = vals + bb * (long long)m * m;
            const double* xb = x + (long long)colidx[bb] * m;
            for (int c = 0; c < m; ++c) acc -= blk[(long long)c * m + r] * xb[c];
        }
        out[t] = acc;
    }
}

// x[j * m + r] += xc[j * mc + r] for r < mc (prolongation of the lower-degree correction)
__global__ void k_inject_add(long long J, int m, int mc, const double* __restrict__ xc, double* __restrict__ x) {
    GRID_STRIDE(t, J * mc) {
        const long long j = t / mc;
        const int r = (int)(t - j * mc);
        x[j * m + r] += xc[t];
    }
}

// ---- structured levels
// first sweep from x = 0: x = omega b / diag
__global__ void k_jac0(SGeom g, const double* __restrict__ st, const double* __restrict__ b, double* __restrict__ x) {
    GRID_STRIDE(i, g.N) {
        const double d = st[i];
        x[i] = (d != 0.0) ? OMEGA * b[i] / d : 0.0;
    }
}

// xo = x + omega (b - A x) / diag
__global__ void k_jac(SGeom g, const double* __restrict__ st, const double* __restrict__ b,
                      const double* __restrict__ x, double* __restrict__ xo) {
    GRID_STRIDE(i, g.N) {
        const double d = st[i];
        xo[i] = x[i] + ((d != 0.0) ? OMEGA * (b[i] - s_apply_row(g, st, x, i)) / d : 0.0);
    }
}

// bc[I] = sum over the cells of aggregate I of (b - A x)
__global__ void k_agg_restrict(SGeom gf, SGeom gc, const double* __restrict__ st, const double* __restrict__ b,
                               const double* __restrict__ x, double* __restrict__ bc) {
    GRID_STRIDE(I, gc.N) {
        int IJK[3];
        s_ijk(gc, I, IJK);
        double acc = 0.0;
        for (int a = 0; a < 8; ++a) {
            int ijk[3];
            bool ok = true;
            for (int d = 0; d < 3; ++d) {
                ijk[d] = 2 * IJK[d] + ((a >> d) & 1);
                ok = ok && ijk[d] < gf.n[d];
            }
            if (!ok) continue;
            long long i = 0;
            for (int d = 0; d < 3; ++d) i += (long long)ijk[d] * gf.stride[d];
            acc += b[i] - s_apply_row(gf, st, x, i);
        }
        bc[I] = acc;
    }
}

// x[i] += xc[aggregate of i]
__global__ void k_agg_prolong(SGeom gf, SGeom gc, const double* __restrict__ xc, double* __restrict__ x) {
    GRID_STRIDE(i, gf.N) {
        int ijk[3];
        s_ijk(gf, i, ijk);
        x[i] += xc[s_agg(gc, ijk)];
    }
}

// x = M b, dense column-major (coarsest level)
__global__ void k_dense_apply(long long N, const double* __restrict__ M, const double* __restrict__ b, double* __restrict__ x) {
    GRID_STRIDE(i, N) {
        double acc = 0.0;
        for (long long j = 0; j < N; ++j) acc += M[j * N + i] * b[j];
        x[i] = acc;
    }
}

int launch_grid(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }

}  // namespace

}  // namespace bosss

using namespace bosss;

struct bosss_pmg {
    struct PLevel {
        int m = 0;
        double* vals = nullptr;   // m x m blocks, column-major, the fine pattern
        double* inv = nullptr;    // block-Jacobi inverses
        double *b = nullptr, *x = nullptr, *r = nullptr;
    };
    struct HLevel {
        SGeom g{};
        double* st = nullptr;     // NS * N couplings
        double *b = nullptr, *x = nullptr, *x2 = nullptr;
    };
    int device = 0;
    long long J = 0;
    int m0 = 0;
    long long* rowptr = nullptr;
    int* colidx = nullptr;
    std::vector<PLevel> P;
    std::vector<HLevel> H;
    double* dense = nullptr;      // coarsest inverse (direct) or nullptr (Jacobi sweeps)
    double* in = nullptr;         // the cycle's input and output (graph-captured buffers)
    double* out = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<void*> owned;

    ~bosss_pmg() {
        if (exec) cudaGraphExecDestroy(exec);
        for (void* p : owned) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    double* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(double) * std::max<size_t>(n, 1)) != cudaSuccess) return nullptr;
        owned.push_back(p);
        return (double*)p;
    }

    // the structured part of the cycle from level l: input H[l].b, output in H[l].x
    void cycle_h(size_t l, cudaStream_t s) {
        HLevel& L = H[l];
        const int gr = launch_grid(L.g.N);
        if (l + 1 == H.size()) {
            if (dense) {
                k_dense_apply<<<gr, 256, 0, s>>>(L.g.N, dense, L.b, L.x);
            } else {
                k_jac0<<<gr, 256, 0, s>>>(L.g, L.st, L.b, L.x);
                for (int i = 1; i < COARSE_SWEEPS; ++i) {
                    k_jac<<<gr, 256, 0, s>>>(L.g, L.st, L.b, L.x, L.x2);
                    std::swap(L.x, L.x2);
                }
            }
            return;
        }
        HLevel& C = H[l + 1];
        k_jac0<<<gr, 256, 0, s>>>(L.g, L.st, L.b, L.x);
        for (int i = 1; i < NU_H; ++i) {
            k_jac<<<gr, 256, 0, s>>>(L.g, L.st, L.b, L.x, L.x2);
            std::swap(L.x, L.x2);
        }
        k_agg_restrict<<<launch_grid(C.g.N), 256, 0, s>>>(L.g, C.g, L.st, L.b, L.x, C.b);
        cycle_h(l + 1, s);
        k_agg_prolong<<<gr, 256, 0, s>>>(L.g, C.g, C.x, L.x);
        for (int i = 0; i < NU_H; ++i) {
            k_jac<<<gr, 256, 0, s>>>(L.g, L.st, L.b, L.x, L.x2);
            std::swap(L.x, L.x2);
        }
    }

    // p-level l: input P[l].b, output P[l].x
    void cycle_p(size_t l, cudaStream_t s) {
        PLevel& L = P[l];
        const int gr = launch_grid(J * L.m);
        k_bdiag<<<gr, 256, 0, s>>>(J, L.m, L.inv, L.b, L.x, 0);
        const bool last = l + 1 == P.size();
        const int mc = last ? 1 : P[l + 1].m;
        double* bc = last ? H[0].b : P[l + 1].b;
        k_resid<<<launch_grid(J * mc), 256, 0, s>>>(J, L.m, mc, rowptr, colidx, L.vals, L.x, L.b, bc);
        if (last) cycle_h(0, s);
        else cycle_p(l + 1, s);
        const double* xc = last ? H[0].x : P[l + 1].x;
        k_inject_add<<<launch_grid(J * mc), 256, 0, s>>>(J, L.m, mc, xc, L.x);
        k_resid<<<gr, 256, 0, s>>>(J, L.m, L.m, rowptr, colidx, L.vals, L.x, L.b, L.r);
        k_bdiag<<<gr, 256, 0, s>>>(J, L.m, L.inv, L.r, L.x, 1);
    }

    void cycle(cudaStream_t s) {
        if (!P.empty()) {
            cycle_p(0, s);   // P[0].b = in, P[0].x = out
        } else {
            cudaMemcpyAsync(H[0].b, in, sizeof(double) * J, cudaMemcpyDeviceToDevice, s);
            cycle_h(0, s);
            cudaMemcpyAsync(out, H[0].x, sizeof(double) * J, cudaMemcpyDeviceToDevice, s);
        }
    }
};

namespace bosss {

int pmg_create(const bosss_handle* h, const bosss_bsr* A, bosss_pmg** out) {
    if (!h || !A || !out) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    const GridConst& g = h->base.g;
    const int m0 = np_of(h->D, h->K);
    if (h->ndom != h->ncod || h->ndom != (int64_t)g.J * m0)
        return fail(BOSSS_ERR_BAD_ARG, "the multigrid preconditioner needs a scalar square operator");
    if (A->nbr != g.J || A->nbc != g.J || A->br != m0 || A->bc != m0 || A->device != h->device)
        return fail(BOSSS_ERR_BAD_ARG, "the matrix is not the cell-block Jacobian of this operator");
    if (h->base.g.gn[0] != g.n[0] || h->base.g.gn[1] != g.n[1] || h->base.g.gn[2] != g.n[2])
        return fail(BOSSS_ERR_BAD_ARG, "the multigrid preconditioner needs a whole grid");
    CUDA_TRY(cudaSetDevice(h->device));
    bosss_pmg* M = new bosss_pmg();
    auto bail = [&](int rc) {
        delete M;
        return rc;
    };
    auto cuda_bail = [&](cudaError_t e, const char* what) {
        delete M;
        return fail(BOSSS_ERR_CUDA, std::string("multigrid setup (") + what + "): " + cudaGetErrorString(e));
    };
    M->device = h->device;
    M->J = g.J;
    M->m0 = m0;
    cudaError_t e = cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_bail(e, "stream");
    cudaStream_t s = M->stream;
    // the pattern (self first, then face neighbours) is shared by every p-level
    M->rowptr = (long long*)M->alloc((size_t)g.J + 1);
    M->colidx = (int*)M->alloc(((size_t)A->nnzb + 1) / 2);
    M->in = M->alloc((size_t)g.J * m0);
    M->out = M->alloc((size_t)g.J * m0);
    if (!M->rowptr || !M->colidx || !M->in || !M->out) return cuda_bail(cudaErrorMemoryAllocation, "alloc");
    e = cudaMemcpyAsync(M->rowptr, A->d_rowptr, sizeof(long long) * (g.J + 1), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(M->colidx, A->d_colidx, sizeof(int) * A->nnzb, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_bail(e, "pattern");
    // p-levels: degrees K, K-1, ..., 1
    int* sing = (int*)M->alloc(1);
    if (!sing) return cuda_bail(cudaErrorMemoryAllocation, "alloc");
    cudaMemsetAsync(sing, 0, sizeof(int), s);
    for (int k = h->K; k >= 1; --k) {
        bosss_pmg::PLevel L;
        L.m = np_of(h->D, k);
        const size_t nv = (size_t)A->nnzb * L.m * L.m, nx = (size_t)g.J * L.m;
        L.vals = M->alloc(nv);
        L.inv = M->alloc((size_t)g.J * L.m * L.m);
        // the finest level reads its right-hand side from `in` and leaves the result in `out`
        L.b = (k == h->K) ? M->in : M->alloc(nx);
        L.x = (k == h->K) ? M->out : M->alloc(nx);
        L.r = M->alloc(nx);
        if (!L.vals || !L.inv || !L.b || !L.x || !L.r) return cuda_bail(cudaErrorMemoryAllocation, "alloc");
        k_sub_blocks<<<launch_grid((long long)nv), 256, 0, s>>>(A->nnzb, m0, L.m, A->d_vals, L.vals);
        const size_t smem = (size_t)2 * L.m * L.m * 8;
        e = cudaFuncSetAttribute(k_invert_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_bail(e, "block inverse");
        k_invert_diag<double><<<(unsigned)g.J, 128, smem, s>>>(L.m, M->rowptr, L.vals, L.inv, sing);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_bail(e, "block inverse");
        M->P.push_back(L);
    }
    // structured levels: the piecewise-constant level of the grid, then aggregates
    {
        bosss_pmg::HLevel L;
        for (int d = 0; d < 3; ++d) {
            L.g.n[d] = d < g.D ? g.n[d] : 1;
            L.g.per[d] = d < g.D ? g.periodic[d] : 0;
            L.g.stride[d] = d < g.D ? g.stride[d] : 1;
        }
        L.g.N = g.J;
        M->H.push_back(L);
    }
    while (true) {
        const SGeom& f = M->H.back().g;
        if (f.N <= COARSE_MAX || (f.n[0] == 1 && f.n[1] == 1 && f.n[2] == 1)) break;
        bosss_pmg::HLevel C;
        for (int d = 0; d < 3; ++d) {
            C.g.n[d] = (f.n[d] + 1) / 2;
            C.g.per[d] = f.per[d];
        }
        C.g.stride[2] = 1;
        C.g.stride[1] = C.g.n[2];
        C.g.stride[0] = (long long)C.g.n[1] * C.g.n[2];
        C.g.N = (long long)C.g.n[0] * C.g.n[1] * C.g.n[2];
        M->H.push_back(C);
    }
    for (auto& L : M->H) {
        L.st = M->alloc((size_t)NS * L.g.N);
        L.b = M->alloc((size_t)L.g.N);
        L.x = M->alloc((size_t)L.g.N);
        L.x2 = M->alloc((size_t)L.g.N);
        if (!L.st || !L.b || !L.x || !L.x2) return cuda_bail(cudaErrorMemoryAllocation, "alloc");
    }
    k_p0_extract<<<launch_grid(g.J), 256, 0, s>>>(M->H[0].g, m0, M->rowptr, M->colidx, A->d_vals, M->H[0].st);
    for (size_t l = 1; l < M->H.size(); ++l)
        k_agg_build<<<launch_grid(M->H[l].g.N), 256, 0, s>>>(M->H[l - 1].g, M->H[l].g, M->H[l - 1].st, M->H[l].st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_bail(e, "structured levels");
    int flag = 0;
    e = cudaMemcpyAsync(&flag, sing, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_bail(e, "setup");
    if (flag) return bail(fail(BOSSS_ERR_BAD_ARG, "singular diagonal block in the multigrid smoother"));
    // coarsest level: dense inverse unless singular
    const bosss_pmg::HLevel& Lc = M->H.back();
    if (Lc.g.N <= COARSE_MAX) {
        const long long N = Lc.g.N;
        double* Md = M->alloc((size_t)N * N);
        double* inv = M->alloc((size_t)N * N);
        if (!Md || !inv) return cuda_bail(cudaErrorMemoryAllocation, "alloc");
        k_dense<<<launch_grid(N), 256, 0, s>>>(Lc.g, Lc.st, Md);
        const size_t smem = (size_t)2 * N * N * 8;
        e = cudaFuncSetAttribute(k_dense_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) e = cudaMemsetAsync(sing, 0, sizeof(int), s);
        if (e == cudaSuccess) k_dense_inverse<<<1, 256, smem, s>>>((int)N, Md, inv, sing);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, sing, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_bail(e, "coarsest level");
        M->dense = flag ? nullptr : inv;
    }
    // capture one V-cycle (input M->in, output M->out) as a graph
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_bail(e, "capture");
    M->cycle(s);
    e = cudaStreamEndCapture(s, &graph);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&M->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_bail(e, "graph");
    *out = M;
    return BOSSS_OK;
}

int pmg_apply(bosss_pmg* M, const double* b, double* x, cudaStream_t s) {
    const size_t bytes = sizeof(double) * (size_t)M->J * M->m0;
    CUDA_TRY(cudaMemcpyAsync(M->in, b, bytes, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaGraphLaunch(M->exec, s));
    CUDA_TRY(cudaMemcpyAsync(x, M->out, bytes, cudaMemcpyDeviceToDevice, s));
    return BOSSS_OK;
}

void pmg_destroy(bosss_pmg* M) {
    if (!M) return;
    cudaSetDevice(M->device);
    delete M;
}

}  // namespace bosss

extern "C" {

int bosss_b200_pmg_create(const bosss_handle* h, const bosss_bsr* A, bosss_pmg** out) {
    return pmg_create(h, A, out);
}

int bosss_b200_pmg_apply_device(bosss_pmg* M, const double* b_dev, double* x_dev, void* stream) {
    if (!M || !b_dev || !x_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(M->device));
    return pmg_apply(M, b_dev, x_dev, stream ? (cudaStream_t)stream : M->stream);
}

int bosss_b200_pmg_info(const bosss_pmg* M, int32_t* n_p_levels, int32_t* n_h_levels, int64_t* coarsest,
                        int32_t* coarsest_direct) {
    if (!M) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (n_p_levels) *n_p_levels = (int32_t)M->P.size();
    if (n_h_levels) *n_h_levels = (int32_t)M->H.size();
    if (coarsest) *coarsest = M->H.back().g.N;
    if (coarsest_direct) *coarsest_direct = M->dense ? 1 : 0;
    return BOSSS_OK;
}

int bosss_b200_pmg_destroy(bosss_pmg* M) {
    pmg_destroy(M);
    return BOSSS_OK;
}

}  // extern "C"
