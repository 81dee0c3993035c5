// solver.cuh -- vector kernels and a restarted GMRES(m) on device vectors.
//
// The Krylov solver is the matrix-free consumer of the operator's JVP that replaces
// the FD directional derivative of the reference's Newton-GMRES (Newton.cs:1231-1495,
// MatrixFreeGMRES.Solve + dirder). Arithmetic type T is double (outer solves) or float
// (inner solves of the mixed-precision iterative refinement).
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <functional>
#include <vector>

namespace bosss {

// ---- vector kernels (grid-stride) ----
template <class T>
__global__ void k_axpby(long long n, T a, const T* __restrict__ x, T b, T* __restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = (b == T(0)) ? a * x[i] : a * x[i] + b * y[i];
}

template <class T>
__global__ void k_scale(long long n, T a, T* __restrict__ x) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] *= a;
}

template <class TI, class TO>
__global__ void k_convert(long long n, const TI* __restrict__ x, TO* __restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = (TO)x[i];
}

// partial dot products: one FP64 partial per block (partials[blockIdx.x]), finished by the
// caller (the grid is a fixed number of blocks)
template <class T>
__global__ void k_dot_partials(long long n, const T* __restrict__ x, const T* __restrict__ y,
                               double* __restrict__ partials) {
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc += (double)x[i] * (double)y[i];
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    }
}

// w -= sum_k h[k] V_k
template <class T>
__global__ void k_multiaxpy(long long n, int m, const T* __restrict__ V, long long ldv, const double* __restrict__ h,
                            T* __restrict__ w) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double acc = (double)w[i];
        for (int k = 0; k < m; ++k) acc -= h[k] * (double)V[(long long)k * ldv + i];
        w[i] = (T)acc;
    }
}

// x += sum_k y[k] Z_k
template <class T>
__global__ void k_multiaxpy_add(long long n, int m, const T* __restrict__ Z, long long ldz, const double* __restrict__ y,
                                T* __restrict__ x) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double acc = (double)x[i];
        for (int k = 0; k < m; ++k) acc += y[k] * (double)Z[(long long)k * ldz + i];
        x[i] = (T)acc;
    }
}

// Gauss-Jordan with partial pivoting of the diagonal block of every block row; one CTA
// per block, the augmented matrix [A | I] in shared memory. Output column-major.
template <class T>
__global__ void k_invert_diag(int nb, const long long* __restrict__ rowptr, const double* __restrict__ vals, T* __restrict__ inv,
                              int* __restrict__ singular) {
    extern __shared__ double sm[];
    const int j = blockIdx.x;
    double* Am = sm;              // nb x nb, row-major
    double* Im = sm + nb * nb;    // nb x nb, row-major
    __shared__ int piv;
    const double* blk = vals + rowptr[j] * (long long)nb * nb;   // diagonal block is the first of the row
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        const int r = t / nb, c = t % nb;
        Am[t] = blk[(long long)c * nb + r];
        Im[t] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        if (threadIdx.x == 0) {
            int p = k;
            double best = fabs(Am[k * nb + k]);
            for (int r = k + 1; r < nb; ++r)
                if (fabs(Am[r * nb + k]) > best) {
                    best = fabs(Am[r * nb + k]);
                    p = r;
                }
            piv = p;
            if (best == 0.0) atomicExch(singular, 1);
        }
        __syncthreads();
        const int p = piv;
        if (p != k)
            for (int c = threadIdx.x; c < nb; c += blockDim.x) {
                double t0 = Am[k * nb + c];
                Am[k * nb + c] = Am[p * nb + c];
                Am[p * nb + c] = t0;
                t0 = Im[k * nb + c];
                Im[k * nb + c] = Im[p * nb + c];
                Im[p * nb + c] = t0;
            }
        __syncthreads();
        const double d = Am[k * nb + k];
        const double inv_d = (d != 0.0) ? 1.0 / d : 0.0;
        __syncthreads();
        for (int c = threadIdx.x; c < nb; c += blockDim.x) {
            Am[k * nb + c] *= inv_d;
            Im[k * nb + c] *= inv_d;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
            const int r = t / nb, c = t % nb;
            if (r == k) continue;
            const double f = Am[r * nb + k];
            if (c != k) Am[t] -= f * Am[k * nb + c];
            Im[t] -= f * Im[k * nb + c];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < nb; r += blockDim.x)
            if (r != k) Am[r * nb + k] = 0.0;
        __syncthreads();
    }
    T* out = inv + (long long)j * nb * nb;
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        const int r = t / nb, c = t % nb;
        out[(long long)c * nb + r] = (T)Im[t];
    }
}

constexpr int RED_BLOCKS = 296;   // 2 x 148 SMs
constexpr int RED_THREADS = 512;
constexpr int MDOT_CH = 8;        // vectors per pass of the multi-dot

// <V_k, w> for k in [k0, min(k0 + MDOT_CH, m)), w read once per pass: one FP64 partial per
// (k, block) in partials[k * RED_BLOCKS + block]
template <class T>
__global__ void __launch_bounds__(RED_THREADS) k_mdot(long long n, int k0, int m, const T* __restrict__ V, long long ldv,
                                                     const T* __restrict__ w, double* __restrict__ partials) {
    double acc[MDOT_CH];
#pragma unroll
    for (int c = 0; c < MDOT_CH; ++c) acc[c] = 0.0;
    const int nc = min(MDOT_CH, m - k0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double wi = (double)w[i];
#pragma unroll
        for (int c = 0; c < MDOT_CH; ++c)
            if (c < nc) acc[c] += (double)V[(long long)(k0 + c) * ldv + i] * wi;
    }
    __shared__ double sh[MDOT_CH][RED_THREADS / 32];
#pragma unroll
    for (int c = 0; c < MDOT_CH; ++c) {
        double a = acc[c];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        for (int c = 0; c < nc; ++c) {
            double a = (threadIdx.x < (blockDim.x >> 5)) ? sh[c][threadIdx.x] : 0.0;
            for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
            if (threadIdx.x == 0) partials[(long long)(k0 + c) * gridDim.x + blockIdx.x] = a;
        }
    }
}

// out[k] = sum_b partials[k * RED_BLOCKS + b] for k < m (one block per k, fixed order)
static __global__ void k_finish_partials(const double* __restrict__ partials, double* __restrict__ out) {
    const int k = blockIdx.x;
    double a = 0.0;
    for (int i = threadIdx.x; i < RED_BLOCKS; i += blockDim.x) a += partials[(long long)k * RED_BLOCKS + i];
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x < 32) {
        a = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (threadIdx.x == 0) out[k] = a;
    }
}

// x *= *f (scale factor in device memory)
template <class T>
__global__ void k_scale_dev(long long n, const double* __restrict__ f, T* __restrict__ x) {
    const double a = *f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = (T)((double)x[i] * a);
}

// Device work area of the GMRES(m) Arnoldi process, (m+1)*(m+8) doubles:
// h[m+1] (Gram-Schmidt coefficients, pass 1), h2[m+1] (pass 2), H[(m+1)*m] (Hessenberg,
// row-major, after the rotations), cs[m], sn[m], g[m+1], sc[8] (sc[0] ||w||^2,
// sc[1] scale of the next basis vector, sc[2] residual estimate, sc[3] breakdown flag)
struct GmresDev {
    double *h, *h2, *H, *cs, *sn, *g, *sc;
    __host__ __device__ GmresDev(double* base, int m) {
        h = base;
        h2 = h + (m + 1);
        H = h2 + (m + 1);
        cs = H + (size_t)(m + 1) * m;
        sn = cs + m;
        g = sn + m;
        sc = g + (m + 1);
    }
};
__host__ __device__ constexpr long long gmres_dev_doubles(int m) { return (long long)(m + 1) * (m + 8); }

// start of a cycle: beta = ||r|| from sc[0]; g = beta e_1; scale 1/beta for V_0
static __global__ void k_gmres_start(double* base, int m) {
    GmresDev d(base, m);
    const double beta = sqrt(fmax(d.sc[0], 0.0));
    for (int i = 0; i <= m; ++i) d.g[i] = 0.0;
    d.g[0] = beta;
    d.sc[1] = beta > 0.0 ? 1.0 / beta : 0.0;
    d.sc[2] = beta;
    d.sc[3] = 0.0;
}

// Arnoldi step k: h += h2 (second Gram-Schmidt pass), h[k+1] = ||w||, Givens rotations,
// column k of H, g, residual estimate |g[k+1]|, scale 1/h[k+1] of the new basis vector
static __global__ void k_gmres_step(double* base, int m, int k) {
    GmresDev d(base, m);
    double h[256];
    for (int j = 0; j <= k; ++j) h[j] = d.h[j] + d.h2[j];
    const double hn = sqrt(fmax(d.sc[0], 0.0));
    h[k + 1] = hn;
    for (int j = 0; j < k; ++j) {
        const double t = d.cs[j] * h[j] + d.sn[j] * h[j + 1];
        h[j + 1] = -d.sn[j] * h[j] + d.cs[j] * h[j + 1];
        h[j] = t;
    }
    const double r = hypot(h[k], h[k + 1]);
    d.cs[k] = (r == 0.0) ? 1.0 : h[k] / r;
    d.sn[k] = (r == 0.0) ? 0.0 : h[k + 1] / r;
    h[k] = r;
    d.g[k + 1] = -d.sn[k] * d.g[k];
    d.g[k] = d.cs[k] * d.g[k];
    for (int j = 0; j <= k; ++j) d.H[(size_t)j * m + k] = h[j];
    d.sc[1] = hn > 0.0 ? 1.0 / hn : 0.0;
    d.sc[2] = fabs(d.g[k + 1]);
    d.sc[3] = (hn == 0.0) ? 1.0 : 0.0;
}

struct GmresResult {
    int iters = 0;
    bool converged = false;
    double res0 = 0.0, res = 0.0;
    int error = 0;   // CUDA error code, 0 = ok
};

// Restarted GMRES(m), m <= 254, with classical Gram-Schmidt and one reorthogonalisation pass,
// solving A x = b for device vectors of type T. `apply(x, y)` computes y = A x on `stream`.
// Convergence: ||b - A x|| <= max(rtol ||b||, atol). The Arnoldi process runs on the device:
// the dot products are reduced, the Hessenberg column is rotated and the residual estimate
// is formed by device kernels, so an iteration enqueues its launches without waiting. The
// host reads the residual estimate of the previous iteration through an event while the
// current one runs (at most one iteration beyond convergence), and reads the small
// Hessenberg system once per restart for the back substitution. Work arrays are device
// buffers owned by the caller: V ((m+1) * n), w (n), partials (RED_BLOCKS * (m+1)),
// work (gmres_dev_doubles(m)).
template <class T>
GmresResult gmres(long long n, const std::function<cudaError_t(const T*, T*)>& apply, const T* b, T* x, int m,
                  int max_iters, double rtol, double atol, T* V, T* w, double* partials, double* work,
                  cudaStream_t s, double* pinned = nullptr) {
    GmresResult R;
    if (m > 254) m = 254;
    auto grid = [&]() { return (int)std::min<long long>((n + 255) / 256, 148LL * 8); };
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && !R.error) R.error = (int)e;
        return e == cudaSuccess;
    };
    GmresDev dv(work, m);
    // sum_k (k < cnt) <V_k, vec> -> out[k] on the device
    auto mdot = [&](int cnt, const T* vec, double* out) {
        for (int k0 = 0; k0 < cnt; k0 += MDOT_CH)
            k_mdot<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, k0, cnt, V, n, vec, partials);
        k_finish_partials<<<cnt, 256, 0, s>>>(partials, out);
        chk(cudaGetLastError());
    };
    auto norm2_dev = [&](const T* a) {   // ||a||^2 -> sc[0]
        k_mdot<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, 0, 1, a, n, a, partials);
        k_finish_partials<<<1, 256, 0, s>>>(partials, dv.sc);
        chk(cudaGetLastError());
    };
    // pinned host slots for the lagged residual checks: the caller's (8 doubles, kept across
    // calls: freeing pinned memory synchronises the device), else allocated here
    double* hres = pinned;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (!hres) chk(cudaMallocHost(&hres, sizeof(double) * 8));
    for (int i = 0; i < 2; ++i) chk(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    auto cleanup = [&]() {
        for (int i = 0; i < 2; ++i)
            if (ev[i]) cudaEventDestroy(ev[i]);
        if (hres && !pinned) cudaFreeHost(hres);
    };
    if (R.error) {
        cleanup();
        return R;
    }
    norm2_dev(b);
    chk(cudaMemcpyAsync(hres, dv.sc, sizeof(double), cudaMemcpyDeviceToHost, s));
    chk(cudaStreamSynchronize(s));
    const double bnorm = std::sqrt(std::max(hres[0], 0.0));
    const double target = std::max(rtol * bnorm, atol);
    std::vector<double> H((size_t)(m + 1) * m), g(m + 1), y(m);
    bool first = true;
    while (R.iters < max_iters && !R.error) {
        // r = b - A x -> w, beta = ||r||
        chk(apply(x, w));
        k_axpby<T><<<grid(), 256, 0, s>>>(n, T(1), b, T(-1), w);
        chk(cudaGetLastError());
        norm2_dev(w);
        k_gmres_start<<<1, 1, 0, s>>>(work, m);
        chk(cudaMemcpyAsync(hres, dv.sc + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
        chk(cudaStreamSynchronize(s));
        const double beta = hres[0];
        if (first) {
            R.res0 = beta;
            first = false;
        }
        R.res = beta;
        if (beta <= target || !(beta > 0.0)) {
            R.converged = beta <= target;
            break;
        }
        chk(cudaMemcpyAsync(V, w, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        k_scale_dev<T><<<grid(), 256, 0, s>>>(n, dv.sc + 1, V);
        int k = 0, used = 0;
        bool stop = false;
        for (; k < m && R.iters < max_iters && !R.error; ++k) {
            T* vk = V + (long long)k * n;
            T* vk1 = V + (long long)(k + 1) * n;
            chk(apply(vk, vk1));
            mdot(k + 1, vk1, dv.h);                                   // classical Gram-Schmidt
            k_multiaxpy<T><<<grid(), 256, 0, s>>>(n, k + 1, V, n, dv.h, vk1);
            mdot(k + 1, vk1, dv.h2);                                  // and a second pass
            k_multiaxpy<T><<<grid(), 256, 0, s>>>(n, k + 1, V, n, dv.h2, vk1);
            norm2_dev(vk1);
            k_gmres_step<<<1, 1, 0, s>>>(work, m, k);
            k_scale_dev<T><<<grid(), 256, 0, s>>>(n, dv.sc + 1, vk1);
            chk(cudaMemcpyAsync(hres + 2 * (k & 1), dv.sc + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
            chk(cudaEventRecord(ev[k & 1], s));
            ++R.iters;
            used = k + 1;
            // residual estimate of the previous iteration (this one is already enqueued)
            if (k > 0) {
                chk(cudaEventSynchronize(ev[(k - 1) & 1]));
                const double res = hres[2 * ((k - 1) & 1)], brk = hres[2 * ((k - 1) & 1) + 1];
                R.res = res;
                if (brk != 0.0) {
                    used = k;   // the basis ended with vector k: this iteration's column is invalid
                    stop = true;
                    break;
                }
                if (res <= target) {
                    stop = true;
                    ++k;
                    break;
                }
            }
        }
        chk(cudaStreamSynchronize(s));
        if (!stop && used > 0) R.res = hres[2 * ((used - 1) & 1)];
        if (used == 0) break;
        // back substitution on the host (the Hessenberg system is (m+1) x m)
        chk(cudaMemcpyAsync(H.data(), dv.H, sizeof(double) * (size_t)(m + 1) * m, cudaMemcpyDeviceToHost, s));
        chk(cudaMemcpyAsync(g.data(), dv.g, sizeof(double) * (m + 1), cudaMemcpyDeviceToHost, s));
        chk(cudaStreamSynchronize(s));
        R.res = std::fabs(g[used]);
        for (int i = used - 1; i >= 0; --i) {
            double acc = g[i];
            for (int j = i + 1; j < used; ++j) acc -= H[(size_t)i * m + j] * y[j];
            y[i] = acc / H[(size_t)i * m + i];
        }
        chk(cudaMemcpyAsync(dv.h, y.data(), sizeof(double) * used, cudaMemcpyHostToDevice, s));
        k_multiaxpy_add<T><<<grid(), 256, 0, s>>>(n, used, V, n, dv.h, x);
        chk(cudaGetLastError());
        chk(cudaStreamSynchronize(s));
        // the residual estimate is confirmed with the true residual at the next restart
    }
    cleanup();
    return R;
}

}  // namespace bosss
