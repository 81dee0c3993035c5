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

// partial dot products: one FP64 partial per block (partials[blockIdx.x]); the host
// finishes the sum (the grid is a fixed number of blocks)
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

// multi-dot: h[k] = <V_k, w> for k < m (classical Gram-Schmidt step), one partial per (k, block)
template <class T>
__global__ void k_multidot_partials(long long n, int m, const T* __restrict__ V, long long ldv,
                                    const T* __restrict__ w, double* __restrict__ partials) {
    for (int k = 0; k < m; ++k) {
        double acc = 0.0;
        const T* v = V + (long long)k * ldv;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
            acc += (double)v[i] * (double)w[i];
        __shared__ double sh[32];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x < 32) {
            acc = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (threadIdx.x == 0) partials[(long long)k * gridDim.x + blockIdx.x] = acc;
        }
        __syncthreads();
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

constexpr int RED_BLOCKS = 296;   // 2 x 148 SMs
constexpr int RED_THREADS = 512;

struct GmresResult {
    int iters = 0;
    bool converged = false;
    double res0 = 0.0, res = 0.0;
    int error = 0;   // CUDA error code, 0 = ok
};

// Restarted GMRES(m) with classical Gram-Schmidt and one reorthogonalisation pass,
// solving A x = b for device vectors of type T. `apply(x, y)` computes y = A x on
// `stream`. Convergence: ||b - A x|| <= max(rtol ||b||, atol). Work arrays are device
// buffers owned by the caller: V ((m+1) * n), w (n), partials (RED_BLOCKS * (m+1)),
// hbuf (m+1 doubles).
template <class T>
GmresResult gmres(long long n, const std::function<cudaError_t(const T*, T*)>& apply, const T* b, T* x, int m,
                  int max_iters, double rtol, double atol, T* V, T* w, double* partials, double* hbuf,
                  cudaStream_t s) {
    GmresResult R;
    auto grid = [&]() { return (int)std::min<long long>((n + 255) / 256, 148LL * 8); };
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && !R.error) R.error = (int)e;
        return e == cudaSuccess;
    };
    std::vector<double> hp((size_t)RED_BLOCKS * (m + 1));
    auto dot = [&](const T* a, const T* c) -> double {
        k_dot_partials<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, a, c, partials);
        chk(cudaGetLastError());
        chk(cudaMemcpyAsync(hp.data(), partials, sizeof(double) * RED_BLOCKS, cudaMemcpyDeviceToHost, s));
        chk(cudaStreamSynchronize(s));
        double acc = 0.0;
        for (int i = 0; i < RED_BLOCKS; ++i) acc += hp[i];
        return acc;
    };
    auto multidot = [&](int k, const T* vv, std::vector<double>& h) {
        k_multidot_partials<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(n, k, V, n, vv, partials);
        chk(cudaGetLastError());
        chk(cudaMemcpyAsync(hp.data(), partials, sizeof(double) * RED_BLOCKS * k, cudaMemcpyDeviceToHost, s));
        chk(cudaStreamSynchronize(s));
        for (int j = 0; j < k; ++j) {
            double acc = 0.0;
            for (int i = 0; i < RED_BLOCKS; ++i) acc += hp[(size_t)j * RED_BLOCKS + i];
            h[j] = acc;
        }
    };
    const double bnorm = std::sqrt(std::max(dot(b, b), 0.0));
    const double target = std::max(rtol * bnorm, atol);
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), h(m + 1), h2(m + 1);
    bool first = true;
    while (R.iters < max_iters && !R.error) {
        // r = b - A x -> V_0
        chk(apply(x, w));
        k_axpby<T><<<grid(), 256, 0, s>>>(n, T(1), b, T(-1), w);   // w = b - A x
        chk(cudaGetLastError());
        const double beta = std::sqrt(std::max(dot(w, w), 0.0));
        if (first) {
            R.res0 = beta;
            first = false;
        }
        R.res = beta;
        if (beta <= target) {
            R.converged = true;
            break;
        }
        k_axpby<T><<<grid(), 256, 0, s>>>(n, T(1.0 / beta), w, T(0), V);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        for (; k < m && R.iters < max_iters; ++k, ++R.iters) {
            T* vk = V + (long long)k * n;
            T* vk1 = V + (long long)(k + 1) * n;
            chk(apply(vk, vk1));
            // classical Gram-Schmidt, twice
            multidot(k + 1, vk1, h);
            chk(cudaMemcpyAsync(hbuf, h.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, s));
            k_multiaxpy<T><<<grid(), 256, 0, s>>>(n, k + 1, V, n, hbuf, vk1);
            multidot(k + 1, vk1, h2);
            chk(cudaMemcpyAsync(hbuf, h2.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, s));
            k_multiaxpy<T><<<grid(), 256, 0, s>>>(n, k + 1, V, n, hbuf, vk1);
            for (int j = 0; j <= k; ++j) h[j] += h2[j];
            const double hn = std::sqrt(std::max(dot(vk1, vk1), 0.0));
            h[k + 1] = hn;
            if (hn > 0.0) k_scale<T><<<grid(), 256, 0, s>>>(n, T(1.0 / hn), vk1);
            // Givens rotations
            for (int j = 0; j < k; ++j) {
                const double t = cs[j] * h[j] + sn[j] * h[j + 1];
                h[j + 1] = -sn[j] * h[j] + cs[j] * h[j + 1];
                h[j] = t;
            }
            const double r = std::hypot(h[k], h[k + 1]);
            cs[k] = (r == 0.0) ? 1.0 : h[k] / r;
            sn[k] = (r == 0.0) ? 0.0 : h[k + 1] / r;
            h[k] = r;
            h[k + 1] = 0.0;
            g[k + 1] = -sn[k] * g[k];
            g[k] = cs[k] * g[k];
            for (int j = 0; j <= k; ++j) H[(size_t)j * m + k] = h[j];
            R.res = std::fabs(g[k + 1]);
            if (R.res <= target || hn == 0.0) {
                ++k;
                ++R.iters;
                break;
            }
        }
        // back substitution, x += V y
        for (int i = k - 1; i >= 0; --i) {
            double acc = g[i];
            for (int j = i + 1; j < k; ++j) acc -= H[(size_t)i * m + j] * y[j];
            y[i] = acc / H[(size_t)i * m + i];
        }
        chk(cudaMemcpyAsync(hbuf, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
        k_multiaxpy_add<T><<<grid(), 256, 0, s>>>(n, k, V, n, hbuf, x);
        chk(cudaGetLastError());
        chk(cudaStreamSynchronize(s));
        if (R.res <= target) {
            // confirm with the true residual at the next restart
            continue;
        }
    }
    return R;
}

}  // namespace bosss
