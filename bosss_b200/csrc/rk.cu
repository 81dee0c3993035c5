// rk.cu -- explicit Runge-Kutta time stepping around the device evaluator.
//
// RungeKutta.Perform / PerformStage (TimeStepping/RungeKutta.cs:242-330) with
// ExplicitEuler.ComputeChangeRate (ExplicitEuler.cs:223-229): k_s = Op(u_s),
// u_s = y0 - dt sum_r a[s][r] k_r, y1 = y0 - dt sum_s b[s] k_s (the operator is the spatial
// residual, du/dt = -Op(u) for the orthonormal basis). Each stage is one residual launch
// plus one fused combination launch; whole steps can be captured into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "handle.h"

namespace bosss {

constexpr int RK_MAX_STAGES = 8;

struct RkCoef {
    int ns;
    double c[RK_MAX_STAGES];
};

// out = y0 + sum_r coef.c[r] * k_r   (k stored stage-major, stride n). The final update of a
// step passes the state as both y0 and out (in place): each element is read before it is
// written by the same thread, so y0 and out are not declared __restrict__.
__global__ void k_rk_combine(long long n, const double* y0, const double* __restrict__ k, RkCoef coef, double* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double v = y0[i];
        for (int r = 0; r < coef.ns; ++r) v += coef.c[r] * k[(long long)r * n + i];
        out[i] = v;
    }
}

struct Tableau {
    int s;
    double a[RK_MAX_STAGES][RK_MAX_STAGES];
    double b[RK_MAX_STAGES];
    double c[RK_MAX_STAGES];
};

static int make_tableau(int stages, const double* a, const double* b, const double* c, Tableau& T) {
    std::memset(&T, 0, sizeof(T));
    if (!a || !b || !c || stages < 1 || stages > RK_MAX_STAGES)
        return fail(BOSSS_ERR_BAD_ARG, "Runge-Kutta tableau: 1.." + std::to_string(RK_MAX_STAGES) + " stages");
    T.s = stages;
    for (int i = 0; i < stages; ++i) {
        for (int j = 0; j < stages; ++j) {
            if (j >= i && a[i * stages + j] != 0.0) return fail(BOSSS_ERR_BAD_ARG, "Runge-Kutta tableau must be explicit");
            T.a[i][j] = a[i * stages + j];
        }
        T.b[i] = b[i];
        T.c[i] = c[i];
    }
    return BOSSS_OK;
}

// one step on device buffers: U (in/out), work = (s+1) * n doubles (k_0..k_{s-1}, stage state)
static int rk_step(bosss_handle* h, const Tableau& T, double dt, double time, double* U, double* work, cudaStream_t st) {
    const long long n = h->ndom;
    double* K = work;
    double* us = work + (long long)T.s * n;
    const int grid = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    for (int s = 0; s < T.s; ++s) {
        const double* in = U;
        if (s > 0) {
            RkCoef cf{};
            cf.ns = s;
            for (int r = 0; r < s; ++r) cf.c[r] = -dt * T.a[s][r];
            k_rk_combine<<<grid, 256, 0, st>>>(n, U, K, cf, us);
            CUDA_TRY(cudaGetLastError());
            in = us;
        }
        int rc = run_mode(h, MODE_RES, 1.0, 0.0, in, nullptr, K + (long long)s * n, time + T.c[s] * dt, st);
        if (rc) return rc;
    }
    RkCoef cf{};
    cf.ns = T.s;
    for (int r = 0; r < T.s; ++r) cf.c[r] = -dt * T.b[r];
    k_rk_combine<<<grid, 256, 0, st>>>(n, U, K, cf, U);
    CUDA_TRY(cudaGetLastError());
    return BOSSS_OK;
}

}  // namespace bosss

using namespace bosss;

extern "C" {

int bosss_b200_rk_work_size(const bosss_handle* h, int32_t stages, int64_t* n_doubles) {
    if (!h || !n_doubles) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (stages < 1 || stages > RK_MAX_STAGES) return fail(BOSSS_ERR_BAD_ARG, "bad number of stages");
    *n_doubles = (int64_t)(stages + 1) * h->ndom;
    return BOSSS_OK;
}

int bosss_b200_rk_steps_device(bosss_handle* h, int32_t stages, const double* a, const double* b, const double* c,
                               double dt, int32_t nsteps, double time, double* U_dev, double* work_dev,
                               int32_t use_graph, void* stream) {
    if (!h || !U_dev || !work_dev || nsteps < 0) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    if (h->ndom != h->ncod) return fail(BOSSS_ERR_BAD_ARG, "time stepping needs a square operator");
    Tableau T;
    int rc = make_tableau(stages, a, b, c, T);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    if (!use_graph) {
        for (int i = 0; i < nsteps; ++i) {
            rc = rk_step(h, T, dt, time + i * dt, U_dev, work_dev, st);
            if (rc) return rc;
        }
        return BOSSS_OK;
    }
    // one step captured once and launched nsteps times; the supported components do not
    // depend on time, so the start time baked into the captured launches is immaterial
    if (nsteps == 0) return BOSSS_OK;
    cudaStream_t cs = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) rc = rk_step(h, T, dt, time, U_dev, work_dev, cs);
    cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(cs, &g) : cudaSuccess;
    if (!rc && e == cudaSuccess && e2 == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
    for (int i = 0; i < nsteps && !rc && e == cudaSuccess && e2 == cudaSuccess; ++i) e = cudaGraphLaunch(ge, st);
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("Runge-Kutta graph: ") + cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("Runge-Kutta capture: ") + cudaGetErrorString(e2));
    return BOSSS_OK;
}

int bosss_b200_rk_steps(bosss_handle* h, int32_t stages, const double* a, const double* b, const double* c, double dt, int32_t nsteps, double time, double* U) {
    if (!h || !U) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    int64_t nw = 0;
    int rc = bosss_b200_rk_work_size(h, stages, &nw);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(h->device));
    double *dU = nullptr, *dW = nullptr;
    cudaError_t e = cudaMalloc(&dU, sizeof(double) * h->ndom);
    if (e == cudaSuccess) e = cudaMalloc(&dW, sizeof(double) * nw);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dU, U, sizeof(double) * h->ndom, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) {
        cudaFree(dU);
        cudaFree(dW);
        return fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    }
    rc = bosss_b200_rk_steps_device(h, stages, a, b, c, dt, nsteps, time, dU, dW, 1, h->stream);
    if (!rc) {
        e = cudaMemcpyAsync(U, dU, sizeof(double) * h->ndom, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaFree(dU);
    cudaFree(dW);
    return rc;
}

}  // extern "C"
