// handle.h -- private definitions shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/bosss_b200.h"
#include "dg_kernel.cuh"
#include "dg_registry.h"

namespace bosss {
struct TcVolume;
}

struct bosss_handle {
    int device = 0;
    int precision = 0;                  // enum bosss_precision
    bosss::TcVolume* tcv = nullptr;     // split-precision volume tables (BOSSS_PRECISION_SPLIT_FP32)
    // boundary-state table of operators with prescribed outer states (CNS viscous terms)
    int64_t n_bnd_nodes = 0;
    long long* d_bnd_off = nullptr;
    double* d_bnd_state = nullptr;
    int* d_bnd_kind = nullptr;          // boundary-condition kinds (null: all prescribed states)
    bool bnd_table_needed = true;       // some node takes the table's state (kind 0)
    // face-once path (3D Euler residual and VJP): enabled flag and the face buffer
    bool faces_once = false;
    double* dFace = nullptr;
    cudaStream_t stream = nullptr;
    int phys = 0, D = 0, K = 0, Q = 0, variant = 0;
    bosss::EvalArgs base{};
    int64_t ndom = 0, ncod = 0;
    bosss::KernelEntry kern[3]{};
    int kern_variant[3]{};   // VARIANT_GENERIC / VARIANT_SLAB per mode
    bosss::KernelEntry kern_vol[3]{};   // face-once path: volume-only slab instances (launch null: none)
    bool check_nan = false;
    // device staging for the host-buffer entry points
    double* dU = nullptr;
    double* dV = nullptr;
    double* dOut = nullptr;
    double* dOut2 = nullptr;   // second output of the combined residual + VJP entry point
    int* dFlag = nullptr;
    // copy streams and chunk events of the pipelined host-buffer entry points
    cudaStream_t s_in = nullptr, s_out = nullptr;
    static constexpr int MAX_CHUNKS = 16;
    cudaEvent_t ev_in[MAX_CHUNKS]{}, ev_done[MAX_CHUNKS]{};
};

namespace bosss {
int fail(int code, const std::string& msg);
int run_mode(bosss_handle* h, int mode, double alpha, double beta, const double* U, const double* V, double* out,
             double time, cudaStream_t s);
int ensure_staging(bosss_handle* h);
}  // namespace bosss

#define CUDA_TRY(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return ::bosss::fail(BOSSS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
    } while (0)
