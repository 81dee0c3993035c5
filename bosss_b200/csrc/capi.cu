// capi.cu -- implementation of the C-ABI declared in include/bosss_b200.h.
//
// create() is the device-side counterpart of DifferentialOperator.GetEvaluatorEx
// (DifferentialOperator.cs:1013-1033): it checks the committed operator, maps each
// registered equation component to a device functor (no CPU fallback: an unknown
// component is an error, as the reference throws NotSupportedException for
// unsupported evaluator configurations), evaluates the quadrature-order function
// (QuadOrderFunc.cs) and picks the Gauss rule like RefElement.GetQuadratureRule
// (RefElement.cs:844-874), tabulates the 1D basis once and binds the kernel instance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bosss_b200.h"
#include "dg_kernel.cuh"
#include "dg_registry.h"
#include "bsr.h"
#include "handle.h"
#include "faces_euler.h"
#include "tc_volume.h"

namespace bosss {

std::map<KernelKey, KernelEntry>& kernel_registry() {
    static std::map<KernelKey, KernelEntry> r;
    return r;
}

static void ensure_registered() {
    static std::once_flag once;
    std::call_once(once, [] {
        register_scalar2();
        register_scalar3();
        register_scalar3_slab();
        register_euler2();
        register_euler3();
        register_cns();
    });
}

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}


// ------------------------------------------------------------------ host tables
// Gauss-Legendre rule with n nodes (Newton iteration on P_n in long double), ascending.
static void gauss_rule(int n, double* x, double* w) {
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double z = std::cos(PI * (i + 0.75L) / (n + 0.5L)), dp = 1.0L;
        for (int it = 0; it < 60; ++it) {
            long double p0 = 1.0L, p1 = z;
            for (int m = 1; m < n; ++m) {
                long double p2 = ((2 * m + 1) * z * p1 - m * p0) / (m + 1);
                p0 = p1;
                p1 = p2;
            }
            long double pn = (n == 1) ? z : p1, pm = (n == 1) ? 1.0L : p0;
            dp = n * (z * pn - pm) / (z * z - 1.0L);
            long double dz = pn / dp;
            z -= dz;
            if (std::fabs((double)dz) < 1e-19) {
                // recompute the derivative at the converged node
                p0 = 1.0L;
                p1 = z;
                for (int m = 1; m < n; ++m) {
                    long double p2 = ((2 * m + 1) * z * p1 - m * p0) / (m + 1);
                    p0 = p1;
                    p1 = p2;
                }
                pn = (n == 1) ? z : p1;
                pm = (n == 1) ? 1.0L : p0;
                dp = n * (z * pn - pm) / (z * z - 1.0L);
                break;
            }
        }
        x[n - 1 - i] = (double)z;
        w[n - 1 - i] = (double)(2.0L / ((1.0L - z * z) * dp * dp));
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// normalised Legendre L_a(x) = sqrt((2a+1)/2) P_a(x) and derivative, a = 0..K
static void legendre(int K, long double x, long double* L, long double* dL) {
    long double P[KMAX + 2], dP[KMAX + 2];
    P[0] = 1.0L;
    dP[0] = 0.0L;
    if (K >= 1) {
        P[1] = x;
        dP[1] = 1.0L;
    }
    for (int m = 1; m < K; ++m) {
        P[m + 1] = ((2 * m + 1) * x * P[m] - m * P[m - 1]) / (m + 1);
        dP[m + 1] = dP[m - 1] + (2 * m + 1) * P[m];
    }
    for (int a = 0; a <= K; ++a) {
        long double s = std::sqrt((2.0L * a + 1.0L) / 2.0L);
        L[a] = s * P[a];
        dL[a] = s * dP[a];
    }
}

static void build_tables(int K, int Q, Tables1D& t) {
    std::memset(&t, 0, sizeof(t));
    double x[QMAX], w[QMAX];
    gauss_rule(Q, x, w);
    for (int q = 0; q < Q; ++q) {
        long double L[KMAX + 1], dL[KMAX + 1];
        legendre(K, x[q], L, dL);
        for (int a = 0; a <= K; ++a) {
            t.A[q][a] = (double)L[a];
            t.dA[q][a] = (double)dL[a];
        }
        t.w[q] = w[q];
        t.xq[q] = x[q];
    }
    for (int s = 0; s < 2; ++s) {
        long double L[KMAX + 1], dL[KMAX + 1];
        legendre(K, s ? 1.0L : -1.0L, L, dL);
        for (int a = 0; a <= K; ++a) {
            t.e[s][a] = (double)L[a];
            t.de[s][a] = (double)dL[a];
        }
    }
}

// QuadOrderFunc.cs
static int quad_order(const bosss_op_desc& op) {
    int maxDom = 0, maxCod = 0;
    for (int i = 0; i < op.n_domain; ++i) maxDom = std::max(maxDom, op.domain_degree[i]);
    for (int i = 0; i < op.n_codomain; ++i) maxCod = std::max(maxCod, op.codomain_degree[i]);
    switch (op.quad_kind) {
        case BOSSS_QUAD_FIXED: return op.quad_param;
        case BOSSS_QUAD_LINEAR: return maxDom + maxCod;
        case BOSSS_QUAD_NONLINEAR: return maxDom * op.quad_param + maxCod;
        case BOSSS_QUAD_MAXDEG_TIMES_TWO: return 2 * std::max(maxDom, maxCod);
        case BOSSS_QUAD_SUM_OF_MAX_DEGREES: {
            int o = maxDom * op.quad_param + maxCod;
            return (o % 2) ? o + 1 : o;
        }
        default: return -1;
    }
}

}  // namespace bosss

using namespace bosss;

namespace bosss {

static int classify(const bosss_op_desc& op, int D, int& phys, PhysParams& ph) {
    std::memset(&ph, 0, sizeof(ph));
    if (op.n_components < 1 || op.n_components > BOSSS_MAX_COMPONENTS)
        return fail(BOSSS_ERR_BAD_ARG, "operator has no equation components");
    bool euler = false, cns = false;
    for (int c = 0; c < op.n_components; ++c) {
        int t = op.components[c].type;
        if (t == BOSSS_COMP_HLLC_DENSITY_FLUX || t == BOSSS_COMP_HLLC_MOMENTUM_FLUX || t == BOSSS_COMP_HLLC_ENERGY_FLUX)
            euler = true;
        else if (t == BOSSS_COMP_CNS_SIPG_DENSITY_FLUX || t == BOSSS_COMP_CNS_SIPG_MOMENTUM_FLUX ||
                 t == BOSSS_COMP_CNS_SIPG_ENERGY_FLUX)
            cns = true;
        else if (t != BOSSS_COMP_SCALAR_TRANSPORT_FLUX && t != BOSSS_COMP_SIP_LAPLACE && t != BOSSS_COMP_CONSTANT_SOURCE)
            return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT,
                        "equation component type " + std::to_string(t) + " has no device functor");
    }
    if (cns) {
        // the complete OptimizedSIPG set: density, D momentum components, energy, one material
        const int NV = D + 2;
        if (euler) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "CNS viscous terms cannot be mixed with HLLC fluxes");
        if (op.n_domain != NV || op.n_codomain != NV)
            return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "CNS viscous operator needs D+2 domain and codomain variables");
        std::vector<int> seen(NV, 0);
        for (int c = 0; c < op.n_components; ++c) {
            const auto& cp = op.components[c];
            if (cp.type != BOSSS_COMP_CNS_SIPG_DENSITY_FLUX && cp.type != BOSSS_COMP_CNS_SIPG_MOMENTUM_FLUX &&
                cp.type != BOSSS_COMP_CNS_SIPG_ENERGY_FLUX)
                return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "CNS viscous terms cannot be mixed with other components");
            if (cp.n_args != NV) return fail(BOSSS_ERR_BAD_ARG, "CNS viscous flux needs D+2 arguments");
            for (int a = 0; a < NV; ++a)
                if (cp.args[a] != a)
                    return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "CNS arguments must be (rho, m_0..m_{D-1}, rhoE)");
            if (cp.type == BOSSS_COMP_CNS_SIPG_MOMENTUM_FLUX && (cp.params[8] < 0 || cp.params[8] >= D))
                return fail(BOSSS_ERR_BAD_ARG, "CNS momentum component out of range");
            const int cod = (cp.type == BOSSS_COMP_CNS_SIPG_DENSITY_FLUX) ? 0
                            : (cp.type == BOSSS_COMP_CNS_SIPG_ENERGY_FLUX) ? D + 1
                                                                          : (int)cp.params[8] + 1;
            if (cp.codomain != cod)
                return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "CNS flux registered on an unexpected codomain variable");
            if (seen[cod]++) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "duplicate CNS viscous flux");
            for (int i = 0; i < 8; ++i)
                if (cp.params[i] != op.components[0].params[i])
                    return fail(BOSSS_ERR_BAD_ARG, "CNS viscous fluxes with different material parameters");
        }
        for (int v = 0; v < NV; ++v)
            if (!seen[v]) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "incomplete CNS viscous flux set");
        const double* pp = op.components[0].params;
        if (!(pp[0] > 1.0) || !(pp[1] > 0.0) || !(pp[2] > 0.0) || !(pp[3] > 0.0))
            return fail(BOSSS_ERR_BAD_ARG, "bad gamma / Mach / Reynolds / Prandtl");
        if (pp[5] != 0.0 && pp[5] != 1.0) return fail(BOSSS_ERR_BAD_ARG, "viscosity law: 0 (constant) or 1 (Sutherland)");
        ph.gamma = pp[0];
        ph.mach = pp[1];
        ph.re = pp[2];
        ph.pr = pp[3];
        ph.visc_ratio = pp[4];
        ph.visc_law = (int)pp[5];
        ph.suth = pp[6];
        ph.pen = pp[7];   // times p^2 in create()
        phys = PHYS_CNS;
        return 0;
    }
    if (euler) {
        const int NV = D + 2;
        if (op.n_domain != NV || op.n_codomain != NV)
            return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "HLLC operator needs D+2 domain and codomain variables");
        std::vector<int> seen(NV, 0);
        double gamma = 0, mach = 0;
        for (int c = 0; c < op.n_components; ++c) {
            const auto& cp = op.components[c];
            if (cp.type != BOSSS_COMP_HLLC_DENSITY_FLUX && cp.type != BOSSS_COMP_HLLC_MOMENTUM_FLUX &&
                cp.type != BOSSS_COMP_HLLC_ENERGY_FLUX)
                return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "HLLC fluxes cannot be mixed with other components");
            if (cp.n_args != NV) return fail(BOSSS_ERR_BAD_ARG, "HLLC flux needs D+2 arguments");
            for (int a = 0; a < NV; ++a)
                if (cp.args[a] != a)
                    return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "HLLC arguments must be (rho, m_0..m_{D-1}, rhoE)");
            int cod = (cp.type == BOSSS_COMP_HLLC_DENSITY_FLUX) ? 0
                      : (cp.type == BOSSS_COMP_HLLC_ENERGY_FLUX) ? D + 1
                                                                 : (int)cp.params[2] + 1;
            if (cp.type == BOSSS_COMP_HLLC_MOMENTUM_FLUX && (cp.params[2] < 0 || cp.params[2] >= D))
                return fail(BOSSS_ERR_BAD_ARG, "HLLC momentum component out of range");
            if (cp.codomain != cod)
                return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "HLLC flux registered on an unexpected codomain variable");
            if (seen[cod]++) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "duplicate HLLC flux");
            if (c == 0) {
                gamma = cp.params[0];
                mach = cp.params[1];
            } else if (gamma != cp.params[0] || mach != cp.params[1]) {
                return fail(BOSSS_ERR_BAD_ARG, "HLLC fluxes with different material parameters");
            }
        }
        for (int v = 0; v < NV; ++v)
            if (!seen[v]) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "incomplete HLLC flux set");
        if (!(gamma > 1.0) || !(mach > 0.0)) return fail(BOSSS_ERR_BAD_ARG, "bad gamma/Mach");
        ph.gamma = gamma;
        ph.mach = mach;
        ph.ims = 1.0 / (gamma * mach * mach);
        ph.imach = 1.0 / mach;
        phys = PHYS_EULER;
        return 0;
    }
    if (op.n_domain != 1 || op.n_codomain != 1)
        return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "scalar components need one domain and one codomain variable");
    int ntr = 0, nsip = 0, nsrc = 0;
    for (int c = 0; c < op.n_components; ++c) {
        const auto& cp = op.components[c];
        if (cp.codomain != 0) return fail(BOSSS_ERR_BAD_ARG, "bad codomain index");
        if (cp.type != BOSSS_COMP_CONSTANT_SOURCE && (cp.n_args != 1 || cp.args[0] != 0))
            return fail(BOSSS_ERR_BAD_ARG, "scalar component must take the domain variable as its argument");
        if (cp.type == BOSSS_COMP_SCALAR_TRANSPORT_FLUX) {
            ++ntr;
            ph.has_transport = 1;
            for (int d = 0; d < 3; ++d) ph.vel[d] = d < D ? cp.params[d] : 0.0;
        } else if (cp.type == BOSSS_COMP_SIP_LAPLACE) {
            ++nsip;
            ph.has_sip = 1;
            ph.pen = cp.params[0];   // multiplied by the degree factor in create()
            ph.nu0 = cp.params[1];
            ph.nu2 = cp.params[2];
            ph.dirichlet = (cp.params[3] == 0.0) ? 1 : 0;
            ph.g0 = cp.params[4];
            for (int d = 0; d < 3; ++d) {
                ph.g1[d] = cp.params[5 + d];
                ph.g2[d] = cp.params[8 + d];
            }
        } else {
            ++nsrc;
            ph.has_source = 1;
            ph.src = cp.params[0];
        }
    }
    if (ntr > 1 || nsip > 1 || nsrc > 1)
        return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "at most one transport, one SIP and one source component");
    phys = (nsip || nsrc) ? PHYS_SIP : PHYS_TRANSPORT;
    return 0;
}

int ensure_staging(bosss_handle* h) {
    if (h->dU) return 0;
    const int64_t n1 = std::max(h->ndom, h->ncod);
    CUDA_TRY(cudaMalloc(&h->dU, sizeof(double) * std::max<int64_t>(h->ndom, 1)));
    CUDA_TRY(cudaMalloc(&h->dV, sizeof(double) * std::max<int64_t>(n1, 1)));
    CUDA_TRY(cudaMalloc(&h->dOut, sizeof(double) * std::max<int64_t>(n1, 1)));
    return 0;
}

__global__ void nan_scan_kernel(const double* x, long long n, int* flag) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!isfinite(x[i])) {
            atomicExch(flag, 1);
            return;
        }
}

// One evaluation launch of `mode` on the cells [a.cbeg, a.cend). A split-precision residual
// (BOSSS_PRECISION_SPLIT_FP32, whole grids only) runs the tensor-core volume kernel
// (out = beta*out + alpha*volume terms), then the slab kernel adds the face terms.
// A face-once handle (3D Euler) evaluates residual and VJP as the slab kernel's volume pass
// (or the tensor-core volume kernel) followed by the face kernels of faces_euler.cu.
static int launch_eval(bosss_handle* h, int mode, EvalArgs a, cudaStream_t s) {
    if (h->n_bnd_nodes > 0 && !a.bnd_state && h->bnd_table_needed)
        return fail(BOSSS_ERR_BAD_ARG, "the operator's boundary terms need the boundary-state table "
                                       "(bosss_b200_set_boundary_state)");
    const bool split = mode == MODE_RES && h->precision == BOSSS_PRECISION_SPLIT_FP32;
    const bool once = h->faces_once && (mode == MODE_RES || mode == MODE_VJP);
    if (split) {
        if (a.cbeg != 0 || a.cend != h->base.g.J)
            return fail(BOSSS_ERR_BAD_ARG, "split-precision residuals evaluate whole grids only");
        int rc = tc_volume_launch(h, a.U, a.out, a.alpha, a.beta, s);
        if (rc) return rc;
        if (once) return faces_once_launch(h, mode, a, s);
        a.faces_only = 1;
        a.beta = 1.0;
    } else if (once) {
        EvalArgs v = a;
        v.volume_only = 1;
        if (h->kern_vol[mode].launch) CUDA_TRY(h->kern_vol[mode].launch(v, s));
        else CUDA_TRY(h->kern[mode].launch(v, s));
        return faces_once_launch(h, mode, a, s);
    }
    CUDA_TRY(h->kern[mode].launch(a, s));
    return 0;
}

int run_mode(bosss_handle* h, int mode, double alpha, double beta, const double* U, const double* V,
                    double* out, double time, cudaStream_t s) {
    EvalArgs a = h->base;
    a.U = U;
    a.V = V;
    a.out = out;
    a.alpha = alpha;
    a.beta = beta;
    a.time = time;
    CUDA_TRY(cudaSetDevice(h->device));
    if ((a.vol_flag || a.face_flag) && (h->faces_once || h->precision != BOSSS_PRECISION_FP64))
        return fail(BOSSS_ERR_BAD_ARG, "species masks: plain FP64 generic or slab kernels only");
    if (h->base.g.J > 0) return launch_eval(h, mode, a, s);
    return 0;
}

static int check_nan(bosss_handle* h, const double* out, int64_t n, cudaStream_t s) {
    if (!h->check_nan) return 0;
    if (!h->dFlag) CUDA_TRY(cudaMalloc(&h->dFlag, sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(h->dFlag, 0, sizeof(int), s));
    nan_scan_kernel<<<592, 256, 0, s>>>(out, (long long)n, h->dFlag);
    CUDA_TRY(cudaGetLastError());
    int flag = 0;
    CUDA_TRY(cudaMemcpyAsync(&flag, h->dFlag, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (flag) return fail(BOSSS_ERR_NAN, "NaN or Inf in the operator output");
    return 0;
}

}  // namespace bosss

extern "C" {

int bosss_b200_version(int32_t* major, int32_t* minor, int32_t* patch) {
    if (major) *major = BOSSS_B200_VERSION_MAJOR;
    if (minor) *minor = BOSSS_B200_VERSION_MINOR;
    if (patch) *patch = BOSSS_B200_VERSION_PATCH;
    return BOSSS_OK;
}

int bosss_b200_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return BOSSS_ERR_BAD_ARG;
    std::strncpy(buf, g_last_error.c_str(), len - 1);
    buf[len - 1] = 0;
    return BOSSS_OK;
}

int bosss_b200_device_count(int32_t* count) {
    if (!count) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    *count = (e == cudaSuccess) ? n : 0;
    if (e != cudaSuccess) cudaGetLastError();
    return BOSSS_OK;
}

int bosss_b200_create(const bosss_op_desc* op, const bosss_grid_desc* grid, const bosss_options* opt,
                      bosss_handle** out) {
    if (!op || !grid || !out) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    const int D = grid->dim;
    if (D != 2 && D != 3) return fail(BOSSS_ERR_BAD_ARG, "grid dimension must be 2 or 3");
    long long J = 1;
    for (int d = 0; d < D; ++d) {
        if (grid->n[d] < 1) return fail(BOSSS_ERR_BAD_ARG, "grid needs at least one cell per direction");
        if (!(grid->hi[d] > grid->lo[d])) return fail(BOSSS_ERR_BAD_ARG, "grid box has non-positive extent");
        J *= grid->n[d];
    }
    if (J > 2000000000LL) return fail(BOSSS_ERR_BAD_ARG, "too many cells");
    if (op->n_domain < 1 || op->n_domain > BOSSS_MAX_VARS || op->n_codomain < 1 || op->n_codomain > BOSSS_MAX_VARS)
        return fail(BOSSS_ERR_BAD_ARG, "bad number of variables");
    const int K = op->domain_degree[0];
    for (int i = 0; i < op->n_domain; ++i)
        if (op->domain_degree[i] != K) return fail(BOSSS_ERR_BAD_ARG, "device path needs one DG degree for all fields");
    for (int i = 0; i < op->n_codomain; ++i)
        if (op->codomain_degree[i] != K) return fail(BOSSS_ERR_BAD_ARG, "device path needs one DG degree for all fields");
    if (K < 0 || K > KMAX) return fail(BOSSS_ERR_BAD_ARG, "DG degree outside 0..4");
    int phys = 0;
    PhysParams ph;
    int rc = classify(*op, D, phys, ph);
    if (rc) return rc;
    // part of a partitioned grid: global extent, offset and periodicity per direction
    bool part = false;
    for (int d = 0; d < D; ++d) part = part || grid->global_n[d] != 0;
    int gper[3] = {0, 0, 0};
    for (int d = 0; d < D; ++d) {
        gper[d] = part ? (grid->global_periodic[d] ? 1 : 0) : (grid->periodic[d] ? 1 : 0);
        if (part) {
            if (grid->global_n[d] < grid->n[d]) return fail(BOSSS_ERR_BAD_ARG, "part larger than the global grid");
            if (grid->periodic[d] && (!gper[d] || grid->n[d] != grid->global_n[d]))
                return fail(BOSSS_ERR_BAD_ARG, "a part is periodic only in directions it spans completely");
        }
    }
    // HLLC on a grid with boundary faces: the outer states come from the boundary-state table
    // (OptimizedHLLCFlux.BorderEdgeFlux); the generic kernel reads it
    bool euler_bounded = false;
    if (phys == PHYS_EULER)
        for (int d = 0; d < D; ++d) euler_bounded = euler_bounded || !gper[d];
    if (phys == PHYS_SIP && ph.has_sip && K < 1)
        return fail(BOSSS_ERR_BAD_ARG, "SIP needs DG degree >= 1 (IsValidDomainDegreeCombination)");
    const int order = quad_order(*op);
    if (order < 0) return fail(BOSSS_ERR_BAD_ARG, "bad quadrature-order function");
    const int Q = std::max(1, (order + 2) / 2);   // smallest Gauss rule with 2Q-1 >= order
    ensure_registered();
    auto& reg = kernel_registry();
    const int prec = opt ? opt->precision : BOSSS_PRECISION_FP64;
    if (prec != BOSSS_PRECISION_FP64 && prec != BOSSS_PRECISION_SPLIT_FP32)
        return fail(BOSSS_ERR_BAD_ARG, "unknown precision");
    const int want = opt ? opt->kernel : 0;
    if (want < 0 || want > 3) return fail(BOSSS_ERR_BAD_ARG, "bad kernel selector");
    bool have_slab = true, have_generic = true;
    for (int m = 0; m < 3; ++m) {
        have_slab = have_slab && !euler_bounded && reg.count(KernelKey(phys, D, K, Q, m, VARIANT_SLAB));
        have_generic = have_generic && reg.count(KernelKey(phys, D, K, Q, m, VARIANT_GENERIC));
    }
    if ((want == 2 || want == 3) && !have_slab) return fail(BOSSS_ERR_BAD_ARG, "no slab kernel for this operator");
    // automatic choice per mode, measured on B200 (16^3-48^3 grids): the slab kernel for 3D
    // systems (Euler, 3-6x); for the scalar family (two threads per node row) the slab residual
    // at every rule (1.1-1.7x faster) and the slab JVP / VJP up to 5 nodes per direction
    // (1.2-1.6x faster; with 7 or 9 nodes the generic tile is 1.4-1.5x faster)
    int mode_variant[3];
    for (int m = 0; m < 3; ++m) {
        const bool slab_pays = phys == PHYS_EULER || m == MODE_RES || Q <= 5;
        mode_variant[m] = (want == 2 || want == 3 || (want == 0 && have_slab && slab_pays)) ? VARIANT_SLAB
                                                                                           : VARIANT_GENERIC;
    }
    if (prec == BOSSS_PRECISION_SPLIT_FP32) {
        // the face terms of a split-precision residual come from the slab kernel's faces-only pass
        if (!have_slab || want == 1)
            return fail(BOSSS_ERR_BAD_ARG, "split precision needs the slab kernel for the face terms");
        mode_variant[MODE_RES] = VARIANT_SLAB;
    }
    bool need_generic = false;
    for (int m = 0; m < 3; ++m) need_generic = need_generic || mode_variant[m] == VARIANT_GENERIC;
    if (need_generic && !have_generic)
        return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "no device kernel for degree " + std::to_string(K) +
                                                         " with " + std::to_string(Q) + " Gauss nodes");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(BOSSS_ERR_NO_DEVICE, "no CUDA device available");
    }
    const int dev = opt ? opt->device : 0;
    if (dev < 0 || dev >= ndev) return fail(BOSSS_ERR_BAD_ARG, "bad device ordinal");

    bosss_handle* h = new bosss_handle();
    h->device = dev;
    h->phys = phys;
    h->D = D;
    h->K = K;
    h->Q = Q;
    h->check_nan = opt && opt->check_nan;
    build_tables(K, Q, h->base.tab);
    GridConst& g = h->base.g;
    std::memset(&g, 0, sizeof(g));
    g.D = D;
    g.J = (int)J;
    for (int d = 0; d < 3; ++d) {
        g.n[d] = d < D ? grid->n[d] : 1;
        g.periodic[d] = d < D ? (grid->periodic[d] ? 1 : 0) : 0;
        g.lo[d] = d < D ? grid->lo[d] : 0.0;
        // a part's box is the global box: the cell width is the global one
        g.h[d] = d < D ? (grid->hi[d] - grid->lo[d]) / (part ? grid->global_n[d] : grid->n[d]) : 1.0;
        g.twoh[d] = 2.0 / g.h[d];
        g.gn[d] = (part && d < D) ? grid->global_n[d] : g.n[d];
        g.goff[d] = (part && d < D) ? grid->global_offset[d] : 0;
        g.gper[d] = d < D ? gper[d] : 0;
    }
    h->base.cbeg = 0;
    h->base.cend = J;
    // 2D: GlobalID = ix*nY + iy (Grid2D.cs:182) is the generator order
    if (grid->cell_order == BOSSS_CELLS_GLOBALID && D == 3) {
        g.stride[0] = 1;
        g.stride[1] = g.n[0];
        g.stride[2] = (long long)g.n[0] * g.n[1];
    } else {
        if (D == 2) {
            g.stride[0] = g.n[1];
            g.stride[1] = 1;
            g.stride[2] = 0;
        } else {
            g.stride[0] = (long long)g.n[1] * g.n[2];
            g.stride[1] = g.n[2];
            g.stride[2] = 1;
        }
    }
    g.detJ = 1.0;
    for (int d = 0; d < D; ++d) g.detJ *= 0.5 * g.h[d];
    g.scaling = 1.0 / std::sqrt(g.detJ);
    for (int d = 0; d < D; ++d) {
        double sg = 1.0;
        for (int d2 = 0; d2 < D; ++d2)
            if (d2 != d) sg *= 0.5 * g.h[d2];
        g.faceSG[d] = sg;
    }
    if (phys == PHYS_CNS) ph.pen *= (double)K * (double)K;   // SIPGPenaltyScaling * p^2
    if (ph.has_sip) {
        // ipLaplace.cs CoefficientUpdate: max(triangle formula, (p+1)^2)
        const double p = K;
        ph.pen *= std::max((p + 1.0) * (p + D) / D, (p + 1.0) * (p + 1.0));
    }
    h->base.ph = ph;
    const int NV = (phys == PHYS_EULER || phys == PHYS_CNS) ? D + 2 : 1;
    h->ndom = (int64_t)J * NV * np_of(D, K);
    h->ncod = h->ndom;
    h->variant = VARIANT_GENERIC;   // generic unless some mode runs on the slab kernel
    for (int m = 0; m < 3; ++m) {
        h->kern[m] = reg[KernelKey(phys, D, K, Q, m, mode_variant[m])];
        h->kern_variant[m] = mode_variant[m];
        if (mode_variant[m] == VARIANT_SLAB) h->variant = VARIANT_SLAB;
    }
    cudaError_t e = cudaSetDevice(dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return fail(BOSSS_ERR_CUDA, std::string("stream creation: ") + cudaGetErrorString(e));
    }
    // face-once face terms (3D Euler): on request only (kernel 3) -- measured on B200 at Euler
    // 32^3 k=3 slower than the slab kernel's two-sided faces (residual 0.51 vs 0.31 ms, VJP 0.83
    // vs 0.60 ms); the face buffer is allocated here, not at the first evaluation, so that
    // evaluations can be captured in CUDA graphs
    if (want == 3 && faces_once_supported(h) && h->variant == VARIANT_SLAB) {
        h->faces_once = true;
        if (faces_once_alloc(h) != BOSSS_OK) {
            const std::string msg = g_last_error;
            bosss_b200_destroy(h);
            return fail(BOSSS_ERR_CUDA, msg);
        }
    }
    if (h->faces_once)
        for (int m : {MODE_RES, MODE_VJP}) {
            auto it = reg.find(KernelKey(phys, D, K, Q, m, VARIANT_SLAB_VOL));
            if (it != reg.end()) h->kern_vol[m] = it->second;
        }
    if (want == 3 && !h->faces_once) {
        bosss_b200_destroy(h);
        return fail(BOSSS_ERR_BAD_ARG, "the face-once path needs 3D Euler on a whole periodic grid");
    }
    if (phys == PHYS_CNS || euler_bounded) {
        // boundary faces numbered cell by cell, direction, side; Q^(D-1) nodes each
        std::vector<long long> off((size_t)J * 2 * D, -1);
        long long nb = 0;
        const long long QF = (D == 3) ? (long long)Q * Q : Q;
        for (long long j = 0; j < J; ++j) {
            int ijk[3];
            for (int d = 0; d < 3; ++d) ijk[d] = d < D ? (int)((j / g.stride[d]) % g.n[d]) : 0;
            for (int d = 0; d < D; ++d)
                for (int sd = 0; sd < 2; ++sd) {
                    const int gi = ijk[d] + g.goff[d];
                    const bool bnd = !g.gper[d] && (sd == 0 ? gi == 0 : gi == g.gn[d] - 1);
                    if (bnd) {
                        off[(size_t)j * 2 * D + 2 * d + sd] = nb;
                        nb += QF;
                    }
                }
        }
        h->n_bnd_nodes = nb;
        if (nb > 0) {
            e = cudaMalloc(&h->d_bnd_off, sizeof(long long) * off.size());
            if (e == cudaSuccess) e = cudaMemcpy(h->d_bnd_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                bosss_b200_destroy(h);
                return fail(BOSSS_ERR_CUDA, std::string("boundary table: ") + cudaGetErrorString(e));
            }
        }
    }
    if (prec == BOSSS_PRECISION_SPLIT_FP32) {
        h->precision = prec;
        if (part) {
            bosss_b200_destroy(h);
            return fail(BOSSS_ERR_BAD_ARG, "split precision evaluates whole grids (no parts of partitioned grids)");
        }
        const int rc = tc_volume_setup(h);
        if (rc) {
            const std::string msg = g_last_error;
            bosss_b200_destroy(h);
            return fail(rc, msg);
        }
    }
    *out = h;
    return BOSSS_OK;
}

int bosss_b200_destroy(bosss_handle* h) {
    if (!h) return BOSSS_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->dU);
    cudaFree(h->dV);
    cudaFree(h->dOut);
    cudaFree(h->dFlag);
    cudaFree(h->dOut2);
    for (int c = 0; c < bosss_handle::MAX_CHUNKS; ++c) {
        if (h->ev_in[c]) cudaEventDestroy(h->ev_in[c]);
        if (h->ev_done[c]) cudaEventDestroy(h->ev_done[c]);
    }
    if (h->s_in) cudaStreamDestroy(h->s_in);
    if (h->s_out) cudaStreamDestroy(h->s_out);
    if (h->stream) cudaStreamDestroy(h->stream);
    cudaFree(h->d_bnd_off);
    cudaFree(h->d_bnd_state);
    cudaFree(h->d_bnd_kind);
    cudaFree(h->dFace);
    tc_volume_destroy(h);
    delete h;
    return BOSSS_OK;
}

int bosss_b200_boundary_nodes(const bosss_handle* h, int64_t* n_nodes, double* xyz) {
    if (!h || !n_nodes) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    *n_nodes = h->n_bnd_nodes;
    if (!xyz || h->n_bnd_nodes == 0) return BOSSS_OK;
    const GridConst& g = h->base.g;
    const Tables1D& T = h->base.tab;
    const int D = h->D, Q = h->Q, QF = (D == 3) ? Q * Q : Q;
    long long k = 0;
    for (long long j = 0; j < g.J; ++j) {
        int ijk[3];
        for (int d = 0; d < 3; ++d) ijk[d] = d < D ? (int)((j / g.stride[d]) % g.n[d]) : 0;
        for (int d = 0; d < D; ++d) {
            const int t1 = (d == 0) ? 1 : 0, t2 = (d == 2) ? 1 : 2;
            for (int sd = 0; sd < 2; ++sd) {
                const int gi = ijk[d] + g.goff[d];
                if (g.gper[d] || !(sd == 0 ? gi == 0 : gi == g.gn[d] - 1)) continue;
                for (int qf = 0; qf < QF; ++qf) {
                    const int q1 = qf % Q, q2 = qf / Q;
                    double x[3];
                    for (int dd = 0; dd < D; ++dd) x[dd] = g.lo[dd] + (ijk[dd] + g.goff[dd] + 0.5) * g.h[dd];
                    x[d] += (sd ? 0.5 : -0.5) * g.h[d];
                    x[t1] += 0.5 * g.h[t1] * T.xq[q1];
                    if (D == 3) x[t2] += 0.5 * g.h[t2] * T.xq[q2];
                    for (int dd = 0; dd < D; ++dd) xyz[k * D + dd] = x[dd];
                    ++k;
                }
            }
        }
    }
    return BOSSS_OK;
}

int bosss_b200_set_boundary_state(bosss_handle* h, const double* state) {
    if (!h || !state) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (h->n_bnd_nodes == 0) return fail(BOSSS_ERR_BAD_ARG, "the operator takes no boundary-state table");
    const int NV = (int)(h->ndom / h->base.g.J / np_of(h->D, h->K));
    const size_t n = (size_t)h->n_bnd_nodes * NV;
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(state[i])) return fail(BOSSS_ERR_BAD_ARG, "non-finite boundary state");
    CUDA_TRY(cudaSetDevice(h->device));
    if (!h->d_bnd_state) CUDA_TRY(cudaMalloc(&h->d_bnd_state, sizeof(double) * n));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaMemcpy(h->d_bnd_state, state, sizeof(double) * n, cudaMemcpyHostToDevice));
    h->base.bnd_off = h->d_bnd_off;
    h->base.bnd_state = h->d_bnd_state;
    return BOSSS_OK;
}

int bosss_b200_set_boundary_kinds(bosss_handle* h, const int32_t* kinds) {
    if (!h || !kinds) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (h->n_bnd_nodes == 0) return fail(BOSSS_ERR_BAD_ARG, "the operator takes no boundary-state table");
    bool any0 = false;
    for (int64_t i = 0; i < h->n_bnd_nodes; ++i) {
        if (kinds[i] < 0 || kinds[i] > 2) return fail(BOSSS_ERR_BAD_ARG, "boundary kind: 0, 1 or 2");
        if (kinds[i] != 0 && h->phys != PHYS_EULER)
            return fail(BOSSS_ERR_BAD_ARG, "boundary kinds 1 and 2 (outlet, slip wall): HLLC fluxes only");
        any0 = any0 || kinds[i] == 0;
    }
    CUDA_TRY(cudaSetDevice(h->device));
    if (!h->d_bnd_kind) CUDA_TRY(cudaMalloc(&h->d_bnd_kind, sizeof(int) * (size_t)h->n_bnd_nodes));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaMemcpy(h->d_bnd_kind, kinds, sizeof(int) * (size_t)h->n_bnd_nodes, cudaMemcpyHostToDevice));
    h->base.bnd_off = h->d_bnd_off;
    h->base.bnd_kind = h->d_bnd_kind;
    h->bnd_table_needed = any0;
    return BOSSS_OK;
}

int bosss_b200_get_sizes(const bosss_handle* h, int64_t* n_domain_dofs, int64_t* n_codomain_dofs,
                         int32_t* quad_nodes_1d) {
    if (!h) return fail(BOSSS_ERR_BAD_ARG, "null handle");
    if (n_domain_dofs) *n_domain_dofs = h->ndom;
    if (n_codomain_dofs) *n_codomain_dofs = h->ncod;
    if (quad_nodes_1d) *quad_nodes_1d = h->Q;
    return BOSSS_OK;
}

int bosss_b200_kernel_info(const bosss_handle* h, int32_t mode, int32_t* kernel, int32_t* launches) {
    if (!h) return fail(BOSSS_ERR_BAD_ARG, "null handle");
    if (mode < MODE_RES || mode > MODE_VJP) return fail(BOSSS_ERR_BAD_ARG, "bad mode");
    const bool split = mode == MODE_RES && h->precision == BOSSS_PRECISION_SPLIT_FP32;
    const bool once = h->faces_once && (mode == MODE_RES || mode == MODE_VJP);
    const bool slab = h->kern_variant[mode] == VARIANT_SLAB;
    int k = slab ? 2 : 1, n = 1;
    if (split) {
        k = 4;
        n = once ? 3 : 2;
    } else if (once) {
        k = 3;
        n = 3;
    }
    if (kernel) *kernel = k;
    if (launches) *launches = n;
    return BOSSS_OK;
}

int bosss_b200_evaluate_device(bosss_handle* h, double alpha, double beta, const double* U_dev, double* out_dev,
                               double time, void* stream) {
    if (!h || !U_dev || !out_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    int rc = run_mode(h, MODE_RES, alpha, beta, U_dev, nullptr, out_dev, time, s);
    if (rc) return rc;
    return check_nan(h, out_dev, h->ncod, s);
}

int bosss_b200_apply_device(bosss_handle* h, int32_t mode, double alpha, double beta, const double* U_dev,
                            const double* V_dev, double* out_dev, double time, int64_t cell_begin, int64_t cell_end,
                            void* stream) {
    if (!h || !U_dev || !out_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (mode < MODE_RES || mode > MODE_VJP) return fail(BOSSS_ERR_BAD_ARG, "bad mode");
    if (mode != MODE_RES && !V_dev) return fail(BOSSS_ERR_BAD_ARG, "JVP / VJP need the second vector");
    if (cell_begin < 0 || cell_end < cell_begin || cell_end > h->base.g.J)
        return fail(BOSSS_ERR_BAD_ARG, "cell range outside the grid");
    if (cell_end == cell_begin) return BOSSS_OK;
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    EvalArgs a = h->base;
    a.U = U_dev;
    a.V = V_dev;
    a.out = out_dev;
    a.alpha = alpha;
    a.beta = beta;
    a.time = time;
    a.cbeg = cell_begin;
    a.cend = cell_end;
    CUDA_TRY(cudaSetDevice(h->device));
    return launch_eval(h, mode, a, s);
}

// Host-buffer evaluation pipelined over chunks of planes of the slowest-varying grid direction
// (the cells of a plane are contiguous in both cell orders): the inputs stream in on one copy
// stream, each chunk's cells are evaluated on the handle's stream as soon as its planes and the
// first plane of the next chunk have arrived (the face neighbours; the last plane comes first
// when that direction is periodic), and each chunk's outputs stream out on a second copy stream
// while later chunks are still computing. Small problems, and the opt-in NaN check, run as one
// chunk. Returns after the last output has reached the host. 8 chunks measured best on B200
// (Euler 32^3 k=3: 4 or 16 chunks, or a second compute stream for the VJP, were slower).
struct HostJob {
    int mode;
    double alpha, beta;
    double* Y;     // host output
    double* dY;    // device staging of the output
};

static int host_pipelined(bosss_handle* h, const HostJob* jobs, int njobs, const double* U, const double* X,
                          double time) {
    int rc = ensure_staging(h);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(h->device));
    const GridConst& g = h->base.g;
    const long long J = g.J;
    const int sd = (g.stride[0] >= g.stride[g.D - 1]) ? 0 : g.D - 1;   // slowest direction
    const long long planes = g.n[sd], pc = J / planes;                 // cells per plane
    const long long nU = h->ndom / J;                                  // DOFs per cell
    long long nX = 0;
    for (int k = 0; k < njobs; ++k)
        if (jobs[k].mode != MODE_RES) nX = (jobs[k].mode == MODE_JVP) ? h->ndom / J : h->ncod / J;
    auto nY = [&](const HostJob& jb) { return (jb.mode == MODE_VJP ? h->ndom : h->ncod) / J; };
    auto y_in = [&](const HostJob& jb) { return jb.mode == MODE_RES && jb.beta != 0.0; };
    size_t bytes = sizeof(double) * (size_t)J * (nU + (X ? nX : 0));
    for (int k = 0; k < njobs; ++k) bytes += sizeof(double) * (size_t)J * nY(jobs[k]);
    int nch = (int)std::min<long long>(bosss_handle::MAX_CHUNKS / 2, planes / 2);
    if (bytes < (size_t)16 << 20 || h->check_nan) nch = 1;
    for (int k = 0; k < njobs; ++k)   // split-precision residuals evaluate the whole grid at once
        if (jobs[k].mode == MODE_RES && h->precision == BOSSS_PRECISION_SPLIT_FP32) nch = 1;
    if (nch < 1) nch = 1;
    if (!h->s_in) CUDA_TRY(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking));
    if (!h->s_out) CUDA_TRY(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
    for (int c = 0; c < nch; ++c) {
        if (!h->ev_in[c]) CUDA_TRY(cudaEventCreateWithFlags(&h->ev_in[c], cudaEventDisableTiming));
        if (!h->ev_done[c]) CUDA_TRY(cudaEventCreateWithFlags(&h->ev_done[c], cudaEventDisableTiming));
    }
    cudaStream_t s = h->stream, si = h->s_in, so = h->s_out;
    auto first_plane = [&](int c) { return (long long)c * planes / nch; };
    auto copy_in = [&](long long p0, long long p1) -> cudaError_t {
        const long long c0 = p0 * pc, n = (p1 - p0) * pc;
        cudaError_t e = cudaMemcpyAsync(h->dU + c0 * nU, U + c0 * nU, sizeof(double) * n * nU, cudaMemcpyHostToDevice, si);
        if (e == cudaSuccess && X)
            e = cudaMemcpyAsync(h->dV + c0 * nX, X + c0 * nX, sizeof(double) * n * nX, cudaMemcpyHostToDevice, si);
        for (int k = 0; k < njobs && e == cudaSuccess; ++k)
            if (y_in(jobs[k])) {
                const long long m = nY(jobs[k]);
                e = cudaMemcpyAsync(jobs[k].dY + c0 * m, jobs[k].Y + c0 * m, sizeof(double) * n * m,
                                    cudaMemcpyHostToDevice, si);
            }
        return e;
    };
    auto finish = [&](int code) {
        cudaStreamSynchronize(si);
        cudaStreamSynchronize(s);
        cudaStreamSynchronize(so);
        return code;
    };
    // the copy streams start after whatever the handle's stream has pending
    CUDA_TRY(cudaEventRecord(h->ev_done[0], s));
    CUDA_TRY(cudaStreamWaitEvent(si, h->ev_done[0], 0));
    CUDA_TRY(cudaStreamWaitEvent(so, h->ev_done[0], 0));
    // copy segment c ends with the first plane of chunk c+1, the last face neighbour the cells
    // of chunk c need: ev_in[c] marks the moment chunk c can be evaluated
    cudaError_t e = cudaSuccess;
    if (nch > 1 && g.periodic[sd]) e = copy_in(planes - 1, planes);
    for (int c = 0; c < nch && e == cudaSuccess; ++c) {
        const long long p0 = first_plane(c) + (c > 0 ? 1 : 0);
        const long long p1 = std::min<long long>(first_plane(c + 1) + 1, planes);
        if (p1 > p0) e = copy_in(p0, p1);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_in[c], si);
    }
    if (e != cudaSuccess) return finish(fail(BOSSS_ERR_CUDA, cudaGetErrorString(e)));
    for (int c = 0; c < nch; ++c) {
        e = cudaStreamWaitEvent(s, h->ev_in[c], 0);
        for (int k = 0; k < njobs && e == cudaSuccess; ++k) {
            EvalArgs a = h->base;
            a.U = h->dU;
            a.V = jobs[k].mode != MODE_RES ? h->dV : nullptr;
            a.out = jobs[k].dY;
            a.alpha = jobs[k].alpha;
            a.beta = jobs[k].beta;
            a.time = time;
            a.cbeg = first_plane(c) * pc;
            a.cend = first_plane(c + 1) * pc;
            rc = launch_eval(h, jobs[k].mode, a, s);
            if (rc) return finish(rc);
        }
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_done[c], s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(so, h->ev_done[c], 0);
        for (int k = 0; k < njobs && e == cudaSuccess; ++k) {
            const long long c0 = first_plane(c) * pc, n = (first_plane(c + 1) - first_plane(c)) * pc, m = nY(jobs[k]);
            e = cudaMemcpyAsync(jobs[k].Y + c0 * m, jobs[k].dY + c0 * m, sizeof(double) * n * m, cudaMemcpyDeviceToHost,
                                so);
        }
        if (e != cudaSuccess) return finish(fail(BOSSS_ERR_CUDA, cudaGetErrorString(e)));
    }
    if (h->check_nan)
        for (int k = 0; k < njobs; ++k) {
            rc = check_nan(h, jobs[k].dY, nY(jobs[k]) * J, s);
            if (rc) return finish(rc);
        }
    e = cudaStreamSynchronize(so);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return finish(fail(BOSSS_ERR_CUDA, cudaGetErrorString(e)));
    return tc_volume_check(h);
}

int bosss_b200_evaluate(bosss_handle* h, double alpha, double beta, const double* U, double* out, double time) {
    if (!h || !U || !out) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    int rc = ensure_staging(h);
    if (rc) return rc;
    const HostJob job{MODE_RES, alpha, beta, out, h->dOut};
    return host_pipelined(h, &job, 1, U, nullptr, time);
}

int bosss_b200_jvp_device(bosss_handle* h, const double* U_dev, const double* V_dev, double* JV_dev, double time,
                          void* stream) {
    if (!h || !U_dev || !V_dev || !JV_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    return run_mode(h, MODE_JVP, 1.0, 0.0, U_dev, V_dev, JV_dev, time, s);
}

int bosss_b200_vjp_device(bosss_handle* h, const double* U_dev, const double* W_dev, double* JTW_dev, double time,
                          void* stream) {
    if (!h || !U_dev || !W_dev || !JTW_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    return run_mode(h, MODE_VJP, 1.0, 0.0, U_dev, W_dev, JTW_dev, time, s);
}

static int host_pair(bosss_handle* h, int mode, const double* U, const double* X, double* Y, double time) {
    if (!h || !U || !X || !Y) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    int rc = ensure_staging(h);
    if (rc) return rc;
    const HostJob job{mode, 1.0, 0.0, Y, h->dOut};
    return host_pipelined(h, &job, 1, U, X, time);
}

int bosss_b200_jvp(bosss_handle* h, const double* U, const double* V, double* JV, double time) {
    return host_pair(h, MODE_JVP, U, V, JV, time);
}

int bosss_b200_vjp(bosss_handle* h, const double* U, const double* W, double* JTW, double time) {
    return host_pair(h, MODE_VJP, U, W, JTW, time);
}

int bosss_b200_residual_vjp(bosss_handle* h, double alpha, double beta, const double* U, double* R, const double* W,
                            double* JTW, double time) {
    if (!h || !U || !R || !W || !JTW) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    int rc = ensure_staging(h);
    if (rc) return rc;
    if (!h->dOut2) CUDA_TRY(cudaMalloc(&h->dOut2, sizeof(double) * std::max<int64_t>(h->ndom, 1)));
    const HostJob jobs[2] = {{MODE_RES, alpha, beta, R, h->dOut}, {MODE_VJP, 1.0, 0.0, JTW, h->dOut2}};
    return host_pipelined(h, jobs, 2, U, W, time);
}

int bosss_b200_synchronize(bosss_handle* h) {
    if (!h) return fail(BOSSS_ERR_BAD_ARG, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return tc_volume_check(h);
}

// ---------------------------------------------------------------- block-sparse matrix
int bosss_b200_bsr_create(int64_t n_block_rows, int64_t n_block_cols, int32_t row_block, int32_t col_block,
                          const int64_t* row_ptr, const int32_t* col_idx, const double* values, int32_t device,
                          bosss_bsr** out) {
    if (!out || !row_ptr || n_block_rows < 0 || n_block_cols < 0 || row_block < 1 || col_block < 1)
        return fail(BOSSS_ERR_BAD_ARG, "bad block-sparse matrix arguments");
    *out = nullptr;
    const int64_t nnzb = row_ptr[n_block_rows];
    if (row_ptr[0] != 0 || nnzb < 0) return fail(BOSSS_ERR_BAD_ARG, "row_ptr must start at 0");
    for (int64_t i = 0; i < n_block_rows; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return fail(BOSSS_ERR_BAD_ARG, "row_ptr not monotone");
    if (nnzb > 0 && (!col_idx || !values)) return fail(BOSSS_ERR_BAD_ARG, "missing col_idx/values");
    for (int64_t b = 0; b < nnzb; ++b)
        if (col_idx[b] < 0 || col_idx[b] >= n_block_cols) return fail(BOSSS_ERR_BAD_ARG, "column index out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(BOSSS_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(BOSSS_ERR_BAD_ARG, "bad device ordinal");
    bosss_bsr* A = new bosss_bsr();
    A->device = device;
    A->nbr = n_block_rows;
    A->nbc = n_block_cols;
    A->nnzb = nnzb;
    A->br = row_block;
    A->bc = col_block;
    const size_t bs = (size_t)row_block * col_block;
    std::vector<double> cm(std::max<size_t>(nnzb * bs, 1));
    for (int64_t b = 0; b < nnzb; ++b)
        for (int r = 0; r < row_block; ++r)
            for (int c = 0; c < col_block; ++c) cm[b * bs + (size_t)c * row_block + r] = values[b * bs + (size_t)r * col_block + c];
    auto cleanup = [&](cudaError_t e) {
        bosss_b200_bsr_destroy(A);
        return fail(BOSSS_ERR_CUDA, std::string("block-sparse upload: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&A->d_rowptr, sizeof(int64_t) * (n_block_rows + 1));
    if (e == cudaSuccess) e = cudaMalloc(&A->d_colidx, sizeof(int32_t) * std::max<int64_t>(nnzb, 1));
    if (e == cudaSuccess) e = cudaMalloc(&A->d_vals, sizeof(double) * cm.size());
    if (e == cudaSuccess) e = cudaMemcpy(A->d_rowptr, row_ptr, sizeof(int64_t) * (n_block_rows + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnzb) e = cudaMemcpy(A->d_colidx, col_idx, sizeof(int32_t) * nnzb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(A->d_vals, cm.data(), sizeof(double) * cm.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cleanup(e);
    *out = A;
    return BOSSS_OK;
}

int bosss_b200_bsr_destroy(bosss_bsr* A) {
    if (!A) return BOSSS_OK;
    cudaSetDevice(A->device);
    if (A->stream) cudaStreamSynchronize(A->stream);
    cudaFree(A->d_rowptr);
    cudaFree(A->d_colidx);
    cudaFree(A->d_vals);
    cudaFree(A->d_vals32);
    cudaFree(A->d_ell_col);
    cudaFree(A->d_ell_vals);
    cudaFree(A->dx);
    cudaFree(A->dy);
    if (A->stream) cudaStreamDestroy(A->stream);
    delete A;
    return BOSSS_OK;
}

int bosss_b200_bsr_spmv_device(bosss_bsr* A, double alpha, const double* x_dev, double beta, double* y_dev,
                               void* stream) {
    if (!A || !x_dev || !y_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(A->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : A->stream;
    return bsr_spmv(A, alpha, x_dev, beta, y_dev, s);
}

int bosss_b200_bsr_spmv(bosss_bsr* A, double alpha, const double* x, double beta, double* y) {
    if (!A || !x || !y) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(A->device));
    const int64_t nx = A->nbc * A->bc, ny = A->nbr * A->br;
    if (!A->dx) {
        CUDA_TRY(cudaMalloc(&A->dx, sizeof(double) * std::max<int64_t>(nx, 1)));
        CUDA_TRY(cudaMalloc(&A->dy, sizeof(double) * std::max<int64_t>(ny, 1)));
    }
    cudaStream_t s = A->stream;
    CUDA_TRY(cudaMemcpyAsync(A->dx, x, sizeof(double) * nx, cudaMemcpyHostToDevice, s));
    if (beta != 0.0) CUDA_TRY(cudaMemcpyAsync(A->dy, y, sizeof(double) * ny, cudaMemcpyHostToDevice, s));
    int rc = bosss_b200_bsr_spmv_device(A, alpha, A->dx, beta, A->dy, s);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(y, A->dy, sizeof(double) * ny, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return BOSSS_OK;
}

int bosss_b200_bsr_get(const bosss_bsr* A, int64_t* n_block_rows, int64_t* n_block_cols, int32_t* row_block,
                       int32_t* col_block, int64_t* nnz_blocks, int64_t* row_ptr, int32_t* col_idx, double* values) {
    if (!A) return fail(BOSSS_ERR_BAD_ARG, "null matrix");
    if (n_block_rows) *n_block_rows = A->nbr;
    if (n_block_cols) *n_block_cols = A->nbc;
    if (row_block) *row_block = A->br;
    if (col_block) *col_block = A->bc;
    if (nnz_blocks) *nnz_blocks = A->nnzb;
    CUDA_TRY(cudaSetDevice(A->device));
    CUDA_TRY(cudaStreamSynchronize(A->stream));
    if (row_ptr) CUDA_TRY(cudaMemcpy(row_ptr, A->d_rowptr, sizeof(int64_t) * (A->nbr + 1), cudaMemcpyDeviceToHost));
    if (col_idx && A->nnzb) CUDA_TRY(cudaMemcpy(col_idx, A->d_colidx, sizeof(int32_t) * A->nnzb, cudaMemcpyDeviceToHost));
    if (values && A->nnzb) {
        const size_t bs = (size_t)A->br * A->bc;
        std::vector<double> cm(A->nnzb * bs);
        CUDA_TRY(cudaMemcpy(cm.data(), A->d_vals, sizeof(double) * cm.size(), cudaMemcpyDeviceToHost));
        for (int64_t b = 0; b < A->nnzb; ++b)
            for (int r = 0; r < A->br; ++r)
                for (int c = 0; c < A->bc; ++c) values[b * bs + (size_t)r * A->bc + c] = cm[b * bs + (size_t)c * A->br + r];
    }
    return BOSSS_OK;
}


}  // extern "C"
