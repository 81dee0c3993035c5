// dg_physics.cuh -- device functors of the equation components the GPU path supports.
//
// Each functor reproduces the pointwise semantics of a reference equation component
// in the vectorised form the reference evaluators use (NonlinFormVectorizer.cs:31-716):
// a volume term is returned as (fV, fG) = coefficients of (v, grad v); an edge term as
// (gA, GA, gB, GB) = coefficients of (v_IN, grad v_IN, v_OUT, grad v_OUT). For an
// INonlinearFlux the volume flux F enters as fG = -F (NECQuadratureVolume.cs:452) and the
// edge flux f as gA = +f, gB = -f (NECQuadratureEdge.cs:998-1000).
//
// All functors are templated on the scalar type, so the same code runs in FP64
// (residual), with DualN<1> (JVP) and with DualN<n> (gradient of the adjoint functional,
// VJP). Outputs are accumulated (+=).
#pragma once
#include "dg_common.cuh"

namespace bosss {

struct PhysParams {
    double vel[3];        // transport velocity (ScalarTransportFlux parameter fields, constant)
    int has_transport;
    int has_sip;
    double pen;           // SIP: penalty_base * penalty_deg   (ipLaplace.cs CoefficientUpdate)
    double nu0, nu2;      // SIP: nu(u) = nu0 + nu2*u^2
    int dirichlet;        // SIP boundary: 1 = Dirichlet g_D(x), 0 = Neumann with g_N = 0
    double g0, g1[3], g2[3];  // g_D(x) = g0 + sum g1_d x_d + g2_d x_d^2
    int has_source;
    double src;           // constant source value
    double gamma, mach;   // HLLC
};

template <class T> __device__ __forceinline__ T tconst(double a) { return T(a); }

// --------------------------------------------------------------- scalar: transport + SIP + source
// ScalarTransportFlux(3D)  ScalarTransport/TransportFlux.cs:29-191
// SIPLaplace               NSECommon/ipLaplace.cs:30-269 (Nu -> nu(u))
template <int D_, bool SIP>
struct PhysScalar {
    static constexpr int D = D_;
    static constexpr int NV = 1, NC = 1;
    static constexpr bool GRAD_U = SIP;     // forms read grad u
    static constexpr bool VOL_V = SIP;      // source term (only instantiated with the SIP family)
    static constexpr bool VOL_G = true;
    static constexpr bool FACE_V = true;
    static constexpr bool FACE_G = SIP;     // symmetry term of SIP

    template <class T>
    __device__ static void volume(const PhysParams& p, const T* U, const T (*G)[D], const double* x, T* fV,
                                  T (*fG)[D]) {
        (void)x;
        if (p.has_transport) {
#pragma unroll
            for (int d = 0; d < D; ++d) fG[0][d] -= U[0] * p.vel[d];   // -F, F = a u
        }
        if constexpr (SIP) {
            if (p.has_sip) {
                T nu = U[0] * U[0] * p.nu2 + p.nu0;
#pragma unroll
                for (int d = 0; d < D; ++d) fG[0][d] -= G[0][d] * nu;   // VolumeForm: -grad u . grad v * Nu
            }
            if (p.has_source) fV[0] += p.src;
        }
    }

    template <class T>
    __device__ static void inner(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D], const T* UB,
                                 const T (*GB)[D], const double* n, const double* x, T* gA, T (*GAv)[D], T* gB,
                                 T (*GBv)[D]) {
        (void)x;
        if (p.has_transport) {
            double an = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) an += p.vel[d] * n[d];
            T f = (an > 0.0) ? UA[0] * an : UB[0] * an;   // upwind (InnerEdgeFlux)
            gA[0] += f;
            gB[0] -= f;
        }
        if constexpr (SIP) {
            if (p.has_sip) {
                T uA = UA[0], uB = UB[0];
                T nuA = uA * uA * p.nu2 + p.nu0;
                T nuB = uB * uB * p.nu2 + p.nu0;
                T jump = uA - uB;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    T cons = (nuA * GA[0][d] + nuB * GB[0][d]) * (0.5 * n[d]);   // consistency
                    gA[0] += cons;
                    gB[0] -= cons;
                    GAv[0][d] += nuA * jump * (0.5 * n[d]);                      // symmetry
                    GBv[0][d] += nuB * jump * (0.5 * n[d]);
                }
                T nuMax = (fabs(pval(nuA)) > fabs(pval(nuB))) ? nuA : nuB;
                T pen = jump * nuMax * pnlty;                                   // penalty
                gA[0] -= pen;
                gB[0] += pen;
            }
        }
    }

    template <class T>
    __device__ static void boundary(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D],
                                    const double* n, const double* x, T* gA, T (*GAv)[D]) {
        if (p.has_transport) {
            double an = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) an += p.vel[d] * n[d];
            if (D == 2) {
                gA[0] += UA[0] * an;                  // 2D: (vel*Uin)*n on in- and outflow
            } else {
                if (an >= 0.0) gA[0] += UA[0] * an;   // 3D: inflow value 0
            }
        }
        if constexpr (SIP) {
            if (p.has_sip && p.dirichlet) {
                double gD = p.g0;
#pragma unroll
                for (int d = 0; d < D; ++d) gD += p.g1[d] * x[d] + p.g2[d] * x[d] * x[d];
                T uA = UA[0];
                T nuA = uA * uA * p.nu2 + p.nu0;
                T diff = uA - gD;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    gA[0] += nuA * GA[0][d] * n[d];       // consistency
                    GAv[0][d] += nuA * diff * n[d];       // symmetry
                }
                gA[0] -= nuA * diff * pnlty;              // penalty (pnlty = 2*GetPenalty)
            }
        }
    }
};

// --------------------------------------------------------------- compressible Euler, HLLC
// OptimizedHLLC{Density,Momentum,Energy}Flux, CompressibleFlowCommon/Convection/*.cs.
// The three reference components share the same wave-speed estimate; the functor
// evaluates it once for all D+2 codomain variables.
template <int D_>
struct PhysEuler {
    static constexpr int D = D_;
    static constexpr int NV = D + 2, NC = D + 2;
    static constexpr bool GRAD_U = false;
    static constexpr bool VOL_V = false;
    static constexpr bool VOL_G = true;
    static constexpr bool FACE_V = true;
    static constexpr bool FACE_G = false;

    template <class T>
    __device__ static void volume(const PhysParams& p, const T* U, const T (*G)[D], const double* x, T* fV,
                                  T (*fG)[D]) {
        (void)G; (void)x; (void)fV;
        const double gMs = p.gamma * p.mach * p.mach;
        T rho = U[0], E = U[D + 1];
        T msq = U[1] * U[1];
#pragma unroll
        for (int d = 1; d < D; ++d) msq += U[d + 1] * U[d + 1];
        T irho = 1.0 / rho;
        // density: F_d = m_d
#pragma unroll
        for (int d = 0; d < D; ++d) fG[0][d] -= U[d + 1];
        // momentum c: F_d = m_c m_d / rho + delta_cd p/(gamma Ma^2)
        T pm = (E - msq * irho * (gMs * 0.5)) * ((p.gamma - 1.0) / gMs);
#pragma unroll
        for (int c = 0; c < D; ++c) {
#pragma unroll
            for (int d = 0; d < D; ++d) {
                T F = U[c + 1] * U[d + 1] / rho;
                if (c == d) F += pm;
                fG[c + 1][d] -= F;
            }
        }
        // energy: F_d = m_d/rho (E + p)
        T pe = (E - msq / rho * (gMs * 0.5)) * (p.gamma - 1.0);
#pragma unroll
        for (int d = 0; d < D; ++d) fG[D + 1][d] -= U[d + 1] / rho * (E + pe);
    }

    template <class T>
    __device__ static void inner(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D], const T* UB,
                                 const T (*GB)[D], const double* n, const double* x, T* gA, T (*GAv)[D], T* gB,
                                 T (*GBv)[D]) {
        (void)pnlty; (void)GA; (void)GB; (void)x; (void)GAv; (void)GBv;
        const double gamma = p.gamma, Mach = p.mach;
        const double MachScaling = gamma * Mach * Mach;
        T rhoIn = UA[0], rhoOut = UB[0];
        T msIn = UA[1] * UA[1], msOut = UB[1] * UB[1];
        T unIn = UA[1] * n[0], unOut = UB[1] * n[0];
#pragma unroll
        for (int d = 1; d < D; ++d) {
            msIn += UA[d + 1] * UA[d + 1];
            msOut += UB[d + 1] * UB[d + 1];
            unIn += UA[d + 1] * n[d];
            unOut += UB[d + 1] * n[d];
        }
        unIn = unIn / rhoIn;
        unOut = unOut / rhoOut;
        T EIn = UA[D + 1], EOut = UB[D + 1];
        T pIn = (EIn - msIn / rhoIn * (MachScaling * 0.5)) * (gamma - 1.0);
        T pOut = (EOut - msOut / rhoOut * (MachScaling * 0.5)) * (gamma - 1.0);
        T cInS = dsqrt(pIn / rhoIn) / Mach;
        T cOutS = dsqrt(pOut / rhoOut) / Mach;
        T rhoMean = (rhoIn + rhoOut) * 0.5;
        T pMean = (pIn + pOut) * 0.5;
        T cMean = (cInS + cOutS) * 0.5;
        T velJump = unOut - unIn;
        T pStar = pMean - velJump * cMean * rhoMean * (0.5 * MachScaling);
        if (0.0 > pval(pStar)) pStar = T(0.0);           // Math.Max(0.0, pStar)
        T qIn = T(1.0), qOut = T(1.0);
        if (pval(pStar) > pval(pIn)) qIn = dsqrt(1.0 + (pStar / pIn - 1.0) * (0.5 * (gamma + 1.0) / gamma));
        if (pval(pStar) > pval(pOut)) qOut = dsqrt(1.0 + (pStar / pOut - 1.0) * (0.5 * (gamma + 1.0) / gamma));
        T sIn = unIn - cInS * qIn;
        T sOut = unOut + cOutS * qOut;
        T cIn = rhoIn * (sIn - unIn);
        T cOut = rhoOut * (sOut - unOut);
        T speedDiff = cOut * unOut - cIn * unIn;
        T dp = pIn - pOut;
        T sStar = (speedDiff + dp / MachScaling) / (cOut - cIn);

        T f[D + 2];
        if (pval(sStar) > 0.0) {
            f[0] = unIn * rhoIn;
#pragma unroll
            for (int c = 0; c < D; ++c) f[c + 1] = unIn * UA[c + 1] + pIn / MachScaling * n[c];
            f[D + 1] = unIn * (EIn + pIn);
            if (pval(sIn) <= 0.0) {
                T ratio = (sIn - unIn) / (sIn - sStar);
                T modRho = rhoIn * ratio;
                f[0] += sIn * (modRho - rhoIn);
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    T modM = rhoIn * ratio * (UA[c + 1] / rhoIn + (sStar - unIn) * n[c]);
                    f[c + 1] += sIn * (modM - UA[c + 1]);
                }
                T factor = rhoIn * sStar * MachScaling + pIn / (sIn - unIn);
                T modE = ratio * (EIn + factor * (sStar - unIn));
                f[D + 1] += sIn * (modE - EIn);
            }
        } else {
            f[0] = unOut * rhoOut;
#pragma unroll
            for (int c = 0; c < D; ++c) f[c + 1] = unOut * UB[c + 1] + pOut / MachScaling * n[c];
            f[D + 1] = unOut * (EOut + pOut);
            if (pval(sOut) >= 0.0) {
                T ratio = (sOut - unOut) / (sOut - sStar);
                T modRho = rhoOut * ratio;
                f[0] += sOut * (modRho - rhoOut);
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    T modM = rhoOut * ratio * (UB[c + 1] / rhoOut + (sStar - unOut) * n[c]);
                    f[c + 1] += sOut * (modM - UB[c + 1]);
                }
                T factor = rhoOut * sStar * MachScaling + pOut / (sOut - unOut);
                T modE = ratio * (EOut + factor * (sStar - unOut));
                f[D + 1] += sOut * (modE - EOut);
            }
        }
#pragma unroll
        for (int c = 0; c < D + 2; ++c) {
            gA[c] += f[c];
            gB[c] -= f[c];
        }
    }

    template <class T>
    __device__ static void boundary(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D],
                                    const double* n, const double* x, T* gA, T (*GAv)[D]) {
        // no boundary-condition map on the device: create() rejects non-periodic Euler grids
        (void)p; (void)pnlty; (void)UA; (void)GA; (void)n; (void)x; (void)gA; (void)GAv;
    }
};

}  // namespace bosss
