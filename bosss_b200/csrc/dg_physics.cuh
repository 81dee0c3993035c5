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
#include <cmath>

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
    double gamma, mach;   // HLLC, CNS viscous terms
    double ims, imach;    // HLLC: 1/(gamma Ma^2), 1/Ma
    // CNS viscous terms (OptimizedSIPG fluxes): Reynolds and Prandtl numbers, bulk / shear
    // viscosity ratio, viscosity law (0: mu = 1, 1: Sutherland with ratio suth = S/T0)
    double re, pr, visc_ratio, suth;
    int visc_law;
};

template <class T> __host__ __device__ __forceinline__ T tconst(double a) { return T(a); }

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
    static constexpr bool ADJOINT = false;  // VJP by forward mode over the node's state
    static constexpr double BND_PEN = 2.0;  // boundary penalty = 2 * GetPenalty (ipLaplace.cs:224)

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

    // ub: the boundary-state table's outer values at this node (null without a table; unused here);
    // kind: the node's boundary-condition kind (0 here: create() rejects other kinds)
    template <class T>
    __device__ static void boundary(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D],
                                    const double* n, const double* x, const double* ub, int kind, T* gA,
                                    T (*GAv)[D]) {
        (void)ub;
        (void)kind;
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

// --------------------------------------------------------------- compressible Navier-Stokes, viscous SIPG
// OptimizedSIPG{Density,Momentum,Energy}Flux of the CNS solver (CNS/Diffusion/OptimizedSIPG*Flux.cs):
// the viscous flux of the D+2 conservative equations F_k = sum_{l,j} G[k][l][j] dU_j/dx_l with
// Hartmann's G tensors (UpdateTensorComponent / UpdateBoundaryTensorComponent, entries in
// closed form below), symmetric interior penalty edge terms with the penalty
// SIPGPenaltyScaling * p^2 * max(cj_in, cj_out) (p.pen = SIPGPenaltyScaling * p^2) inside and
// p^2 cj_in on boundary faces, where the outer state is the boundary-state table's value at
// the node (SupersonicInlet.GetBoundaryState). Every edge term applies the same linear map
// G(U) . X to X = grad U or X = jump (x) normal, so the functor evaluates that map directly.
template <int D_>
struct PhysCNSVisc {
    static constexpr int D = D_;
    static constexpr int NV = D + 2, NC = D + 2;
    static constexpr bool GRAD_U = true;
    static constexpr bool VOL_V = false;
    static constexpr bool VOL_G = true;
    static constexpr bool FACE_V = true;
    static constexpr bool FACE_G = true;
    static constexpr bool ADJOINT = false;
    static constexpr double BND_PEN = 1.0;   // NonlinBoundaryEdge_V: p^2 cj_in, not doubled

    // F_k = sum_{l,j} G_e[k][l][j] X[j][l] for equation e (1..D momentum, D+1 energy; 0 density
    // has no viscous flux) at the state U
    template <class T>
    __host__ __device__ static void vflux(const PhysParams& p, int e, const T* U, const T (*X)[D], T* F) {
        const double MS = p.gamma * p.mach * p.mach, gPr = p.gamma / p.pr;
        const double a43 = p.visc_ratio + 4.0 / 3.0, a23 = p.visc_ratio - 2.0 / 3.0, a13 = p.visc_ratio + 1.0 / 3.0;
        const T irho = 1.0 / U[0];
        T v[D];
        T q = U[1] * (U[1] * irho) * irho;
        v[0] = U[1] * irho;
#pragma unroll
        for (int i = 1; i < D; ++i) {
            v[i] = U[1 + i] * irho;
            q += v[i] * v[i];
        }
        const T en = U[D + 1] * irho;
        const T temp = (en - q * (0.5 * MS)) * (p.gamma - 1.0);
        T mu = T(1.0);
        if (p.visc_law == 1) mu = temp * dsqrt(temp) * (1.0 + p.suth) / (temp + p.suth);   // SutherlandLaw
        const T mh = mu * irho * (1.0 / p.re);
#pragma unroll
        for (int k = 0; k < D; ++k) F[k] = T(0.0);
        if (e >= 1 && e <= D) {
            const int c = e - 1;
            // tau_ck on the conservative gradients: d_l v_i = (X[1+i][l] - v_i X[0][l]) / rho
#pragma unroll
            for (int k = 0; k < D; ++k)
#pragma unroll
                for (int l = 0; l < D; ++l)
#pragma unroll
                    for (int i = 0; i < D; ++i) {
                        double coef = 0.0;
                        if (l == k && i == c) coef += 1.0;
                        if (l == c && i == k) coef += 1.0;
                        if (c == k && i == l) coef += a23;
                        if (coef != 0.0) F[k] += (X[1 + i][l] - v[i] * X[0][l]) * (coef * mh);
                    }
            // two dimensions, y-momentum: the reference's G[x][y][rho] is -v_y mu_hat
            // (OptimizedSIPGMomentumFlux.cs:767, SIPGMomentumFlux.cs:63)
            if (D == 2 && c == 1) F[0] += (v[0] - v[D - 1]) * X[0][1] * mh;
        } else if (e == D + 1) {
#pragma unroll
            for (int k = 0; k < D; ++k)
#pragma unroll
                for (int l = 0; l < D; ++l) {
                    if (k == l) {
                        T g0 = -((v[k] * v[k] * a13 + q) * MS + (en - q * MS) * gPr);
                        T acc = g0 * X[0][k] + X[D + 1][k] * gPr;
#pragma unroll
                        for (int i = 0; i < D; ++i)
                            acc += X[1 + i][k] * v[i] * (MS * ((i == k) ? (a43 - gPr) : (1.0 - gPr)));
                        F[k] += acc * mh;
                    } else {
                        T acc = -(v[k] * v[l]) * (MS * a13) * X[0][l] + v[l] * MS * X[1 + k][l] +
                                v[k] * (MS * a23) * X[1 + l][l];
                        F[k] += acc * mh;
                    }
                }
        }
    }

    template <class T>
    __host__ __device__ static void volume(const PhysParams& p, const T* U, const T (*G)[D], const double* x, T* fV,
                                           T (*fG)[D]) {
        (void)x; (void)fV;
#pragma unroll
        for (int e = 1; e < NC; ++e) {
            T F[D];
            vflux(p, e, U, G, F);
#pragma unroll
            for (int k = 0; k < D; ++k) fG[e][k] += F[k];   // INonlinVolumeForm_GradV: f[k] += G . grad U
        }
    }

    template <class T>
    __host__ __device__ static void inner(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D],
                                          const T* UB, const T (*GB)[D], const double* n, const double* x, T* gA,
                                          T (*GAv)[D], T* gB, T (*GBv)[D]) {
        (void)x;
        T J[NV][D];
#pragma unroll
        for (int j = 0; j < NV; ++j)
#pragma unroll
            for (int l = 0; l < D; ++l) J[j][l] = (UA[j] - UB[j]) * n[l];
#pragma unroll
        for (int e = 1; e < NC; ++e) {
            T FA[D], FB[D], PA[D], PB[D];
            vflux(p, e, UA, GA, FA);
            vflux(p, e, UB, GB, FB);
            vflux(p, e, UA, J, PA);
            vflux(p, e, UB, J, PB);
            T flux = T(0.0);
#pragma unroll
            for (int k = 0; k < D; ++k) {
                flux += (FA[k] + FB[k]) * (-0.5 * n[k]);            // consistency
                flux += (PA[k] + PB[k]) * (0.5 * pnlty * n[k]);     // penalty
                GAv[e][k] -= PA[k] * 0.5;                           // NonlinInternalEdge_GradV
                GBv[e][k] -= PB[k] * 0.5;
            }
            gA[e] += flux;
            gB[e] -= flux;
        }
    }

    template <class T>
    __host__ __device__ static void boundary(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D],
                                             const double* n, const double* x, const double* ub, int kind, T* gA,
                                             T (*GAv)[D]) {
        (void)x;
        (void)kind;   // prescribed states only (set_boundary_kinds rejects other kinds for this operator)
        if (!ub) return;   // create() requires the boundary-state table when the grid has boundary faces
        T Uo[NV], J[NV][D];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            Uo[j] = T(ub[j]);
#pragma unroll
            for (int l = 0; l < D; ++l) J[j][l] = (UA[j] - ub[j]) * n[l];
        }
#pragma unroll
        for (int e = 1; e < NC; ++e) {
            T F[D], P[D];
            vflux(p, e, Uo, GA, F);      // G of the outer state applied to grad U_in
            vflux(p, e, Uo, J, P);
            T flux = T(0.0);
#pragma unroll
            for (int k = 0; k < D; ++k) {
                flux += F[k] * (-n[k]) + P[k] * (pnlty * n[k]);
                GAv[e][k] -= P[k];
            }
            gA[e] += flux;
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
    static constexpr double BND_PEN = 2.0;   // (no penalty terms)

    // FP64 divisions are costly on the GPU (a reciprocal estimate plus Newton steps): every
    // quotient by a state-dependent value below is a product with one reciprocal, and the
    // constants 1/(gamma Ma^2), 1/Ma come precomputed in PhysParams (ims, imach)
    template <class T>
    __host__ __device__ static void volume(const PhysParams& p, const T* U, const T (*G)[D], const double* x, T* fV,
                                           T (*fG)[D]) {
        (void)G; (void)x; (void)fV;
        const double gMs = p.gamma * p.mach * p.mach;
        T rho = U[0], E = U[D + 1];
        T irho = 1.0 / rho;
        T u[D];
#pragma unroll
        for (int d = 0; d < D; ++d) u[d] = U[d + 1] * irho;
        T kin = U[1] * u[0];                  // |m|^2 / rho
#pragma unroll
        for (int d = 1; d < D; ++d) kin += U[d + 1] * u[d];
        // density: F_d = m_d
#pragma unroll
        for (int d = 0; d < D; ++d) fG[0][d] -= U[d + 1];
        // momentum c: F_d = m_c u_d + delta_cd p/(gamma Ma^2)
        T pm = (E - kin * (gMs * 0.5)) * ((p.gamma - 1.0) * p.ims);
#pragma unroll
        for (int c = 0; c < D; ++c) {
#pragma unroll
            for (int d = 0; d < D; ++d) {
                T F = U[c + 1] * u[d];
                if (c == d) F += pm;
                fG[c + 1][d] -= F;
            }
        }
        // energy: F_d = u_d (E + p)
        T pe = (E - kin * (gMs * 0.5)) * (p.gamma - 1.0);
#pragma unroll
        for (int d = 0; d < D; ++d) fG[D + 1][d] -= u[d] * (E + pe);
    }

    template <class T>
    __host__ __device__ static void inner(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D], const T* UB,
                                          const T (*GB)[D], const double* n, const double* x, T* gA, T (*GAv)[D],
                                          T* gB, T (*GBv)[D]) {
        (void)pnlty; (void)GA; (void)GB; (void)x; (void)GAv; (void)GBv;
        const double gamma = p.gamma;
        const double MachScaling = gamma * p.mach * p.mach, iMS = p.ims;
        const double G2 = 0.5 * (gamma + 1.0) / gamma;
        T rhoIn = UA[0], rhoOut = UB[0];
        T irIn = 1.0 / rhoIn, irOut = 1.0 / rhoOut;
        T msIn = UA[1] * UA[1], msOut = UB[1] * UB[1];
        T unIn = UA[1] * n[0], unOut = UB[1] * n[0];
#pragma unroll
        for (int d = 1; d < D; ++d) {
            msIn += UA[d + 1] * UA[d + 1];
            msOut += UB[d + 1] * UB[d + 1];
            unIn += UA[d + 1] * n[d];
            unOut += UB[d + 1] * n[d];
        }
        unIn = unIn * irIn;
        unOut = unOut * irOut;
        T EIn = UA[D + 1], EOut = UB[D + 1];
        T pIn = (EIn - msIn * irIn * (MachScaling * 0.5)) * (gamma - 1.0);
        T pOut = (EOut - msOut * irOut * (MachScaling * 0.5)) * (gamma - 1.0);
        T cInS = dsqrt(pIn * irIn) * p.imach;
        T cOutS = dsqrt(pOut * irOut) * p.imach;
        T rhoMean = (rhoIn + rhoOut) * 0.5;
        T pMean = (pIn + pOut) * 0.5;
        T cMean = (cInS + cOutS) * 0.5;
        T velJump = unOut - unIn;
        T pStar = pMean - velJump * cMean * rhoMean * (0.5 * MachScaling);
        if (0.0 > pval(pStar)) pStar = T(0.0);           // Math.Max(0.0, pStar)
        T qIn = T(1.0), qOut = T(1.0);
        if (pval(pStar) > pval(pIn)) qIn = dsqrt(1.0 + (pStar / pIn - 1.0) * G2);
        if (pval(pStar) > pval(pOut)) qOut = dsqrt(1.0 + (pStar / pOut - 1.0) * G2);
        T sIn = unIn - cInS * qIn;
        T sOut = unOut + cOutS * qOut;
        T cIn = rhoIn * (sIn - unIn);
        T cOut = rhoOut * (sOut - unOut);
        T speedDiff = cOut * unOut - cIn * unIn;
        T dp = pIn - pOut;
        T sStar = (speedDiff + dp * iMS) / (cOut - cIn);

        // upwind side of the contact wave
        const bool left = pval(sStar) > 0.0;
        const T* Us = left ? UA : UB;
        const T r = left ? rhoIn : rhoOut, ir = left ? irIn : irOut, E = left ? EIn : EOut;
        const T pp = left ? pIn : pOut, un = left ? unIn : unOut, s = left ? sIn : sOut;
        T f[D + 2];
        f[0] = un * r;
        const T pms = pp * iMS;
#pragma unroll
        for (int c = 0; c < D; ++c) f[c + 1] = un * Us[c + 1] + pms * n[c];
        f[D + 1] = un * (E + pp);
        if (left ? (pval(s) <= 0.0) : (pval(s) >= 0.0)) {
            T ratio = (s - un) / (s - sStar);
            T modRho = r * ratio;
            f[0] += s * (modRho - r);
            const T t = sStar - un;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                T modM = r * ratio * (Us[c + 1] * ir + t * n[c]);
                f[c + 1] += s * (modM - Us[c + 1]);
            }
            T factor = r * sStar * MachScaling + pp / (s - un);
            T modE = ratio * (E + factor * t);
            f[D + 1] += s * (modE - E);
        }
#pragma unroll
        for (int c = 0; c < D + 2; ++c) {
            gA[c] += f[c];
            gB[c] -= f[c];
        }
    }

    template <class T>
    __host__ __device__ static void boundary(const PhysParams& p, double pnlty, const T* UA, const T (*GA)[D],
                                             const double* n, const double* x, const double* ub, int kind, T* gA,
                                             T (*GAv)[D]) {
        // OptimizedHLLCFlux.BorderEdgeFlux (OptimizedHLLCFlux.cs:61-131): the outer state of the
        // boundary condition, then the inner-edge HLLC flux with the outward normal. Outer state:
        // kind 0 the boundary-state table's value (a constant of the linearisation), kind 1 the
        // inner state (SupersonicOutlet.GetBoundaryState), kind 2 the inner state with the
        // normal momentum reflected, m - 2 (m . n) n (AdiabaticSlipWall.GetBoundaryState without
        // wall velocities)
        (void)GA;
        if (kind == 0 && !ub) return;   // the entry points require the table for kind-0 nodes
        T Uo[NV], GB[NV][D], gB[NC], GBv[NC][D];
        T mn = T(0.0);
        if (kind == 2)
#pragma unroll
            for (int d = 0; d < D; ++d) mn += UA[1 + d] * n[d];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            if (kind == 0) Uo[i] = T(ub[i]);
            else if (kind == 2 && i >= 1 && i <= D) Uo[i] = UA[i] - 2.0 * mn * n[i - 1];
            else Uo[i] = UA[i];
#pragma unroll
            for (int d = 0; d < D; ++d) GB[i][d] = T(0.0);
        }
#pragma unroll
        for (int e = 0; e < NC; ++e) gB[e] = T(0.0);
        inner<T>(p, pnlty, UA, GA, Uo, GB, n, x, gA, GAv, gB, GBv);
    }

    // ---- reverse-mode adjoints (VJP): one primal sweep plus one reverse sweep per node in
    // place of the NV-slot forward mode. Same functions as volume() / inner() above,
    // differentiated by hand.
    static constexpr bool ADJOINT = true;

    // Ub[i] = d/dU_i sum_{e,d} fG[e][d] * Gw[e][d] with fG = -F(U) (volume flux)
    __host__ __device__ static void volume_adj(const PhysParams& p, const double* U, const double (*Gw)[D],
                                               double* Ub) {
        const double g = p.gamma, gMs = g * p.mach * p.mach;
        const double rho = U[0], E = U[D + 1], irho = 1.0 / rho;
        double u[D], kin = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            u[d] = U[d + 1] * irho;
            kin += U[d + 1] * u[d];
        }
        const double pm = (E - kin * (gMs * 0.5)) * ((g - 1.0) * p.ims);
        const double pe = gMs * pm;
        double A = 0.0, gu = 0.0, uMu = 0.0, usq = 0.0;
        double Mu[D], Mtu[D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            A += Gw[c + 1][c];
            gu += Gw[D + 1][c] * u[c];
            usq += u[c] * u[c];
            Mu[c] = 0.0;
            Mtu[c] = 0.0;
        }
#pragma unroll
        for (int c = 0; c < D; ++c)
#pragma unroll
            for (int d = 0; d < D; ++d) {
                Mu[c] += Gw[c + 1][d] * u[d];
                Mtu[c] += Gw[d + 1][c] * u[d];
            }
#pragma unroll
        for (int c = 0; c < D; ++c) uMu += u[c] * Mu[c];
        const double Epe = (E + pe) * irho;
        const double gm1 = g - 1.0;
        const double s = A + gMs * gu;
        Ub[0] = uMu - 0.5 * gm1 * usq * s + gu * Epe;
#pragma unroll
        for (int k = 0; k < D; ++k) Ub[k + 1] = -(Gw[0][k] + Mu[k] + Mtu[k] - gm1 * u[k] * s + Gw[D + 1][k] * Epe);
        Ub[D + 1] = -(A * gm1 * p.ims + gu * g);
    }

    // UAb / UBb = gradient of sum_c f_c(UA, UB) * fb[c] (f: the HLLC flux of inner())
    __host__ __device__ static void inner_adj(const PhysParams& p, const double* UA, const double* UB,
                                              const double* n, const double* fb, double* UAb, double* UBb) {
        const double g = p.gamma, MS = g * p.mach * p.mach, iMS = p.ims, G2 = 0.5 * (g + 1.0) / g;
        // ---- primal (as inner())
        const double rA = UA[0], rB = UB[0], EA = UA[D + 1], EB = UB[D + 1];
        const double irA = 1.0 / rA, irB = 1.0 / rB;
        double msA = 0.0, msB = 0.0, unrA = 0.0, unrB = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            msA += UA[d + 1] * UA[d + 1];
            msB += UB[d + 1] * UB[d + 1];
            unrA += UA[d + 1] * n[d];
            unrB += UB[d + 1] * n[d];
        }
        const double unA = unrA * irA, unB = unrB * irB;
        const double kA = msA * irA, kB = msB * irB;
        const double pA = (EA - kA * (MS * 0.5)) * (g - 1.0), pB = (EB - kB * (MS * 0.5)) * (g - 1.0);
        const double yA = pA * irA, yB = pB * irB;
        const double cA = sqrt(yA) * p.imach, cB = sqrt(yB) * p.imach;
        const double rhoMean = (rA + rB) * 0.5, pMean = (pA + pB) * 0.5, cMean = (cA + cB) * 0.5;
        const double vJ = unB - unA;
        const double pSraw = pMean - vJ * cMean * rhoMean * (0.5 * MS);
        const bool clamp = 0.0 > pSraw;
        const double pS = clamp ? 0.0 : pSraw;
        const bool qAact = pS > pA, qBact = pS > pB;
        const double ipA = qAact ? 1.0 / pA : 0.0, ipB = qBact ? 1.0 / pB : 0.0;
        const double qA = qAact ? sqrt(1.0 + (pS * ipA - 1.0) * G2) : 1.0;
        const double qB = qBact ? sqrt(1.0 + (pS * ipB - 1.0) * G2) : 1.0;
        const double sA = unA - cA * qA, sB = unB + cB * qB;
        const double CA = rA * (sA - unA), CB = rB * (sB - unB);
        const double Dd = CB - CA, iDd = 1.0 / Dd;
        const double S = (CB * unB - CA * unA + (pA - pB) * iMS) * iDd;
        const bool left = S > 0.0;
        const bool star = left ? (sA <= 0.0) : (sB >= 0.0);
        // ---- reverse: the upwind side's flux
        const double* Us = left ? UA : UB;
        const double r = Us[0], E = Us[D + 1], pp = left ? pA : pB, un = left ? unA : unB, s = left ? sA : sB;
        double rb = fb[0] * un, unb = fb[0] * r, Eb = fb[D + 1] * un, pb = fb[D + 1] * un, sb = 0.0, Sb = 0.0;
        double mb[D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            unb += fb[c + 1] * Us[c + 1];
            mb[c] = fb[c + 1] * un;
            pb += fb[c + 1] * n[c] * iMS;
        }
        unb += fb[D + 1] * (E + pp);
        if (star) {
            const double a = s - un, b = s - S, ia = 1.0 / a, ib = 1.0 / b, rr = a * ib, t = S - un;
            double rrb = fb[0] * s * r, tb = 0.0;
            sb += fb[0] * r * (rr - 1.0);
            rb += fb[0] * s * (rr - 1.0);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const double w = fb[c + 1], wb = w * s;
                sb += w * ((rr - 1.0) * Us[c + 1] + r * rr * t * n[c]);
                rrb += wb * (Us[c + 1] + r * t * n[c]);
                mb[c] += wb * (rr - 1.0);
                rb += wb * rr * t * n[c];
                tb += wb * r * rr * n[c];
            }
            const double factor = r * S * MS + pp * ia;
            const double modE = rr * (E + factor * t);
            sb += fb[D + 1] * (modE - E);
            const double mEb = fb[D + 1] * s;
            Eb += mEb * rr - fb[D + 1] * s;
            rrb += mEb * (E + factor * t);
            const double fab = mEb * rr * t;
            tb += mEb * rr * factor;
            rb += fab * S * MS;
            Sb += fab * r * MS;
            pb += fab * ia;
            const double ab = -fab * pp * ia * ia + rrb * ib;
            const double bb = -rrb * rr * ib;
            sb += ab + bb;
            unb -= ab + tb;
            Sb += tb - bb;
        }
        double rAb = 0.0, rBb = 0.0, EAb = 0.0, EBb = 0.0, pAb = 0.0, pBb = 0.0, unAb = 0.0, unBb = 0.0;
        double sAb = 0.0, sBb = 0.0, mAb[D], mBb[D];
#pragma unroll
        for (int c = 0; c < D; ++c) mAb[c] = mBb[c] = 0.0;
        if (left) {
            rAb = rb; EAb = Eb; pAb = pb; unAb = unb; sAb = sb;
#pragma unroll
            for (int c = 0; c < D; ++c) mAb[c] = mb[c];
        } else {
            rBb = rb; EBb = Eb; pBb = pb; unBb = unb; sBb = sb;
#pragma unroll
            for (int c = 0; c < D; ++c) mBb[c] = mb[c];
        }
        // ---- reverse: contact speed S = (CB unB - CA unA + (pA - pB)/MS) / (CB - CA)
        const double Nb = Sb * iDd, Ddb = -Sb * S * iDd;
        double CAb = -Ddb - Nb * unA, CBb = Ddb + Nb * unB;
        unBb += Nb * CB;
        unAb -= Nb * CA;
        pAb += Nb * iMS;
        pBb -= Nb * iMS;
        rAb += CAb * (sA - unA);
        sAb += CAb * rA;
        unAb -= CAb * rA;
        rBb += CBb * (sB - unB);
        sBb += CBb * rB;
        unBb -= CBb * rB;
        // wave speeds sA = unA - cA qA, sB = unB + cB qB
        unAb += sAb;
        unBb += sBb;
        double cAb = -sAb * qA, cBb = sBb * qB;
        const double qAb = -sAb * cA, qBb = sBb * cB;
        double pSb = 0.0;
        if (qAact) {
            const double zb = qAb * 0.5 / qA;
            pSb += zb * G2 * ipA;
            pAb -= zb * G2 * pS * ipA * ipA;
        }
        if (qBact) {
            const double zb = qBb * 0.5 / qB;
            pSb += zb * G2 * ipB;
            pBb -= zb * G2 * pS * ipB * ipB;
        }
        if (!clamp) {
            const double h = 0.5 * MS;
            pAb += 0.5 * pSb;
            pBb += 0.5 * pSb;
            const double vJb = -pSb * cMean * rhoMean * h;
            unBb += vJb;
            unAb -= vJb;
            const double cMb = -pSb * vJ * rhoMean * h;
            cAb += 0.5 * cMb;
            cBb += 0.5 * cMb;
            const double rMb = -pSb * vJ * cMean * h;
            rAb += 0.5 * rMb;
            rBb += 0.5 * rMb;
        }
        // ---- reverse: per-side primitives (c = sqrt(p/rho)/Ma, p, un); dc/dy = 1/(2 Ma^2 c)
        const double i2M2 = 0.5 * p.imach * p.imach;
        {
            const double ybA = cAb * i2M2 / cA;
            pAb += ybA * irA;
            rAb -= ybA * yA * irA;
            EAb += pAb * (g - 1.0);
            const double kbA = -pAb * (g - 1.0) * (MS * 0.5);
            const double msbA = kbA * irA;
            rAb -= kbA * kA * irA;
            const double unrbA = unAb * irA;
            rAb -= unAb * unA * irA;
            UAb[0] = rAb;
#pragma unroll
            for (int d = 0; d < D; ++d) UAb[d + 1] = mAb[d] + unrbA * n[d] + 2.0 * msbA * UA[d + 1];
            UAb[D + 1] = EAb;
        }
        {
            const double ybB = cBb * i2M2 / cB;
            pBb += ybB * irB;
            rBb -= ybB * yB * irB;
            EBb += pBb * (g - 1.0);
            const double kbB = -pBb * (g - 1.0) * (MS * 0.5);
            const double msbB = kbB * irB;
            rBb -= kbB * kB * irB;
            const double unrbB = unBb * irB;
            rBb -= unBb * unB * irB;
            UBb[0] = rBb;
#pragma unroll
            for (int d = 0; d < D; ++d) UBb[d + 1] = mBb[d] + unrbB * n[d] + 2.0 * msbB * UB[d + 1];
            UBb[D + 1] = EBb;
        }
    }
};

}  // namespace bosss
