// dg_slab_kernel.cuh -- register-blocked 3D DG kernel for systems (several fields).
//
// Same algorithm and results as dg_cell_kernel (NECQuadratureVolume / NECQuadratureEdge
// restated with sum factorisation, cell-centric faces), different work split:
//
//  * one thread per (cell, output field o, slab q). For the volume, slab q is the
//    z-node index: sum factorisation contracting z first keeps every later stage
//    inside the slab, so a thread interpolates u (and grad u) at the Q^2 nodes of its
//    slab from the field's Np coefficients entirely in registers, and projects the
//    slab's pointwise results back onto all Np test functions, again in registers.
//    For a face normal to d the slab is the node row along the face's second in-plane
//    direction. The Q partial residuals of a (cell, field) are summed once at the end;
//  * 1D table entries with compile-time indices are read from the kernel-parameter
//    constant bank (free FMA operands); the thread's own slab row lives in registers;
//  * shared memory only carries the node values between the contraction threads and
//    the pointwise threads (padded strides against bank conflicts).
#pragma once
#include <type_traits>

#include "dg_kernel.cuh"

namespace bosss {

// Row strides of the node blocks in shared memory: odd, so that the threads of a warp (one
// slab row each, cells S_CELL apart) spread their 8-byte accesses over all bank pairs; with
// Q odd the unpadded Q^2 / Q are odd already (an even stride left half the banks unused:
// 5.7 wavefronts per store in the k = 4 scalar VJP)
__host__ __device__ constexpr int slab_slv(int Q) { return (Q * Q) | 1; }
__host__ __device__ constexpr int slab_slf(int Q) { return Q | 1; }

// PASS: 0 = volume and face terms (runtime flags may skip either), 1 = volume terms only
// (compiled without the face passes: the volume pass of the face-once path)
template <class Phys, int K, int Q, int MODE, int PASS = 0>
struct SlabCfg {
    using B = Cfg<Phys, K, Q, MODE>;
    static constexpr int D = 3;
    static_assert(Phys::D == 3, "slab kernel is three-dimensional");
    static constexpr int NP = B::NP, NV = B::NV, NC = B::NC, NFI = B::NFI, NO = B::NO, NF1 = B::NF1;
    static constexpr int NPAIR = B::NPAIR, NS = B::NS;
    static constexpr bool VOL_OV = B::VOL_OV, VOL_OG = B::VOL_OG, FACE_OV = B::FACE_OV, FACE_OG = B::FACE_OG;
    // which interpolated groups need gradients: the state (and the JVP direction) only
    // if the forms read grad u; the VJP adjoint only where test-function gradients enter
    static constexpr bool G_STATE = Phys::GRAD_U;
    static constexpr bool G_SECOND_VOL = (MODE == MODE_VJP) ? Phys::VOL_G : Phys::GRAD_U;
    static constexpr bool G_SECOND_FACE = (MODE == MODE_VJP) ? Phys::FACE_G : Phys::GRAD_U;
    static constexpr int NCI0 = G_STATE ? 4 : 1;
    static constexpr int NCI1V = G_SECOND_VOL ? 4 : 1;
    static constexpr int NCI1F = G_SECOND_FACE ? 4 : 1;
    static constexpr int NCOV = (VOL_OV ? 1 : 0) + (VOL_OG ? 3 : 0);
    static constexpr int NCOF = (FACE_OV ? 1 : 0) + (FACE_OG ? 3 : 0);
    static constexpr int SLV = slab_slv(Q);        // padded volume slab
    static constexpr int FV = Q * SLV;             // one (field, comp) volume block
    static constexpr int SLF = slab_slf(Q);        // padded face row
    static constexpr int FF = Q * SLF;             // one (field, comp) face block
    // work split of a slab over SPLIT warp-uniform parts: volume rows qy = part mod SPLIT,
    // faces: part s handles the lower (s=0) / upper (s=1) face. Measured on B200 (Euler
    // k=3): the split pays for the register-heavy VJP (more resident warps), not for the
    // residual/JVP
#ifndef BOSSS_SLAB_SPLIT_VJP
#define BOSSS_SLAB_SPLIT_VJP 2
#endif
#ifndef BOSSS_SLAB_SPLIT_SCALAR
#define BOSSS_SLAB_SPLIT_SCALAR 2
#endif
    static constexpr int SPLIT = (Q < 3) ? 1
                                 : (MODE == MODE_VJP) ? BOSSS_SLAB_SPLIT_VJP
                                 : (Phys::NV == 1) ? BOSSS_SLAB_SPLIT_SCALAR : 1;
    static constexpr int TPC = NO * Q * SPLIT;     // threads per cell
    static constexpr int NODEV = (NV * NCI0 + NF1 * NCI1V) * FV;   // interpolated node values
    static constexpr int S_CIN = NFI * NP;
    // the pointwise outputs overwrite the node values in place: every node is read and
    // written by one thread (all its inputs before any output), and output comp c of field o
    // sits at block c*NO + o, so no node's inputs are overwritten by another node's outputs
    static constexpr int S_VOL = NODEV > NO * NCOV * FV ? NODEV : NO * NCOV * FV;
    static constexpr int TRB = (NV * NCI0 + NF1 * NCI1F) * FF;      // one (face, side) trace block
    static constexpr int S_FACE = 2 * 2 * TRB + 2 * NO * NCOF * FF;
    static constexpr int S_RED = NO * SPLIT * Q * NP;
    static constexpr int S_W0 = (PASS == 1 || S_VOL > S_FACE) ? S_VOL : S_FACE;
    static constexpr int S_WORK = S_W0 > S_RED ? S_W0 : S_RED;
    // one field (the scalar family): the per-cell stride is odd as well (the threads of a warp
    // span several cells); the multi-field tiles keep their measured layout
    static constexpr int S_CELL = (NV == 1) ? ((S_CIN + S_WORK) | 1) : S_CIN + S_WORK;
    static constexpr int BUDGET = 110 * 1024 / 8;
    static constexpr int CPB_SMEM = BUDGET / S_CELL;
    // threads per block target and minimum resident blocks per SM (register budget):
    // tuned on B200 for the Euler k=3 tile (profiles/)
#ifndef BOSSS_SLAB_THREADS
#define BOSSS_SLAB_THREADS 256
#endif
#ifndef BOSSS_SLAB_THREADS_VJP
#define BOSSS_SLAB_THREADS_VJP 128
#endif
    // residual / JVP: resident blocks per SM (residual k <= 2: 3, measured as for the VJP)
#ifdef BOSSS_SLAB_MINB
    static constexpr int MINB_FWD = BOSSS_SLAB_MINB;
#else
    static constexpr int MINB_FWD = (MODE == MODE_RES && K <= 2) ? 3 : 2;
#endif
    // VJP: resident blocks per SM by degree, measured on B200 (Euler, 32^3, k = 1..4): more
    // resident warps beat the register spills this forces (k=3: 8 -> 16 warps, 1.27 -> 0.82 ms)
#ifdef BOSSS_SLAB_MINB_VJP
    static constexpr int MINB_VJP = BOSSS_SLAB_MINB_VJP;
#else
    static constexpr int MINB_VJP = K <= 1 ? 5 : (K <= 3 ? 4 : 3);
#endif
    static constexpr int CPB_THR = ((MODE == MODE_VJP) ? BOSSS_SLAB_THREADS_VJP : BOSSS_SLAB_THREADS) / TPC;
    static constexpr int MINB_REQ = (MODE == MODE_VJP) ? MINB_VJP : MINB_FWD;
    static constexpr int CPB_MAX = (CPB_SMEM < CPB_THR ? CPB_SMEM : CPB_THR) < 1 ? 1
                                   : (CPB_SMEM < CPB_THR ? CPB_SMEM : CPB_THR);
    static constexpr int CPB = CPB_MAX;
    static constexpr int HALF = CPB * NO * Q;                 // threads of one part
    // with SPLIT > 1 each part is padded to whole warps, so `part` is warp-uniform
    static constexpr int HALFP = (SPLIT > 1) ? (HALF + 31) / 32 * 32 : HALF;
    static constexpr int NT = SPLIT * HALFP;
    static constexpr size_t SMEM_BYTES = (size_t)CPB * S_CELL * 8;
    // resident blocks the shared memory admits (228 KB per SM, 1 KB reserved per block): asking
    // the register allocator for more than these only forces spills (the scalar family's tiles
    // are shared-memory bound at 2 blocks: k=4 VJP 168 registers with spills under a 3-block cap)
    static constexpr int BLK_SMEM = (int)(233472 / (SMEM_BYTES + 1024)) < 1 ? 1 : (int)(233472 / (SMEM_BYTES + 1024));
    static constexpr int MINB = MINB_REQ < BLK_SMEM ? MINB_REQ : BLK_SMEM;
    // offset of field f's first comp block
    __host__ __device__ static constexpr int vnode(int f) { return f < NV ? f * NCI0 * FV : (NV * NCI0 + (f - NV) * NCI1V) * FV; }
    __host__ __device__ static constexpr int fnode(int f) { return f < NV ? f * NCI0 * FF : (NV * NCI0 + (f - NV) * NCI1F) * FF; }
};

template <int DIR> struct FaceDirs {
    static constexpr int t1 = (DIR == 0) ? 1 : 0;
    static constexpr int t2 = (DIR == 2) ? 1 : 2;
};

template <int DIR>
__host__ __device__ constexpr int mode_dpr(int m, int p, int r) {
    return DIR == 0 ? mode3(m, p, r) : (DIR == 1 ? mode3(p, m, r) : mode3(p, r, m));
}

// ------------------------------------------------------------------ pointwise helpers
// Volume node: in(f, comp) reads interpolated fields, out(o, c, v) stores projected
// coefficients (c = 0: test function, 1+d: gradient d) already scaled by `fac` and 2/h.
template <class Phys, int MODE, bool GS, bool G2, bool OV, bool OG, class In, class Out>
__device__ __forceinline__ void volume_point(const PhysParams& ph, const double* x, double fac,
                                             const double* twoh, In in, Out out) {
    constexpr int D = Phys::D, NV = Phys::NV, NC = Phys::NC;
    if constexpr (MODE == MODE_RES) {
        double U[NV], Gr[NV][D], fV[NC], fG[NC][D];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            U[i] = in(i, 0);
#pragma unroll
            for (int d = 0; d < D; ++d) Gr[i][d] = GS ? in(i, 1 + d) : 0.0;
        }
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            fV[e] = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) fG[e][d] = 0.0;
        }
        Phys::volume(ph, U, Gr, x, fV, fG);
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            if (OV) out(e, 0, fV[e] * fac);
            if (OG)
#pragma unroll
                for (int d = 0; d < D; ++d) out(e, 1 + d, fG[e][d] * fac * twoh[d]);
        }
    } else if constexpr (MODE == MODE_JVP) {
        using T = DualN<1>;
        T U[NV], Gr[NV][D], fV[NC], fG[NC][D];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            U[i].v = in(i, 0);
            U[i].d[0] = in(NV + i, 0);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                Gr[i][d].v = GS ? in(i, 1 + d) : 0.0;
                Gr[i][d].d[0] = (GS && G2) ? in(NV + i, 1 + d) : 0.0;
            }
        }
        Phys::volume(ph, U, Gr, x, fV, fG);
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            if (OV) out(e, 0, fV[e].d[0] * fac);
            if (OG)
#pragma unroll
                for (int d = 0; d < D; ++d) out(e, 1 + d, fG[e][d].d[0] * fac * twoh[d]);
        }
    } else if constexpr (Phys::ADJOINT) {
        // reverse mode: gradient of sum fG . grad w with respect to the node state
        double U[NV], Gw[NC][D], Ub[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) U[i] = in(i, 0);
#pragma unroll
        for (int e = 0; e < NC; ++e)
#pragma unroll
            for (int d = 0; d < D; ++d) Gw[e][d] = G2 ? in(NV + e, 1 + d) : 0.0;
        Phys::volume_adj(ph, U, Gw, Ub);
#pragma unroll
        for (int i = 0; i < NV; ++i) out(i, 0, Ub[i] * fac);
    } else {
        constexpr int NS = NV * (Phys::GRAD_U ? 1 + D : 1);
        using T = DualN<NS>;
        T U[NV], Gr[NV][D], fV[NC], fG[NC][D];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            U[i] = T(in(i, 0));
            U[i].d[Phys::GRAD_U ? i * (1 + D) : i] = 1.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                Gr[i][d] = T(GS ? in(i, 1 + d) : 0.0);
                if (Phys::GRAD_U) Gr[i][d].d[i * (1 + D) + 1 + d] = 1.0;
            }
        }
        Phys::volume(ph, U, Gr, x, fV, fG);
        T phi(0.0);
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            if (Phys::VOL_V) phi += fV[e] * in(NV + e, 0);
            if (Phys::VOL_G && G2)
#pragma unroll
                for (int d = 0; d < D; ++d) phi += fG[e][d] * in(NV + e, 1 + d);
        }
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            out(i, 0, phi.d[Phys::GRAD_U ? i * (1 + D) : i] * fac);
            if (Phys::GRAD_U)
#pragma unroll
                for (int d = 0; d < D; ++d) out(i, 1 + d, phi.d[i * (1 + D) + 1 + d] * fac * twoh[d]);
        }
    }
}

// Face node: inA/inB read the traces of the IN (lower) and OUT (upper) cell,
// out(o, c, v) stores the own side's coefficients.
template <class Phys, int MODE, bool GS, bool G2, bool OV, bool OG, class InA, class InB, class Out>
__device__ __forceinline__ void face_point(const PhysParams& ph, bool inner, bool selfA, double pnlty,
                                           const double* nrm, const double* x, double fac, const double* twoh,
                                           InA inA, InB inB, Out out) {
    constexpr int D = Phys::D, NV = Phys::NV, NC = Phys::NC;
    if constexpr (MODE == MODE_RES) {
        double UA[NV], GA[NV][D], UB[NV], GB[NV][D], gA[NC], GAv[NC][D], gB[NC], GBv[NC][D];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            UA[i] = inA(i, 0);
            UB[i] = inner ? inB(i, 0) : 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                GA[i][d] = GS ? inA(i, 1 + d) : 0.0;
                GB[i][d] = (GS && inner) ? inB(i, 1 + d) : 0.0;
            }
        }
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            gA[e] = gB[e] = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) GAv[e][d] = GBv[e][d] = 0.0;
        }
        if (inner) Phys::inner(ph, pnlty, UA, GA, UB, GB, nrm, x, gA, GAv, gB, GBv);
        else Phys::boundary(ph, pnlty, UA, GA, nrm, x, nullptr, 0, gA, GAv);
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            if (OV) out(e, 0, (selfA ? gA[e] : gB[e]) * fac);
            if (OG)
#pragma unroll
                for (int d = 0; d < D; ++d) out(e, 1 + d, (selfA ? GAv[e][d] : GBv[e][d]) * fac * twoh[d]);
        }
    } else if constexpr (MODE == MODE_JVP) {
        using T = DualN<1>;
        T UA[NV], GA[NV][D], UB[NV], GB[NV][D], gA[NC], GAv[NC][D], gB[NC], GBv[NC][D];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            UA[i].v = inA(i, 0);
            UA[i].d[0] = inA(NV + i, 0);
            UB[i].v = inner ? inB(i, 0) : 0.0;
            UB[i].d[0] = inner ? inB(NV + i, 0) : 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                GA[i][d].v = GS ? inA(i, 1 + d) : 0.0;
                GA[i][d].d[0] = (GS && G2) ? inA(NV + i, 1 + d) : 0.0;
                GB[i][d].v = (GS && inner) ? inB(i, 1 + d) : 0.0;
                GB[i][d].d[0] = (GS && G2 && inner) ? inB(NV + i, 1 + d) : 0.0;
            }
        }
        if (inner) Phys::inner(ph, pnlty, UA, GA, UB, GB, nrm, x, gA, GAv, gB, GBv);
        else Phys::boundary(ph, pnlty, UA, GA, nrm, x, nullptr, 0, gA, GAv);
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            if (OV) out(e, 0, (selfA ? gA[e].d[0] : gB[e].d[0]) * fac);
            if (OG)
#pragma unroll
                for (int d = 0; d < D; ++d)
                    out(e, 1 + d, (selfA ? GAv[e][d].d[0] : GBv[e][d].d[0]) * fac * twoh[d]);
        }
    } else if constexpr (Phys::ADJOINT) {
        // reverse mode: gradient of sum_e f_e (w_IN,e - w_OUT,e) with respect to the own trace
        // (the adjoint physics has no boundary terms: its grids are periodic)
        if (inner) {
            double UA[NV], UB[NV], fb[NC], UAb[NV], UBb[NV];
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                UA[i] = inA(i, 0);
                UB[i] = inB(i, 0);
            }
#pragma unroll
            for (int e = 0; e < NC; ++e) fb[e] = inA(NV + e, 0) - inB(NV + e, 0);
            Phys::inner_adj(ph, UA, UB, nrm, fb, UAb, UBb);
#pragma unroll
            for (int i = 0; i < NV; ++i) out(i, 0, (selfA ? UAb[i] : UBb[i]) * fac);
        } else {
#pragma unroll
            for (int i = 0; i < NV; ++i) out(i, 0, 0.0);
        }
    } else {
        constexpr int NS = NV * (Phys::GRAD_U ? 1 + D : 1);
        using T = DualN<NS>;
        T UA[NV], GA[NV][D], UB[NV], GB[NV][D], gA[NC], GAv[NC][D], gB[NC], GBv[NC][D];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            UA[i] = T(inA(i, 0));
            UB[i] = T(inner ? inB(i, 0) : 0.0);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                GA[i][d] = T(GS ? inA(i, 1 + d) : 0.0);
                GB[i][d] = T((GS && inner) ? inB(i, 1 + d) : 0.0);
            }
            (selfA ? UA[i] : UB[i]).d[Phys::GRAD_U ? i * (1 + D) : i] = 1.0;
            if (Phys::GRAD_U)
#pragma unroll
                for (int d = 0; d < D; ++d) (selfA ? GA[i][d] : GB[i][d]).d[i * (1 + D) + 1 + d] = 1.0;
        }
        if (inner) Phys::inner(ph, pnlty, UA, GA, UB, GB, nrm, x, gA, GAv, gB, GBv);
        else Phys::boundary(ph, pnlty, UA, GA, nrm, x, nullptr, 0, gA, GAv);
        T phi(0.0);
#pragma unroll
        for (int e = 0; e < NC; ++e) {
            const int fe = NV + e;
            if (Phys::FACE_V) {
                phi += gA[e] * inA(fe, 0);
                if (inner) phi += gB[e] * inB(fe, 0);
            }
            if (Phys::FACE_G && G2)
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    phi += GAv[e][d] * inA(fe, 1 + d);
                    if (inner) phi += GBv[e][d] * inB(fe, 1 + d);
                }
        }
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            out(i, 0, phi.d[Phys::GRAD_U ? i * (1 + D) : i] * fac);
            if (Phys::GRAD_U)
#pragma unroll
                for (int d = 0; d < D; ++d) out(i, 1 + d, phi.d[i * (1 + D) + 1 + d] * fac * twoh[d]);
        }
    }
}

// ------------------------------------------------------------------ contraction helpers
// interpolation of one field at the slab qz = q (Q*Q nodes), into node block `nb`
template <int K, int Q, bool GRAD, int PART, int SPLIT>
__device__ __forceinline__ void slab_interp(const Tables1D& T, const double* cf, const double* Az, const double* dAz,
                                            int q, double scaling, const double* twoh, double* nb) {
    constexpr int NPAIR = (K + 1) * (K + 2) / 2;
    constexpr int SLV = slab_slv(Q), FV = Q * SLV;
    double T1[NPAIR], T1z[NPAIR];
#pragma unroll
    for (int a = 0; a <= K; ++a)
#pragma unroll
        for (int b = 0; b <= K - a; ++b) {
            double s = 0.0, sz = 0.0;
#pragma unroll
            for (int c = 0; c <= K - a - b; ++c) {
                const double v = cf[mode3(a, b, c)];
                s += v * Az[c];
                if (GRAD) sz += v * dAz[c];
            }
            T1[pair_index(K, a, b)] = s;
            T1z[pair_index(K, a, b)] = sz;
        }
    double* base = nb + q * SLV;
#pragma unroll
    for (int qy = PART; qy < Q; qy += SPLIT) {
        double T2[K + 1], T2y[K + 1], T2z[K + 1];
#pragma unroll
        for (int a = 0; a <= K; ++a) {
            double s = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
            for (int b = 0; b <= K - a; ++b) {
                const double v = T1[pair_index(K, a, b)];
                s += v * T.A[qy][b];
                if (GRAD) {
                    sy += v * T.dA[qy][b];
                    sz += T1z[pair_index(K, a, b)] * T.A[qy][b];
                }
            }
            T2[a] = s;
            T2y[a] = sy;
            T2z[a] = sz;
        }
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
            double u = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
#pragma unroll
            for (int a = 0; a <= K; ++a) {
                u += T2[a] * T.A[qx][a];
                if (GRAD) {
                    ux += T2[a] * T.dA[qx][a];
                    uy += T2y[a] * T.A[qx][a];
                    uz += T2z[a] * T.A[qx][a];
                }
            }
            base[qy * Q + qx] = u * scaling;
            if (GRAD) {
                base[FV + qy * Q + qx] = ux * scaling * twoh[0];
                base[2 * FV + qy * Q + qx] = uy * scaling * twoh[1];
                base[3 * FV + qy * Q + qx] = uz * scaling * twoh[2];
            }
        }
    }
}

// projection of the slab qz = q of one output field (block `ob`, comps CS doubles apart) into R[NP]
template <int K, int Q, bool OV, bool OG, int PART, int SPLIT, int CS>
__device__ __forceinline__ void slab_project(const Tables1D& T, const double* ob, const double* Az, const double* dAz,
                                             int q, double* R) {
    constexpr int NPAIR = (K + 1) * (K + 2) / 2;
    constexpr int SLV = slab_slv(Q), FV = Q * SLV;
    constexpr int G0 = OV ? 1 : 0;
    double P2[NPAIR], P2z[NPAIR];
#pragma unroll
    for (int i = 0; i < NPAIR; ++i) P2[i] = P2z[i] = 0.0;
    const double* base = ob + q * SLV;
#pragma unroll
    for (int qy = PART; qy < Q; qy += SPLIT) {
        double P[K + 1], Py[K + 1], Pz[K + 1];
#pragma unroll
        for (int a = 0; a <= K; ++a) P[a] = Py[a] = Pz[a] = 0.0;
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
            const int n = qy * Q + qx;
            const double s = OV ? base[n] : 0.0;
            const double gx = OG ? base[G0 * CS + n] : 0.0;
            const double gy = OG ? base[(G0 + 1) * CS + n] : 0.0;
            const double gz = OG ? base[(G0 + 2) * CS + n] : 0.0;
#pragma unroll
            for (int a = 0; a <= K; ++a) {
                P[a] += s * T.A[qx][a] + gx * T.dA[qx][a];
                Py[a] += gy * T.A[qx][a];
                Pz[a] += gz * T.A[qx][a];
            }
        }
#pragma unroll
        for (int a = 0; a <= K; ++a)
#pragma unroll
            for (int b = 0; b <= K - a; ++b) {
                P2[pair_index(K, a, b)] += P[a] * T.A[qy][b] + Py[a] * T.dA[qy][b];
                P2z[pair_index(K, a, b)] += Pz[a] * T.A[qy][b];
            }
    }
#pragma unroll
    for (int a = 0; a <= K; ++a)
#pragma unroll
        for (int b = 0; b <= K - a; ++b)
#pragma unroll
            for (int c = 0; c <= K - a - b; ++c)
                R[mode3(a, b, c)] += P2[pair_index(K, a, b)] * Az[c] + P2z[pair_index(K, a, b)] * dAz[c];
}

// trace of one field at face DIR, own face side fs (0: xi_d = -1, 1: +1), row q2 = q
template <int DIR, int K, int Q, bool GRAD>
__device__ __forceinline__ void face_interp(const Tables1D& T, const double* cf, int fs, const double* A2,
                                            const double* dA2, double scaling, const double* twoh, double* tb) {
    constexpr int t1 = FaceDirs<DIR>::t1, t2 = FaceDirs<DIR>::t2;
    constexpr int SLF = slab_slf(Q), FF = Q * SLF;
    double Tv[K + 1], Tn[K + 1], Tt2[K + 1];
#pragma unroll
    for (int p = 0; p <= K; ++p) {
        double s0 = 0.0, sn = 0.0, st = 0.0;
#pragma unroll
        for (int r = 0; r <= K - p; ++r) {
            double S = 0.0, Sn = 0.0;
#pragma unroll
            for (int m = 0; m <= K - p - r; ++m) {
                const double v = cf[mode_dpr<DIR>(m, p, r)];
                S += v * (fs ? T.e[1][m] : T.e[0][m]);
                if (GRAD) Sn += v * (fs ? T.de[1][m] : T.de[0][m]);
            }
            s0 += S * A2[r];
            if (GRAD) {
                sn += Sn * A2[r];
                st += S * dA2[r];
            }
        }
        Tv[p] = s0;
        Tn[p] = sn;
        Tt2[p] = st;
    }
#pragma unroll
    for (int q1 = 0; q1 < Q; ++q1) {
        double u = 0.0, u1 = 0.0, u2 = 0.0, un = 0.0;
#pragma unroll
        for (int p = 0; p <= K; ++p) {
            u += Tv[p] * T.A[q1][p];
            if (GRAD) {
                u1 += Tv[p] * T.dA[q1][p];
                u2 += Tt2[p] * T.A[q1][p];
                un += Tn[p] * T.A[q1][p];
            }
        }
        tb[q1] = u * scaling;
        if (GRAD) {
            tb[(1 + DIR) * FF + q1] = un * scaling * twoh[DIR];
            tb[(1 + t1) * FF + q1] = u1 * scaling * twoh[t1];
            tb[(1 + t2) * FF + q1] = u2 * scaling * twoh[t2];
        }
    }
}

template <int DIR, int K, int Q, bool OV, bool OG>
__device__ __forceinline__ void face_project(const Tables1D& T, const double* ob, int fs, const double* A2,
                                             const double* dA2, double* R) {
    constexpr int t1 = FaceDirs<DIR>::t1, t2 = FaceDirs<DIR>::t2;
    constexpr int SLF = slab_slf(Q), FF = Q * SLF;
    constexpr int G0 = OV ? 1 : 0;
    double P[K + 1], Pn[K + 1], Pt2[K + 1];
#pragma unroll
    for (int p = 0; p <= K; ++p) P[p] = Pn[p] = Pt2[p] = 0.0;
#pragma unroll
    for (int q1 = 0; q1 < Q; ++q1) {
        const double g = OV ? ob[q1] : 0.0;
        const double gn = OG ? ob[(G0 + DIR) * FF + q1] : 0.0;
        const double g1 = OG ? ob[(G0 + t1) * FF + q1] : 0.0;
        const double g2 = OG ? ob[(G0 + t2) * FF + q1] : 0.0;
#pragma unroll
        for (int p = 0; p <= K; ++p) {
            P[p] += g * T.A[q1][p] + g1 * T.dA[q1][p];
            Pn[p] += gn * T.A[q1][p];
            Pt2[p] += g2 * T.A[q1][p];
        }
    }
#pragma unroll
    for (int p = 0; p <= K; ++p)
#pragma unroll
        for (int r = 0; r <= K - p; ++r) {
            const double w0 = P[p] * A2[r] + Pt2[p] * dA2[r];
            const double wn = Pn[p] * A2[r];
#pragma unroll
            for (int m = 0; m <= K - p - r; ++m)
                R[mode_dpr<DIR>(m, p, r)] += w0 * (fs ? T.e[1][m] : T.e[0][m]) + wn * (fs ? T.de[1][m] : T.de[0][m]);
        }
}

// ------------------------------------------------------------------ the kernel
template <class Phys, int K, int Q, int MODE, int PART>
__device__ __forceinline__ void slab_volume_interp(const EvalArgs& args, const Tables1D& T, const double* cin, double* wk,
                                                   int o, int q,
                                                   const double* Aq, const double* dAq) {
    using C = SlabCfg<Phys, K, Q, MODE>;
    constexpr int NP = C::NP;
    for (int f = o; f < C::NFI; f += C::NO) {
        double cf[NP];
#pragma unroll
        for (int n = 0; n < NP; ++n) cf[n] = cin[f * NP + n];
        double* nb = wk + C::vnode(f);
        if (f < C::NV) slab_interp<K, Q, C::G_STATE, PART, C::SPLIT>(T, cf, Aq, dAq, q, args.g.scaling, args.g.twoh, nb);
        else slab_interp<K, Q, C::G_SECOND_VOL, PART, C::SPLIT>(T, cf, Aq, dAq, q, args.g.scaling, args.g.twoh, nb);
    }
}

// traces of all interpolated fields at face (DIR, s): own (side 0) and neighbour (side 1)
template <class Phys, int K, int Q, int MODE, int DIR, int S>
__device__ __forceinline__ void slab_face_traces(const EvalArgs& args, const Tables1D& T, const double* cin, double* wk,
                                                 int o, int q,
                                                 const int* ijk, const double* Aq, const double* dAq) {
    using C = SlabCfg<Phys, K, Q, MODE>;
    constexpr int NP = C::NP, NV = C::NV, SLF = C::SLF;
    const long long nb = neighbour(args.g, ijk, DIR, S);
    constexpr bool GG = C::G_STATE || C::G_SECOND_FACE;
    for (int f = o; f < C::NFI; f += C::NO) {
        const bool fg = f < NV ? C::G_STATE : C::G_SECOND_FACE;
        {   // own cell
            double cf[NP];
#pragma unroll
            for (int n = 0; n < NP; ++n) cf[n] = cin[f * NP + n];
            double* t0 = wk + (S * 2 + 0) * C::TRB + C::fnode(f) + q * SLF;
            if (fg) face_interp<DIR, K, Q, GG>(T, cf, S, Aq, dAq, args.g.scaling, args.g.twoh, t0);
            else face_interp<DIR, K, Q, false>(T, cf, S, Aq, dAq, args.g.scaling, args.g.twoh, t0);
        }
        {   // neighbour across the face
            double cn[NP];
            if (nb >= 0) {
                const double* src = (f < NV) ? args.U + nb * (NV * NP) + f * NP : args.V + nb * (C::NF1 * NP) + (f - NV) * NP;
#pragma unroll
                for (int n = 0; n < NP; ++n) cn[n] = __ldg(src + n);
            } else {
#pragma unroll
                for (int n = 0; n < NP; ++n) cn[n] = 0.0;
            }
            double* t1 = wk + (S * 2 + 1) * C::TRB + C::fnode(f) + q * SLF;
            if (fg) face_interp<DIR, K, Q, GG>(T, cn, 1 - S, Aq, dAq, args.g.scaling, args.g.twoh, t1);
            else face_interp<DIR, K, Q, false>(T, cn, 1 - S, Aq, dAq, args.g.scaling, args.g.twoh, t1);
        }
    }
}

// Evaluates the tile of cells [c0, c0 + CPB) (clipped to args.cend); the first C::NT threads
// of the CTA do the work, any further threads only take part in the barriers (the batched
// persistent kernel runs tiles of several degrees in CTAs of one size). T: the 1D tables,
// passed apart from args so that a caller can keep them in the kernel-parameter bank.
template <class Phys, int K, int Q, int MODE, int PASS = 0>
__device__ __forceinline__ void slab_tile(const EvalArgs& args, const Tables1D& T, long long c0, double* smem) {
    using C = SlabCfg<Phys, K, Q, MODE, PASS>;
    constexpr int NP = C::NP, NV = C::NV, NO = C::NO, CPB = C::CPB, NT = C::NT, SPLIT = C::SPLIT;
    constexpr int SLV = C::SLV, FV = C::FV, SLF = C::SLF, FF = C::FF, QF = Q * Q;
    const GridConst& g = args.g;
    const int tid = threadIdx.x;
    const int tt = tid < NT ? tid : (1 << 30);   // start of the strided loops (threads beyond NT: none)
    const int ncell = (int)((args.cend - c0) < CPB ? (args.cend - c0) : CPB);
    // own (part, cell, output field, slab); part is warp-uniform (parts padded to warps)
    const int part = tid / C::HALFP, r0 = tid % C::HALFP;
    const int q = r0 % Q, o = (r0 / Q) % NO, cl = (r0 < C::HALF) ? r0 / (Q * NO) : CPB;
    const bool active = tid < NT && cl < ncell;
    auto CIN = [&](int c) { return smem + (size_t)c * C::S_CELL; };
    auto WK = [&](int c) { return smem + (size_t)c * C::S_CELL + C::S_CIN; };

    constexpr int NVPC = NV * NP;
    constexpr int N1PC = C::NF1 * NP;
    for (int i = tt; i < ncell * NVPC; i += NT) CIN(i / NVPC)[i % NVPC] = args.U[c0 * NVPC + i];
    if constexpr (C::NF1 > 0)
        for (int i = tt; i < ncell * N1PC; i += NT) CIN(i / N1PC)[NVPC + i % N1PC] = args.V[c0 * N1PC + i];

    double Aq[K + 1], dAq[K + 1];
#pragma unroll
    for (int a = 0; a <= K; ++a) {
        Aq[a] = T.A[q][a];
        dAq[a] = T.dA[q][a];
    }
    double R[NP];
#pragma unroll
    for (int n = 0; n < NP; ++n) R[n] = 0.0;
    int ijk[3];
    cell_ijk(g, c0 + (active ? cl : 0), ijk);
    __syncthreads();

    // ---------------------------------------------------------- volume
    constexpr int OUT0 = 0;
    if (!args.faces_only) {   // uniform over the CTA
    if (active) {
        if (part == 0) slab_volume_interp<Phys, K, Q, MODE, 0>(args, T, CIN(cl), WK(cl), o, q, Aq, dAq);
        else if constexpr (SPLIT > 1) slab_volume_interp<Phys, K, Q, MODE, 1>(args, T, CIN(cl), WK(cl), o, q, Aq, dAq);
    }
    __syncthreads();
    for (int it = tt; it < CPB * Q * Q * Q; it += NT) {
        const int n = it % (Q * Q * Q), c = it / (Q * Q * Q);
        if (c >= ncell) continue;
        const int qx = n % Q, qy = (n / Q) % Q, qz = n / (Q * Q);
        const int off = qz * SLV + qy * Q + qx;
        int cijk[3];
        cell_ijk(g, c0 + c, cijk);
        double x[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = g.lo[d] + (cijk[d] + g.goff[d] + 0.5) * g.h[d];
        x[0] += 0.5 * g.h[0] * T.xq[qx];
        x[1] += 0.5 * g.h[1] * T.xq[qy];
        x[2] += 0.5 * g.h[2] * T.xq[qz];
        const double fac = T.w[qx] * T.w[qy] * T.w[qz] * g.detJ * g.scaling;
        const double* nb = WK(c);
        double* ob = WK(c) + OUT0;
        if (args.vol_flag && args.vol_flag[c0 + c] != 1) {   // XDG species mask: term skipped
            for (int e = 0; e < C::NCOV * NO; ++e) ob[e * FV + off] = 0.0;
            continue;
        }
        volume_point<Phys, MODE, C::G_STATE, C::G_SECOND_VOL, C::VOL_OV, C::VOL_OG>(
            args.ph, x, fac, g.twoh, [&](int f, int comp) { return nb[C::vnode(f) + comp * FV + off]; },
            [&](int oo, int comp, double v) {
                const int cc = C::VOL_OV ? comp : comp - 1;
                ob[(cc * NO + oo) * FV + off] = v;
            });
    }
    __syncthreads();
    if (active) {
        const double* ob = WK(cl) + OUT0 + o * FV;
        if (part == 0) slab_project<K, Q, C::VOL_OV, C::VOL_OG, 0, SPLIT, NO * FV>(T, ob, Aq, dAq, q, R);
        else if constexpr (SPLIT > 1)
            slab_project<K, Q, C::VOL_OV, C::VOL_OG, 1, SPLIT, NO * FV>(T, ob, Aq, dAq, q, R);
    }
    __syncthreads();
    }

    // ---------------------------------------------------------- faces
    auto face_pass = [&](auto dirc) {
        constexpr int DIR = decltype(dirc)::value;
        constexpr int t1 = FaceDirs<DIR>::t1, t2 = FaceDirs<DIR>::t2;
        constexpr int OUTF0 = 2 * 2 * C::TRB;
        if (active) {
            if constexpr (SPLIT > 1) {
                if (part == 0) slab_face_traces<Phys, K, Q, MODE, DIR, 0>(args, T, CIN(cl), WK(cl), o, q, ijk, Aq, dAq);
                else slab_face_traces<Phys, K, Q, MODE, DIR, 1>(args, T, CIN(cl), WK(cl), o, q, ijk, Aq, dAq);
            } else {
                slab_face_traces<Phys, K, Q, MODE, DIR, 0>(args, T, CIN(cl), WK(cl), o, q, ijk, Aq, dAq);
                slab_face_traces<Phys, K, Q, MODE, DIR, 1>(args, T, CIN(cl), WK(cl), o, q, ijk, Aq, dAq);
            }
        }
        __syncthreads();
        for (int it = tt; it < CPB * 2 * QF; it += NT) {
            const int qf = it % QF, s = (it / QF) % 2, c = it / (2 * QF);
            if (c >= ncell) continue;
            const int q1 = qf % Q, q2 = qf / Q;
            const int off = q2 * SLF + q1;
            if (args.face_flag && args.face_flag[(c0 + c) * 6 + 2 * DIR + s] != 1) {   // XDG species mask
                double* ob = WK(c) + OUTF0 + s * NO * C::NCOF * FF;
                for (int e = 0; e < NO * C::NCOF; ++e) ob[e * FF + off] = 0.0;
                continue;
            }
            int cijk[3];
            cell_ijk(g, c0 + c, cijk);
            const long long nbc = neighbour(g, cijk, DIR, s);
            const bool inner = nbc >= 0;
            double x[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) x[d] = g.lo[d] + (cijk[d] + g.goff[d] + 0.5) * g.h[d];
            x[DIR] += (s ? 0.5 : -0.5) * g.h[DIR];
            x[t1] += 0.5 * g.h[t1] * T.xq[q1];
            x[t2] += 0.5 * g.h[t2] * T.xq[q2];
            double nrm[3] = {0.0, 0.0, 0.0};
            nrm[DIR] = inner ? 1.0 : (s ? 1.0 : -1.0);
            double pnlty;
            if (inner) {
                int ijk2[3] = {cijk[0], cijk[1], cijk[2]};
                ijk2[DIR] = (int)((nbc / g.stride[DIR]) % g.n[DIR]);
                pnlty = args.ph.pen * fmax(penalty_size(args.cell_pf, g, cijk), penalty_size(args.cell_pf, g, ijk2));
            } else {
                pnlty = Phys::BND_PEN * args.ph.pen * penalty_size(args.cell_pf, g, cijk);
            }
            const bool selfA = !inner || s == 1;
            const double* trOwn = WK(c) + (s * 2 + 0) * C::TRB;
            const double* trNb = WK(c) + (s * 2 + 1) * C::TRB;
            const double* trA = selfA ? trOwn : trNb;
            const double* trB = selfA ? trNb : trOwn;
            double* ob = WK(c) + OUTF0 + s * NO * C::NCOF * FF;
            const double fac = T.w[q1] * T.w[q2] * g.faceSG[DIR] * g.scaling;
            face_point<Phys, MODE, C::G_STATE, C::G_SECOND_FACE, C::FACE_OV, C::FACE_OG>(
                args.ph, inner, selfA, pnlty, nrm, x, fac, g.twoh,
                [&](int f, int comp) { return trA[C::fnode(f) + comp * FF + off]; },
                [&](int f, int comp) { return trB[C::fnode(f) + comp * FF + off]; },
                [&](int oo, int comp, double v) {
                    const int cc = C::FACE_OV ? comp : comp - 1;
                    ob[(oo * C::NCOF + cc) * FF + off] = v;
                });
        }
        __syncthreads();
        if (active) {
            auto proj = [&](auto sc) {
                constexpr int S = decltype(sc)::value;
                face_project<DIR, K, Q, C::FACE_OV, C::FACE_OG>(
                    T, WK(cl) + OUTF0 + (S * NO + o) * C::NCOF * FF + q * SLF, S, Aq, dAq, R);
            };
            if constexpr (SPLIT > 1) {
                if (part == 0) proj(std::integral_constant<int, 0>{});
                else proj(std::integral_constant<int, 1>{});
            } else {
                proj(std::integral_constant<int, 0>{});
                proj(std::integral_constant<int, 1>{});
            }
        }
        __syncthreads();
    };
    if constexpr (PASS == 0) {
        if (!args.volume_only) {   // uniform over the CTA
            face_pass(std::integral_constant<int, 0>{});
            face_pass(std::integral_constant<int, 1>{});
            face_pass(std::integral_constant<int, 2>{});
        }
    }

    // ---------------------------------------------------------- reduce partials and store
    if (active) {
        double* red = WK(cl) + ((o * SPLIT + part) * Q + q) * NP;
#pragma unroll
        for (int n = 0; n < NP; ++n) red[n] = R[n];
    }
    __syncthreads();
    for (int it = tt; it < ncell * NO * NP; it += NT) {
        const int n = it % NP, oo = (it / NP) % NO, c = it / (NP * NO);
        double v = 0.0;
#pragma unroll
        for (int pq = 0; pq < SPLIT * Q; ++pq) v += WK(c)[(oo * SPLIT * Q + pq) * NP + n];
        const long long gi = c0 * (long long)(NO * NP) + it;
        if constexpr (MODE == MODE_RES) {
            args.out[gi] = (args.beta == 0.0) ? args.alpha * v : args.beta * args.out[gi] + args.alpha * v;
        } else {
            args.out[gi] = v;
        }
    }
}

template <class Phys, int K, int Q, int MODE, int PASS = 0>
__global__ void __launch_bounds__(SlabCfg<Phys, K, Q, MODE, PASS>::NT, SlabCfg<Phys, K, Q, MODE, PASS>::MINB)
dg_slab_kernel(const __grid_constant__ EvalArgs args) {
    extern __shared__ double smem[];
    slab_tile<Phys, K, Q, MODE, PASS>(args, args.tab,
                                      args.cbeg + (long long)blockIdx.x * SlabCfg<Phys, K, Q, MODE, PASS>::CPB, smem);
}

}  // namespace bosss
