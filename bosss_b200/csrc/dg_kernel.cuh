// dg_kernel.cuh -- fused, cell-centric DG operator kernel for uniform Cartesian grids.
//
// One CTA owns a tile of CPB consecutive cells (consecutive in the reference's
// cell-major DOF layout, so the tile's coefficients are one contiguous, coalesced
// range). For its cells it evaluates
//   volume:  NECQuadratureVolume.EvaluateEx   (NECQuadratureVolume.cs:328-750)
//   faces:   NECQuadratureEdge.EvaluateEx     (NECQuadratureEdge.cs:642-1427)
// and writes each cell's result exactly once:  out = beta*out + alpha*R
// (DifferentialOperator.cs:1593-1594, NECQuadratureVolume.cs:794, NECQuadratureEdge.cs:395-400).
//
// Design choices (B200):
//  * sum factorisation: the reference basis is a product of 1D normalised Legendre
//    polynomials and the rules are tensor Gauss rules, so the dense [Np x Nq]
//    contractions of DGField.Evaluate (DGField_Evaluation.cs:59-129, a BLAS dgemm)
//    and of the test-function projection (NECQuadratureVolume.cs:689-716) are done
//    dimension by dimension with 1D tables held in shared memory;
//  * faces are cell-centric: every cell integrates all 2D of its faces and keeps
//    only its own side's contribution. The numerical flux is evaluated once per
//    face side with the reference's IN/OUT roles (IN = lower cell, normal +e_d), so
//    both cells see bit-identical flux values, and no atomics, no colouring and no
//    second pass over the residual are needed (the reference's edge scatter
//    SaveIntegrationResults is a read-modify-write of both cells);
//  * one kernel for residual, JVP and VJP: the pointwise functors are templated on
//    the scalar type; DualN<1> gives J*v, DualN<n> gives the gradient of the adjoint
//    functional  sum_q  (fV lambda + fG . grad lambda)  w.r.t. the own-side inputs,
//    which projected on the trial functions is J^T w.
#pragma once
#include "dg_common.cuh"
#include "dg_physics.cuh"

namespace bosss {

enum { MODE_RES = 0, MODE_JVP = 1, MODE_VJP = 2 };

struct EvalArgs {
    Tables1D tab;
    GridConst g;
    PhysParams ph;
    const double* U;   // state, domain layout
    const double* V;   // JVP: direction (domain layout); VJP: adjoint weights (codomain layout)
    double* out;       // RES/JVP: codomain layout; VJP: domain layout
    double alpha, beta;
    double time;
    // optional species masks of the XDG bulk evaluation (null: every cell and face):
    // vol_flag[j] == 1 -> the cell's volume integral uses the standard rule;
    // face_flag[j*2D + 2d + s] == 1 -> face (d, s) of cell j uses the standard rule.
    // Any other value: the term is skipped here (not in the species, or integrated with a
    // cut-cell rule by the explicit-rule kernel).
    const unsigned char* vol_flag;
    const unsigned char* face_flag;
    // the launch evaluates the cells [cbeg, cend) (the whole grid: 0, J)
    long long cbeg, cend;
    // 1: face terms only (the slab kernel skips its volume pass; the split-precision path
    // evaluates the volume terms on the tensor cores first and the faces add with beta = 1)
    int faces_only;
    // 1: volume terms only (the slab kernel skips its face passes; the face-once path adds
    // the face terms from its face buffer afterwards)
    int volume_only;
    // optional per-cell penalty size factor (1 / cell length scale) of the SIP penalty, in the
    // local cell order; null: the grid's 1 / CellLengthScale. The XDG bulk sets the species'
    // cut-cell length scales here (CoefficientSet.CellLengthScales, XLaplace.cs:104-113).
    const double* cell_pf;
    // optional boundary-state table: outer values of the NV domain variables at every boundary
    // face node, bnd_state[(bnd_off[j*2D + 2d + s] + q) * NV + f] for boundary face (d, s) of
    // cell j and face node q (bnd_off -1: interior face); read by functors whose boundary
    // terms take a prescribed outer state (CNS viscous terms)
    const long long* bnd_off;
    const double* bnd_state;
    // optional boundary-condition kind per boundary face node (same numbering; null: all 0):
    // 0 the table's outer state, 1 the inner state (supersonic outlet), 2 the inner state with
    // its normal momentum reflected (adiabatic slip wall); kinds 1 and 2: HLLC fluxes only
    const int* bnd_kind;
};

template <class Phys, int K, int Q, int MODE>
struct Cfg {
    static constexpr int D = Phys::D;
    static constexpr int NP = np_of(D, K);
    static constexpr int QF = (D == 2) ? Q : Q * Q;
    static constexpr int QV = QF * Q;
    static constexpr int NV = Phys::NV, NC = Phys::NC;
    static constexpr int NF1 = (MODE == MODE_RES) ? 0 : ((MODE == MODE_JVP) ? NV : NC);
    static constexpr int NFI = NV + NF1;   // interpolated fields
    static constexpr bool GRAD_IN = Phys::GRAD_U || (MODE == MODE_VJP && (Phys::VOL_G || Phys::FACE_G));
    static constexpr int NCI = GRAD_IN ? 1 + D : 1;
    static constexpr int NO = (MODE == MODE_VJP) ? NV : NC;    // projected outputs
    static constexpr bool VOL_OV = (MODE == MODE_VJP) ? true : Phys::VOL_V;
    static constexpr bool VOL_OG = (MODE == MODE_VJP) ? Phys::GRAD_U : Phys::VOL_G;
    static constexpr bool FACE_OV = (MODE == MODE_VJP) ? true : Phys::FACE_V;
    static constexpr bool FACE_OG = (MODE == MODE_VJP) ? Phys::GRAD_U : Phys::FACE_G;
    static constexpr int NCO = 1 + D;
    static constexpr int NPAIR = (K + 1) * (K + 2) / 2;
    // VJP: number of own-side tangent slots (values + gradients of the state)
    static constexpr int NS = NV * (Phys::GRAD_U ? 1 + D : 1);

    // ---- shared memory per cell (doubles)
    static constexpr int S_CIN = NFI * NP;
    static constexpr int S_R = NO * NP;
    static constexpr int S_T1 = (D == 3) ? NFI * 2 * NPAIR * Q : 0;
    static constexpr int S_P1 = (D == 3) ? NO * 3 * (K + 1) * Q * Q : NO * 2 * (K + 1) * Q;
    static constexpr int S_VA = (S_T1 > S_P1) ? S_T1 : S_P1;
    static constexpr int S_NODEVAL = NFI * NCI * QV;
    static constexpr int S_NODEOUT = NO * NCO * QV;
    static constexpr int S_VOL = S_VA + S_NODEVAL + S_NODEOUT;
    // faces, per direction (2 faces: lower, upper)
    static constexpr int S_CNB = 2 * NFI * NP;
    static constexpr int S_F1 = (D == 3) ? 2 * 2 * NFI * 3 * (K + 1) * Q : 0;
    static constexpr int S_TR = 2 * 2 * NFI * NCI * QF;
    static constexpr int S_FOUT = 2 * NO * NCO * QF;
    static constexpr int S_G1 = (D == 3) ? 2 * NO * 3 * (K + 1) * Q : 0;
    static constexpr int S_FACE = S_CNB + S_F1 + S_TR + S_FOUT + S_G1;
    static constexpr int S_CELL = S_CIN + S_R + ((S_VOL > S_FACE) ? S_VOL : S_FACE);
    static constexpr int BUDGET = 110 * 1024 / 8;   // doubles per CTA: two CTAs per SM
    static constexpr int CPB_RAW = BUDGET / S_CELL;
    static constexpr int CPB = CPB_RAW < 1 ? 1 : (CPB_RAW > 16 ? 16 : CPB_RAW);
    static constexpr int NT = 256;
    static constexpr int S_TAB = sizeof(Tables1D) / 8 + 2 * NP;  // tables + mode decode
    static constexpr size_t SMEM_BYTES = (size_t)(CPB * S_CELL + S_TAB) * 8;
};

__host__ __device__ constexpr int pair_index(int K, int a, int b) { return a * (K + 1) - a * (a - 1) / 2 + b; }

__device__ __forceinline__ void cell_ijk(const GridConst& g, long long j, int* ijk) {
#pragma unroll
    for (int d = 0; d < 3; ++d) ijk[d] = (d < g.D) ? (int)((j / g.stride[d]) % g.n[d]) : 0;
}

// neighbour across the face (d, s); s = 0 lower, 1 upper; -1 on a non-periodic boundary
__device__ __forceinline__ long long neighbour(const GridConst& g, const int* ijk, int d, int s) {
    int i = ijk[d] + (s ? 1 : -1);
    if (i < 0 || i >= g.n[d]) {
        if (!g.periodic[d]) return -1;
        i = (i + g.n[d]) % g.n[d];
    }
    long long j = 0;
#pragma unroll
    for (int dd = 0; dd < 3; ++dd)
        if (dd < g.D) j += (long long)((dd == d) ? i : ijk[dd]) * g.stride[dd];
    return j;
}

// cj = 1/CellLengthScale = (surface + boundary surface) * 0.5 / volume  (GridData_CellData.cs:683-684)
__device__ __forceinline__ double cell_cj(const GridConst& g, const int* ijk);

// penalty size factor of a cell: the per-cell array when given (whole grids), else cj
__device__ __forceinline__ double penalty_size(const double* pf, const GridConst& g, const int* ijk) {
    if (pf) {
        long long j = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d < g.D) j += (long long)ijk[d] * g.stride[d];
        return pf[j];
    }
    return cell_cj(g, ijk);
}

__device__ __forceinline__ double cell_cj(const GridConst& g, const int* ijk) {
    double cj = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d >= g.D) break;
        // boundary faces of the global grid count twice (GridData_CellData.cs:663-684)
        int nb = 0;
        if (!g.gper[d]) {
            const int gi = ijk[d] + g.goff[d];
            nb = (gi == 0) + (gi == g.gn[d] - 1);
        }
        cj += (2.0 + nb) / g.h[d];
    }
    return 0.5 * cj;
}

// ------------------------------------------------------------------ one tile
// Evaluates the tile of cells [c0, c0 + CPB) of one operator instance; all NT threads of
// the CTA take part. Used by dg_cell_kernel (one tile per CTA) and by the persistent
// batched kernel (tiles of many instances pulled from a work queue).
template <class Phys, int K, int Q, int MODE>
__device__ __forceinline__ void cell_tile(const EvalArgs& args, long long c0, double* smem) {
    using C = Cfg<Phys, K, Q, MODE>;
    constexpr int D = C::D, NP = C::NP, QF = C::QF, QV = C::QV, NV = C::NV, NC = C::NC;
    constexpr int NFI = C::NFI, NCI = C::NCI, NO = C::NO, NCO = C::NCO, CPB = C::CPB, NT = C::NT;
    constexpr int NPAIR = C::NPAIR;

    const GridConst& g = args.g;
    const int tid = threadIdx.x;
    const int ncell = (int)((args.cend - c0) < CPB ? (args.cend - c0) : CPB);

    // ---- carve shared memory
    Tables1D* tab = reinterpret_cast<Tables1D*>(smem);
    int* modes = reinterpret_cast<int*>(smem + sizeof(Tables1D) / 8);   // packed (a,b,c) per mode
    double* cellbase = smem + C::S_TAB;
    auto CIN = [&](int cl) { return cellbase + (size_t)cl * C::S_CELL; };
    auto RR = [&](int cl) { return cellbase + (size_t)cl * C::S_CELL + C::S_CIN; };
    auto WORK = [&](int cl) { return cellbase + (size_t)cl * C::S_CELL + C::S_CIN + C::S_R; };

    for (int i = tid; i < (int)(sizeof(Tables1D) / 8); i += NT)
        reinterpret_cast<double*>(tab)[i] = reinterpret_cast<const double*>(&args.tab)[i];
    if (tid == 0) {
        int n = 0;
        for (int deg = 0; deg <= K; ++deg) {
            if (D == 2) {
                for (int a = 0; a <= deg; ++a) modes[n++] = a | ((deg - a) << 8);
            } else {
                for (int a = 0; a <= deg; ++a)
                    for (int b = 0; b <= deg - a; ++b) modes[n++] = a | (b << 8) | ((deg - a - b) << 16);
            }
        }
    }
    // ---- load coefficients (contiguous per tile) and clear R
    constexpr int NVPC = NV * NP;
    constexpr int N1PC = C::NF1 * NP;
    for (int i = tid; i < ncell * NVPC; i += NT) {
        int cl = i / NVPC, r = i % NVPC;
        CIN(cl)[r] = args.U[c0 * NVPC + i];
    }
    if constexpr (C::NF1 > 0) {
        for (int i = tid; i < ncell * N1PC; i += NT) {
            int cl = i / N1PC, r = i % N1PC;
            CIN(cl)[NVPC + r] = args.V[c0 * N1PC + i];
        }
    }
    for (int i = tid; i < CPB * C::S_R; i += NT) RR(i / C::S_R)[i % C::S_R] = 0.0;
    __syncthreads();

    const double scaling = g.scaling;

    // ================================================================== volume
    {
        double* VA = nullptr;   // per-cell pointers computed inside loops
        (void)VA;
        auto T1 = [&](int cl) { return WORK(cl); };
        auto P1 = [&](int cl) { return WORK(cl); };
        auto NVAL = [&](int cl) { return WORK(cl) + C::S_VA; };
        auto NOUT = [&](int cl) { return WORK(cl) + C::S_VA + C::S_NODEVAL; };

        // ---- interpolation: u, grad u at the volume nodes (DGField.Evaluate / EvaluateGradient)
        if constexpr (D == 2) {
            for (int it = tid; it < CPB * NFI * Q; it += NT) {
                const int qy = it % Q, f = (it / Q) % NFI, cl = it / (Q * NFI);
                if (cl >= ncell) continue;
                const double* c = CIN(cl) + f * NP;
                double T[K + 1], Ty[K + 1];
#pragma unroll
                for (int a = 0; a <= K; ++a) {
                    double s = 0.0, sy = 0.0;
#pragma unroll
                    for (int b = 0; b <= K - a; ++b) {
                        double cf = c[mode2(a, b)];
                        s += cf * tab->A[qy][b];
                        if (C::GRAD_IN) sy += cf * tab->dA[qy][b];
                    }
                    T[a] = s;
                    Ty[a] = sy;
                }
                double* nv = NVAL(cl) + f * NCI * QV;
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    double u = 0.0, ux = 0.0, uy = 0.0;
#pragma unroll
                    for (int a = 0; a <= K; ++a) {
                        u += T[a] * tab->A[qx][a];
                        if (C::GRAD_IN) {
                            ux += T[a] * tab->dA[qx][a];
                            uy += Ty[a] * tab->A[qx][a];
                        }
                    }
                    const int q = qy * Q + qx;
                    nv[q] = u * scaling;
                    if (C::GRAD_IN) {
                        nv[QV + q] = ux * scaling * g.twoh[0];
                        nv[2 * QV + q] = uy * scaling * g.twoh[1];
                    }
                }
            }
            __syncthreads();
        } else {
            // stage 1: contract z
            for (int it = tid; it < CPB * NFI * Q; it += NT) {
                const int qz = it % Q, f = (it / Q) % NFI, cl = it / (Q * NFI);
                if (cl >= ncell) continue;
                const double* c = CIN(cl) + f * NP;
                double* t1 = T1(cl) + f * 2 * NPAIR * Q;
#pragma unroll
                for (int a = 0; a <= K; ++a)
#pragma unroll
                    for (int b = 0; b <= K - a; ++b) {
                        double s = 0.0, sz = 0.0;
#pragma unroll
                        for (int cc = 0; cc <= K - a - b; ++cc) {
                            double cf = c[mode3(a, b, cc)];
                            s += cf * tab->A[qz][cc];
                            if (C::GRAD_IN) sz += cf * tab->dA[qz][cc];
                        }
                        t1[pair_index(K, a, b) * Q + qz] = s;
                        if (C::GRAD_IN) t1[(NPAIR + pair_index(K, a, b)) * Q + qz] = sz;
                    }
            }
            __syncthreads();
            // stage 2: contract y, then x (register resident)
            for (int it = tid; it < CPB * NFI * Q * Q; it += NT) {
                const int qz = it % Q, qy = (it / Q) % Q, f = (it / (Q * Q)) % NFI, cl = it / (Q * Q * NFI);
                if (cl >= ncell) continue;
                const double* t1 = T1(cl) + f * 2 * NPAIR * Q;
                double T2[K + 1], T2y[K + 1], T2z[K + 1];
#pragma unroll
                for (int a = 0; a <= K; ++a) {
                    double s = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
                    for (int b = 0; b <= K - a; ++b) {
                        double v = t1[pair_index(K, a, b) * Q + qz];
                        s += v * tab->A[qy][b];
                        if (C::GRAD_IN) {
                            sy += v * tab->dA[qy][b];
                            sz += t1[(NPAIR + pair_index(K, a, b)) * Q + qz] * tab->A[qy][b];
                        }
                    }
                    T2[a] = s;
                    T2y[a] = sy;
                    T2z[a] = sz;
                }
                double* nv = NVAL(cl) + f * NCI * QV;
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    double u = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
#pragma unroll
                    for (int a = 0; a <= K; ++a) {
                        u += T2[a] * tab->A[qx][a];
                        if (C::GRAD_IN) {
                            ux += T2[a] * tab->dA[qx][a];
                            uy += T2y[a] * tab->A[qx][a];
                            uz += T2z[a] * tab->A[qx][a];
                        }
                    }
                    const int q = (qz * Q + qy) * Q + qx;
                    nv[q] = u * scaling;
                    if (C::GRAD_IN) {
                        nv[QV + q] = ux * scaling * g.twoh[0];
                        nv[2 * QV + q] = uy * scaling * g.twoh[1];
                        nv[3 * QV + q] = uz * scaling * g.twoh[2];
                    }
                }
            }
            __syncthreads();
        }

        // ---- pointwise forms at the volume nodes
        for (int it = tid; it < CPB * QV; it += NT) {
            const int q = it % QV, cl = it / QV;
            if (cl >= ncell) continue;
            if (args.vol_flag && args.vol_flag[c0 + cl] != 1) {
                double* no0 = NOUT(cl);
                for (int e = 0; e < NO * NCO; ++e) no0[e * QV + q] = 0.0;
                continue;
            }
            int qi[3] = {q % Q, (q / Q) % Q, q / (Q * Q)};
            double W = 1.0;
            double x[3] = {0, 0, 0};
            int ijk[3];
            cell_ijk(g, c0 + cl, ijk);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                W *= tab->w[qi[d]];
                x[d] = g.lo[d] + (ijk[d] + g.goff[d] + 0.5 + 0.5 * tab->xq[qi[d]]) * g.h[d];
            }
            const double* nv = NVAL(cl);
            double* no = NOUT(cl);
            const double fac = W * g.detJ * scaling;
            if constexpr (MODE == MODE_RES) {
                double Uq[NV], Gq[NV][D], fV[NC], fG[NC][D];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    Uq[i] = nv[i * NCI * QV + q];
#pragma unroll
                    for (int d = 0; d < D; ++d) Gq[i][d] = C::GRAD_IN ? nv[(i * NCI + 1 + d) * QV + q] : 0.0;
                }
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    fV[e] = 0.0;
#pragma unroll
                    for (int d = 0; d < D; ++d) fG[e][d] = 0.0;
                }
                Phys::volume(args.ph, Uq, Gq, x, fV, fG);
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    if (C::VOL_OV) no[(e * NCO) * QV + q] = fV[e] * fac;
                    if (C::VOL_OG)
#pragma unroll
                        for (int d = 0; d < D; ++d) no[(e * NCO + 1 + d) * QV + q] = fG[e][d] * fac * g.twoh[d];
                }
            } else if constexpr (MODE == MODE_JVP) {
                using T = DualN<1>;
                T Uq[NV], Gq[NV][D], fV[NC], fG[NC][D];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    Uq[i].v = nv[i * NCI * QV + q];
                    Uq[i].d[0] = nv[((NV + i) * NCI) * QV + q];
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        Gq[i][d].v = C::GRAD_IN ? nv[(i * NCI + 1 + d) * QV + q] : 0.0;
                        Gq[i][d].d[0] = C::GRAD_IN ? nv[((NV + i) * NCI + 1 + d) * QV + q] : 0.0;
                    }
                }
                Phys::volume(args.ph, Uq, Gq, x, fV, fG);
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    if (C::VOL_OV) no[(e * NCO) * QV + q] = fV[e].d[0] * fac;
                    if (C::VOL_OG)
#pragma unroll
                        for (int d = 0; d < D; ++d) no[(e * NCO + 1 + d) * QV + q] = fG[e][d].d[0] * fac * g.twoh[d];
                }
            } else {
                constexpr int NS = C::NS;
                using T = DualN<NS>;
                T Uq[NV], Gq[NV][D], fV[NC], fG[NC][D];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    Uq[i] = T(nv[i * NCI * QV + q]);
                    Uq[i].d[Phys::GRAD_U ? i * (1 + D) : i] = 1.0;
#pragma unroll
                    for (int d = 0; d < D; ++d) {
                        Gq[i][d] = T(C::GRAD_IN ? nv[(i * NCI + 1 + d) * QV + q] : 0.0);
                        if (Phys::GRAD_U) Gq[i][d].d[i * (1 + D) + 1 + d] = 1.0;
                    }
                }
                Phys::volume(args.ph, Uq, Gq, x, fV, fG);
                T phi(0.0);
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    const int fe = NV + e;
                    if (Phys::VOL_V) phi += fV[e] * nv[(fe * NCI) * QV + q];
                    if (Phys::VOL_G)
#pragma unroll
                        for (int d = 0; d < D; ++d) phi += fG[e][d] * nv[(fe * NCI + 1 + d) * QV + q];
                }
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    no[(i * NCO) * QV + q] = phi.d[Phys::GRAD_U ? i * (1 + D) : i] * fac;
                    if (Phys::GRAD_U)
#pragma unroll
                        for (int d = 0; d < D; ++d)
                            no[(i * NCO + 1 + d) * QV + q] = phi.d[i * (1 + D) + 1 + d] * fac * g.twoh[d];
                }
            }
        }
        __syncthreads();

        // ---- projection onto the test functions (einsum "jn" = "jke"."kne" + "jk"."kn")
        if constexpr (D == 2) {
            for (int it = tid; it < CPB * NO * Q; it += NT) {
                const int qy = it % Q, o = (it / Q) % NO, cl = it / (Q * NO);
                if (cl >= ncell) continue;
                const double* no = NOUT(cl) + o * NCO * QV;
                double* p1 = P1(cl) + o * 2 * (K + 1) * Q;
                double P[K + 1], Py[K + 1];
#pragma unroll
                for (int a = 0; a <= K; ++a) P[a] = Py[a] = 0.0;
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    const int q = qy * Q + qx;
                    const double s = C::VOL_OV ? no[q] : 0.0;
                    const double gx = C::VOL_OG ? no[QV + q] : 0.0;
                    const double gy = C::VOL_OG ? no[2 * QV + q] : 0.0;
#pragma unroll
                    for (int a = 0; a <= K; ++a) {
                        P[a] += s * tab->A[qx][a] + gx * tab->dA[qx][a];
                        Py[a] += gy * tab->A[qx][a];
                    }
                }
#pragma unroll
                for (int a = 0; a <= K; ++a) {
                    p1[a * Q + qy] = P[a];
                    p1[((K + 1) + a) * Q + qy] = Py[a];
                }
            }
            __syncthreads();
            for (int it = tid; it < CPB * NO * NP; it += NT) {
                const int n = it % NP, o = (it / NP) % NO, cl = it / (NP * NO);
                if (cl >= ncell) continue;
                const int a = modes[n] & 0xff, b = (modes[n] >> 8) & 0xff;
                const double* p1 = P1(cl) + o * 2 * (K + 1) * Q;
                double acc = 0.0;
#pragma unroll
                for (int qy = 0; qy < Q; ++qy)
                    acc += p1[a * Q + qy] * tab->A[qy][b] + p1[((K + 1) + a) * Q + qy] * tab->dA[qy][b];
                RR(cl)[o * NP + n] += acc;
            }
            __syncthreads();
        } else {
            // stage 1: contract x
            for (int it = tid; it < CPB * NO * Q * Q; it += NT) {
                const int qz = it % Q, qy = (it / Q) % Q, o = (it / (Q * Q)) % NO, cl = it / (Q * Q * NO);
                if (cl >= ncell) continue;
                const double* no = NOUT(cl) + o * NCO * QV;
                double* p1 = P1(cl) + o * 3 * (K + 1) * Q * Q;
                double P[K + 1], Py[K + 1], Pz[K + 1];
#pragma unroll
                for (int a = 0; a <= K; ++a) P[a] = Py[a] = Pz[a] = 0.0;
#pragma unroll
                for (int qx = 0; qx < Q; ++qx) {
                    const int q = (qz * Q + qy) * Q + qx;
                    const double s = C::VOL_OV ? no[q] : 0.0;
                    const double gx = C::VOL_OG ? no[QV + q] : 0.0;
                    const double gy = C::VOL_OG ? no[2 * QV + q] : 0.0;
                    const double gz = C::VOL_OG ? no[3 * QV + q] : 0.0;
#pragma unroll
                    for (int a = 0; a <= K; ++a) {
                        P[a] += s * tab->A[qx][a] + gx * tab->dA[qx][a];
                        Py[a] += gy * tab->A[qx][a];
                        Pz[a] += gz * tab->A[qx][a];
                    }
                }
#pragma unroll
                for (int a = 0; a <= K; ++a) {
                    p1[(a * Q + qz) * Q + qy] = P[a];
                    p1[(((K + 1) + a) * Q + qz) * Q + qy] = Py[a];
                    p1[((2 * (K + 1) + a) * Q + qz) * Q + qy] = Pz[a];
                }
            }
            __syncthreads();
            // stage 2: contract y then z, per (a,b) pair
            for (int it = tid; it < CPB * NO * NPAIR; it += NT) {
                int pr = it % NPAIR;
                const int o = (it / NPAIR) % NO, cl = it / (NPAIR * NO);
                if (cl >= ncell) continue;
                int a = 0;
                while (pr > K - a) { pr -= K - a + 1; ++a; }
                const int b = pr;
                const double* p1 = P1(cl) + o * 3 * (K + 1) * Q * Q;
                double t[Q], tz[Q];
#pragma unroll
                for (int qz = 0; qz < Q; ++qz) {
                    double s = 0.0, sz = 0.0;
#pragma unroll
                    for (int qy = 0; qy < Q; ++qy) {
                        s += p1[(a * Q + qz) * Q + qy] * tab->A[qy][b] +
                             p1[(((K + 1) + a) * Q + qz) * Q + qy] * tab->dA[qy][b];
                        sz += p1[((2 * (K + 1) + a) * Q + qz) * Q + qy] * tab->A[qy][b];
                    }
                    t[qz] = s;
                    tz[qz] = sz;
                }
                for (int cc = 0; cc <= K - a - b; ++cc) {
                    double acc = 0.0;
#pragma unroll
                    for (int qz = 0; qz < Q; ++qz) acc += t[qz] * tab->A[qz][cc] + tz[qz] * tab->dA[qz][cc];
                    RR(cl)[o * NP + mode3(a, b, cc)] += acc;
                }
            }
            __syncthreads();
        }
    }

    // ================================================================== faces
#pragma unroll 1
    for (int d = 0; d < D; ++d) {
        // tangential directions (ascending)
        const int t1 = (d == 0) ? 1 : 0;
        const int t2 = (D == 3) ? ((d == 2) ? 1 : 2) : -1;
        auto CNB = [&](int cl, int s) { return WORK(cl) + s * NFI * NP; };
        auto F1 = [&](int cl) { return WORK(cl) + C::S_CNB; };
        auto TR = [&](int cl) { return WORK(cl) + C::S_CNB + C::S_F1; };
        auto FOUT = [&](int cl) { return WORK(cl) + C::S_CNB + C::S_F1 + C::S_TR; };
        auto G1 = [&](int cl) { return WORK(cl) + C::S_CNB + C::S_F1 + C::S_TR + C::S_FOUT; };

        // ---- neighbour coefficients for the lower (s=0) and upper (s=1) face
        for (int i = tid; i < 2 * CPB * NFI * NP; i += NT) {
            const int r = i % (NFI * NP), cl = (i / (NFI * NP)) % CPB, s = i / (NFI * NP * CPB);
            if (cl >= ncell) continue;
            int ijk[3];
            cell_ijk(g, c0 + cl, ijk);
            long long nb = neighbour(g, ijk, d, s);
            double v = 0.0;
            if (nb >= 0) {
                const int f = r / NP, n = r % NP;
                v = (f < NV) ? args.U[nb * NVPC + f * NP + n] : args.V[nb * N1PC + (f - NV) * NP + n];
            }
            CNB(cl, s)[r] = v;
        }
        __syncthreads();

        // m = exponent along d, p along t1, r along t2
        auto modeDPR = [&](int m, int p, int r) -> int {
            int e[3];
            e[d] = m;
            e[t1] = p;
            if (D == 3) e[t2] = r;
            return (D == 2) ? mode2(e[0], e[1]) : mode3(e[0], e[1], e[2]);
        };

        // ---- traces of own (side 0) and neighbour (side 1) cell at both faces
        // TR layout: [s][side][f][comp][qf]
        if constexpr (D == 2) {
            for (int it = tid; it < 2 * 2 * CPB * NFI * Q; it += NT) {
                const int q1 = it % Q, f = (it / Q) % NFI, cl = (it / (Q * NFI)) % CPB, side = (it / (Q * NFI * CPB)) % 2,
                          s = it / (Q * NFI * CPB * 2);
                if (cl >= ncell) continue;
                const double* c = side ? CNB(cl, s) + f * NP : CIN(cl) + f * NP;
                const int fs = side ? 1 - s : s;   // which face of that cell (0: xi_d=-1, 1: +1)
                double u = 0.0, ut = 0.0, un = 0.0;
#pragma unroll
                for (int p = 0; p <= K; ++p) {
                    double S = 0.0, Sn = 0.0;
#pragma unroll
                    for (int m = 0; m <= K - p; ++m) {
                        double cf = c[modeDPR(m, p, 0)];
                        S += cf * tab->e[fs][m];
                        if (C::GRAD_IN) Sn += cf * tab->de[fs][m];
                    }
                    u += S * tab->A[q1][p];
                    if (C::GRAD_IN) {
                        ut += S * tab->dA[q1][p];
                        un += Sn * tab->A[q1][p];
                    }
                }
                double* tr = TR(cl) + ((s * 2 + side) * NFI + f) * NCI * QF;
                tr[q1] = u * scaling;
                if (C::GRAD_IN) {
                    tr[(1 + d) * QF + q1] = un * scaling * g.twoh[d];
                    tr[(1 + t1) * QF + q1] = ut * scaling * g.twoh[t1];
                }
            }
            __syncthreads();
        } else {
            // stage 1: collapse along d, contract t2
            for (int it = tid; it < 2 * 2 * CPB * NFI * Q; it += NT) {
                const int q2 = it % Q, f = (it / Q) % NFI, cl = (it / (Q * NFI)) % CPB, side = (it / (Q * NFI * CPB)) % 2,
                          s = it / (Q * NFI * CPB * 2);
                if (cl >= ncell) continue;
                const double* c = side ? CNB(cl, s) + f * NP : CIN(cl) + f * NP;
                const int fs = side ? 1 - s : s;
                double* f1 = F1(cl) + ((s * 2 + side) * NFI + f) * 3 * (K + 1) * Q;
#pragma unroll
                for (int p = 0; p <= K; ++p) {
                    double T = 0.0, Tn = 0.0, Tt2 = 0.0;
#pragma unroll
                    for (int r = 0; r <= K - p; ++r) {
                        double S = 0.0, Sn = 0.0;
#pragma unroll
                        for (int m = 0; m <= K - p - r; ++m) {
                            double cf = c[modeDPR(m, p, r)];
                            S += cf * tab->e[fs][m];
                            if (C::GRAD_IN) Sn += cf * tab->de[fs][m];
                        }
                        T += S * tab->A[q2][r];
                        if (C::GRAD_IN) {
                            Tn += Sn * tab->A[q2][r];
                            Tt2 += S * tab->dA[q2][r];
                        }
                    }
                    f1[p * Q + q2] = T;
                    if (C::GRAD_IN) {
                        f1[((K + 1) + p) * Q + q2] = Tn;
                        f1[(2 * (K + 1) + p) * Q + q2] = Tt2;
                    }
                }
            }
            __syncthreads();
            // stage 2: contract t1
            for (int it = tid; it < 2 * 2 * CPB * NFI * QF; it += NT) {
                const int qf = it % QF, f = (it / QF) % NFI, cl = (it / (QF * NFI)) % CPB,
                          side = (it / (QF * NFI * CPB)) % 2, s = it / (QF * NFI * CPB * 2);
                if (cl >= ncell) continue;
                const int q1 = qf % Q, q2 = qf / Q;
                const double* f1 = F1(cl) + ((s * 2 + side) * NFI + f) * 3 * (K + 1) * Q;
                double u = 0.0, ut1 = 0.0, ut2 = 0.0, un = 0.0;
#pragma unroll
                for (int p = 0; p <= K; ++p) {
                    const double T = f1[p * Q + q2];
                    u += T * tab->A[q1][p];
                    if (C::GRAD_IN) {
                        ut1 += T * tab->dA[q1][p];
                        un += f1[((K + 1) + p) * Q + q2] * tab->A[q1][p];
                        ut2 += f1[(2 * (K + 1) + p) * Q + q2] * tab->A[q1][p];
                    }
                }
                double* tr = TR(cl) + ((s * 2 + side) * NFI + f) * NCI * QF;
                tr[qf] = u * scaling;
                if (C::GRAD_IN) {
                    tr[(1 + d) * QF + qf] = un * scaling * g.twoh[d];
                    tr[(1 + t1) * QF + qf] = ut1 * scaling * g.twoh[t1];
                    tr[(1 + t2) * QF + qf] = ut2 * scaling * g.twoh[t2];
                }
            }
            __syncthreads();
        }

        // ---- pointwise edge forms (own side kept); FOUT layout [s][o][comp][qf]
        for (int it = tid; it < 2 * CPB * QF; it += NT) {
            const int qf = it % QF, cl = (it / QF) % CPB, s = it / (QF * CPB);
            if (cl >= ncell) continue;
            if (args.face_flag && args.face_flag[(c0 + cl) * (2 * D) + 2 * d + s] != 1) {
                double* fo0 = FOUT(cl) + s * NO * NCO * QF;
                for (int e = 0; e < NO * NCO; ++e) fo0[e * QF + qf] = 0.0;
                continue;
            }
            int ijk[3];
            cell_ijk(g, c0 + cl, ijk);
            const long long nb = neighbour(g, ijk, d, s);
            const bool inner = nb >= 0;
            int q1 = qf % Q, q2 = qf / Q;
            double Wf = tab->w[q1] * ((D == 3) ? tab->w[q2] : 1.0);
            const double fac = Wf * g.faceSG[d] * scaling;
            double x[3] = {0, 0, 0};
#pragma unroll
            for (int dd = 0; dd < D; ++dd) x[dd] = g.lo[dd] + (ijk[dd] + g.goff[dd] + 0.5) * g.h[dd];
            x[d] += (s ? 0.5 : -0.5) * g.h[d];
            x[t1] += 0.5 * g.h[t1] * tab->xq[q1];
            if (D == 3) x[t2] += 0.5 * g.h[t2] * tab->xq[q2];
            double nrm[D];
#pragma unroll
            for (int dd = 0; dd < D; ++dd) nrm[dd] = 0.0;
            nrm[d] = inner ? 1.0 : (s ? 1.0 : -1.0);
            double pnlty = 0.0;
            if (inner) {
                int ijk2[3] = {ijk[0], ijk[1], ijk[2]};
                ijk2[d] = (int)((nb / g.stride[d]) % g.n[d]);
                pnlty = args.ph.pen * fmax(penalty_size(args.cell_pf, g, ijk), penalty_size(args.cell_pf, g, ijk2));
            } else {
                pnlty = Phys::BND_PEN * args.ph.pen * penalty_size(args.cell_pf, g, ijk);
            }
            const double* ub = nullptr;   // outer state of the boundary-state table at this node
            int bkind = 0;                // boundary-condition kind of the node
            if (!inner && args.bnd_off) {
                const long long o = args.bnd_off[(c0 + cl) * (2 * D) + 2 * d + s];
                if (o >= 0) {
                    if (args.bnd_state) ub = args.bnd_state + (o + qf) * NV;
                    if (args.bnd_kind) bkind = args.bnd_kind[o + qf];
                }
            }
            const bool selfA = !inner || s == 1;   // own cell is IN (lower) unless it is the upper cell
            const double* trOwn = TR(cl) + ((s * 2 + 0) * NFI) * NCI * QF;
            const double* trNb = TR(cl) + ((s * 2 + 1) * NFI) * NCI * QF;
            const double* trA = selfA ? trOwn : trNb;
            const double* trB = selfA ? trNb : trOwn;
            double* fo = FOUT(cl) + s * NO * NCO * QF;
            auto rd = [&](const double* tr, int f, int comp) { return tr[(f * NCI + comp) * QF + qf]; };

            if constexpr (MODE == MODE_RES) {
                double UA[NV], GA[NV][D], UB[NV], GB[NV][D], gA[NC], GAv[NC][D], gB[NC], GBv[NC][D];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    UA[i] = rd(trA, i, 0);
                    UB[i] = inner ? rd(trB, i, 0) : 0.0;
#pragma unroll
                    for (int dd = 0; dd < D; ++dd) {
                        GA[i][dd] = C::GRAD_IN ? rd(trA, i, 1 + dd) : 0.0;
                        GB[i][dd] = (C::GRAD_IN && inner) ? rd(trB, i, 1 + dd) : 0.0;
                    }
                }
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    gA[e] = gB[e] = 0.0;
#pragma unroll
                    for (int dd = 0; dd < D; ++dd) GAv[e][dd] = GBv[e][dd] = 0.0;
                }
                if (inner) Phys::inner(args.ph, pnlty, UA, GA, UB, GB, nrm, x, gA, GAv, gB, GBv);
                else Phys::boundary(args.ph, pnlty, UA, GA, nrm, x, ub, bkind, gA, GAv);
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    const double gv = selfA ? gA[e] : gB[e];
                    if (C::FACE_OV) fo[(e * NCO) * QF + qf] = gv * fac;
                    if (C::FACE_OG)
#pragma unroll
                        for (int dd = 0; dd < D; ++dd)
                            fo[(e * NCO + 1 + dd) * QF + qf] = (selfA ? GAv[e][dd] : GBv[e][dd]) * fac * g.twoh[dd];
                }
            } else if constexpr (MODE == MODE_JVP) {
                using T = DualN<1>;
                T UA[NV], GA[NV][D], UB[NV], GB[NV][D], gA[NC], GAv[NC][D], gB[NC], GBv[NC][D];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    UA[i].v = rd(trA, i, 0);
                    UA[i].d[0] = rd(trA, NV + i, 0);
                    UB[i].v = inner ? rd(trB, i, 0) : 0.0;
                    UB[i].d[0] = inner ? rd(trB, NV + i, 0) : 0.0;
#pragma unroll
                    for (int dd = 0; dd < D; ++dd) {
                        GA[i][dd].v = C::GRAD_IN ? rd(trA, i, 1 + dd) : 0.0;
                        GA[i][dd].d[0] = C::GRAD_IN ? rd(trA, NV + i, 1 + dd) : 0.0;
                        GB[i][dd].v = (C::GRAD_IN && inner) ? rd(trB, i, 1 + dd) : 0.0;
                        GB[i][dd].d[0] = (C::GRAD_IN && inner) ? rd(trB, NV + i, 1 + dd) : 0.0;
                    }
                }
                if (inner) Phys::inner(args.ph, pnlty, UA, GA, UB, GB, nrm, x, gA, GAv, gB, GBv);
                else Phys::boundary(args.ph, pnlty, UA, GA, nrm, x, ub, bkind, gA, GAv);
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    const double gv = selfA ? gA[e].d[0] : gB[e].d[0];
                    if (C::FACE_OV) fo[(e * NCO) * QF + qf] = gv * fac;
                    if (C::FACE_OG)
#pragma unroll
                        for (int dd = 0; dd < D; ++dd)
                            fo[(e * NCO + 1 + dd) * QF + qf] =
                                (selfA ? GAv[e][dd].d[0] : GBv[e][dd].d[0]) * fac * g.twoh[dd];
                }
            } else {
                constexpr int NS = C::NS;
                using T = DualN<NS>;
                T UA[NV], GA[NV][D], UB[NV], GB[NV][D], gA[NC], GAv[NC][D], gB[NC], GBv[NC][D];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    UA[i] = T(rd(trA, i, 0));
                    UB[i] = T(inner ? rd(trB, i, 0) : 0.0);
#pragma unroll
                    for (int dd = 0; dd < D; ++dd) {
                        GA[i][dd] = T(C::GRAD_IN ? rd(trA, i, 1 + dd) : 0.0);
                        GB[i][dd] = T((C::GRAD_IN && inner) ? rd(trB, i, 1 + dd) : 0.0);
                    }
                    T* Us = selfA ? &UA[i] : &UB[i];
                    Us->d[Phys::GRAD_U ? i * (1 + D) : i] = 1.0;
                    if (Phys::GRAD_U)
#pragma unroll
                        for (int dd = 0; dd < D; ++dd) (selfA ? GA : GB)[i][dd].d[i * (1 + D) + 1 + dd] = 1.0;
                }
                if (inner) Phys::inner(args.ph, pnlty, UA, GA, UB, GB, nrm, x, gA, GAv, gB, GBv);
                else Phys::boundary(args.ph, pnlty, UA, GA, nrm, x, ub, bkind, gA, GAv);
                T phi(0.0);
#pragma unroll
                for (int e = 0; e < NC; ++e) {
                    const int fe = NV + e;
                    if (Phys::FACE_V) {
                        phi += gA[e] * rd(trA, fe, 0);
                        if (inner) phi += gB[e] * rd(trB, fe, 0);
                    }
                    if (Phys::FACE_G)
#pragma unroll
                        for (int dd = 0; dd < D; ++dd) {
                            phi += GAv[e][dd] * rd(trA, fe, 1 + dd);
                            if (inner) phi += GBv[e][dd] * rd(trB, fe, 1 + dd);
                        }
                }
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    fo[(i * NCO) * QF + qf] = phi.d[Phys::GRAD_U ? i * (1 + D) : i] * fac;
                    if (Phys::GRAD_U)
#pragma unroll
                        for (int dd = 0; dd < D; ++dd)
                            fo[(i * NCO + 1 + dd) * QF + qf] = phi.d[i * (1 + D) + 1 + dd] * fac * g.twoh[dd];
                }
            }
        }
        __syncthreads();

        // ---- project on the own test functions, both faces
        if constexpr (D == 2) {
            for (int it = tid; it < CPB * NO * NP; it += NT) {
                const int n = it % NP, o = (it / NP) % NO, cl = it / (NP * NO);
                if (cl >= ncell) continue;
                int e[2] = {modes[n] & 0xff, (modes[n] >> 8) & 0xff};
                const int m = e[d], p = e[t1];
                double acc = 0.0;
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const double* fo = FOUT(cl) + (s * NO + o) * NCO * QF;
                    double a0 = 0.0, an = 0.0;
#pragma unroll
                    for (int q1 = 0; q1 < Q; ++q1) {
                        const double gv = C::FACE_OV ? fo[q1] : 0.0;
                        const double gn = C::FACE_OG ? fo[(1 + d) * QF + q1] : 0.0;
                        const double gt = C::FACE_OG ? fo[(1 + t1) * QF + q1] : 0.0;
                        a0 += gv * tab->A[q1][p] + gt * tab->dA[q1][p];
                        an += gn * tab->A[q1][p];
                    }
                    acc += a0 * tab->e[s][m] + an * tab->de[s][m];
                }
                RR(cl)[o * NP + n] += acc;
            }
            __syncthreads();
        } else {
            // stage 1: contract t1; G1 layout [s][o][3][p][q2]
            for (int it = tid; it < 2 * CPB * NO * Q; it += NT) {
                const int q2 = it % Q, o = (it / Q) % NO, cl = (it / (Q * NO)) % CPB, s = it / (Q * NO * CPB);
                if (cl >= ncell) continue;
                const double* fo = FOUT(cl) + (s * NO + o) * NCO * QF;
                double P[K + 1], Pn[K + 1], Pt2[K + 1];
#pragma unroll
                for (int p = 0; p <= K; ++p) P[p] = Pn[p] = Pt2[p] = 0.0;
#pragma unroll
                for (int q1 = 0; q1 < Q; ++q1) {
                    const int qf = q2 * Q + q1;
                    const double gv = C::FACE_OV ? fo[qf] : 0.0;
                    const double gn = C::FACE_OG ? fo[(1 + d) * QF + qf] : 0.0;
                    const double g1 = C::FACE_OG ? fo[(1 + t1) * QF + qf] : 0.0;
                    const double g2 = C::FACE_OG ? fo[(1 + t2) * QF + qf] : 0.0;
#pragma unroll
                    for (int p = 0; p <= K; ++p) {
                        P[p] += gv * tab->A[q1][p] + g1 * tab->dA[q1][p];
                        Pn[p] += gn * tab->A[q1][p];
                        Pt2[p] += g2 * tab->A[q1][p];
                    }
                }
                double* g1p = G1(cl) + (s * NO + o) * 3 * (K + 1) * Q;
#pragma unroll
                for (int p = 0; p <= K; ++p) {
                    g1p[p * Q + q2] = P[p];
                    g1p[((K + 1) + p) * Q + q2] = Pn[p];
                    g1p[(2 * (K + 1) + p) * Q + q2] = Pt2[p];
                }
            }
            __syncthreads();
            // stage 2: contract t2 and expand along d
            for (int it = tid; it < CPB * NO * NP; it += NT) {
                const int n = it % NP, o = (it / NP) % NO, cl = it / (NP * NO);
                if (cl >= ncell) continue;
                int e[3] = {modes[n] & 0xff, (modes[n] >> 8) & 0xff, (modes[n] >> 16) & 0xff};
                const int m = e[d], p = e[t1], r = e[t2];
                double acc = 0.0;
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const double* g1p = G1(cl) + (s * NO + o) * 3 * (K + 1) * Q;
                    double a0 = 0.0, an = 0.0;
#pragma unroll
                    for (int q2 = 0; q2 < Q; ++q2) {
                        a0 += g1p[p * Q + q2] * tab->A[q2][r] + g1p[(2 * (K + 1) + p) * Q + q2] * tab->dA[q2][r];
                        an += g1p[((K + 1) + p) * Q + q2] * tab->A[q2][r];
                    }
                    acc += a0 * tab->e[s][m] + an * tab->de[s][m];
                }
                RR(cl)[o * NP + n] += acc;
            }
            __syncthreads();
        }
    }

    // ================================================================== store
    constexpr int NOPC = NO * NP;
    for (int i = tid; i < ncell * NOPC; i += NT) {
        const int cl = i / NOPC, r = i % NOPC;
        const long long gi = c0 * NOPC + i;
        const double v = RR(cl)[r];
        if constexpr (MODE == MODE_RES) {
            args.out[gi] = (args.beta == 0.0) ? args.alpha * v : args.beta * args.out[gi] + args.alpha * v;
        } else {
            args.out[gi] = v;
        }
    }
}

// ------------------------------------------------------------------ the kernel
template <class Phys, int K, int Q, int MODE>
__global__ void __launch_bounds__(256) dg_cell_kernel(const __grid_constant__ EvalArgs args) {
    extern __shared__ double smem[];
    cell_tile<Phys, K, Q, MODE>(args, args.cbeg + (long long)blockIdx.x * Cfg<Phys, K, Q, MODE>::CPB, smem);
}

}  // namespace bosss
