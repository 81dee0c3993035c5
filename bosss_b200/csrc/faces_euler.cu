// faces_euler.cu -- face terms of the 3D Euler (HLLC) residual and adjoint product, each
// face evaluated once.
//
// The reference scatters every edge integral to both neighbouring cells
// (NECQuadratureEdge.SaveIntegrationResults, NECQuadratureEdge.cs:326-412; IN +, OUT -,
// :998-1000). The cell-centric slab kernel evaluates each face twice, once from each side,
// and on the Euler 32^3 k=3 residual its face passes are ~90 % of the launch. Here each face
// (owner = the lower cell, normal +e_d) is evaluated once:
//
//   A  face kernel: one thread per face node evaluates both traces (the owner's upper face,
//      the neighbour's lower face) directly from the two cells' coefficients staged in
//      shared memory, then the HLLC flux (residual) or its reverse-mode adjoint (VJP, with
//      the adjoint weights' traces), and stores the quadrature-weighted values in a face
//      buffer: residual buf[owner][d][e][q] = f_e w_q SqrtGramian Scaling; VJP two sides,
//      the derivatives with respect to the owner's and the neighbour's traces;
//   B  volume terms: the slab kernel's volume pass only (or the tensor-core volume kernel
//      of the split-precision residual), out = beta out + alpha R_vol (residual) / out = the
//      volume part (VJP);
//   C  projection: one thread per (cell, field, test function) sums its six faces' buffer
//      values against the test function's values at the face nodes (residual: +f on the
//      cell's upper faces, -f on its lower faces, times alpha; VJP: the own side's values)
//      and adds to out.
//
// Cell ranges [cbeg, cend) of a whole periodic grid (the host-buffer pipeline's chunks):
// a cell computes its upper faces, and its lower face too when the lower neighbour is outside
// the range, so every face a range's cells need is in the buffer after A.
#include <cmath>

#include "faces_euler.h"
#include "handle.h"

namespace bosss {

namespace {

constexpr int NV = 5;          // conservative variables (3D Euler)
constexpr int FPB = 8;         // faces per CTA of the face kernel

template <int K, int Q>
struct FaceCfg {
    static constexpr int NP = np_of(3, K);
    static constexpr int QF = Q * Q;
    static constexpr int NT = FPB * QF;       // threads of the face kernel
    static constexpr int CPB_P = (NV * NP <= 100) ? 4 : 2;   // cells per CTA of the projection
};

// value of basis function (a, b, c) at face node (q1, q2) of face (d, side)
template <int K, int Q>
__device__ __forceinline__ double face_phi(const Tables1D& T, int d, int side, int q1, int q2, int a, int b, int c) {
    // in-plane directions t1 < t2; the face coordinate of d is -1 (side 0) or +1 (side 1)
    const int ex[3] = {a, b, c};
    const int t1 = (d == 0) ? 1 : 0, t2 = (d == 2) ? 1 : 2;
    return T.e[side][ex[d]] * T.A[q1][ex[t1]] * T.A[q2][ex[t2]];
}

struct FaceArgs {
    EvalArgs a;          // grid, physics, tables, U, V (VJP: W), out, alpha
    double* buf;         // face buffer
    int mode;            // MODE_RES or MODE_VJP
};

// A: face values. Items: (cell c in [cbeg, cend), direction d, side): side 1 = the cell's upper
// face (owner c), side 0 = its lower face, only when the lower neighbour is outside the range.
template <int K, int Q, int MODE>
__global__ void __launch_bounds__(FaceCfg<K, Q>::NT) k_euler_faces(const __grid_constant__ FaceArgs f, int side) {
    using C = FaceCfg<K, Q>;
    constexpr int NP = C::NP, QF = C::QF, NCF = (MODE == MODE_VJP) ? 2 * NV : NV;
    const EvalArgs& a = f.a;
    const GridConst& g = a.g;
    const Tables1D& T = a.tab;
    __shared__ double cf[FPB][2][NCF * NP];   // owner, neighbour: U (and W for the VJP)
    const int t = threadIdx.x, lf = t / QF, q = t % QF;
    const long long ncells = a.cend - a.cbeg;
    const long long item = (long long)blockIdx.x * FPB + lf;   // (cell, d) pairs
    const bool live = item < ncells * 3;
    long long own = -1, nb = -1;
    int d = 0;
    if (live) {
        const long long c = a.cbeg + item / 3;
        d = (int)(item % 3);
        int ijk[3];
        cell_ijk(g, c, ijk);
        if (side == 1) {
            own = c;
            nb = neighbour(g, ijk, d, 1);
        } else {
            const long long ln = neighbour(g, ijk, d, 0);
            if (ln < a.cbeg || ln >= a.cend) {   // lower neighbour outside the range
                own = ln;
                nb = c;
            }
        }
    }
    // stage the two cells' coefficients (threads of the face cooperate)
    for (int i = q; i < 2 * NCF * NP; i += QF) {
        const int s = i / (NCF * NP), r = i % (NCF * NP);
        double v = 0.0;
        if (own >= 0) {
            const long long cell = s ? nb : own;
            v = (r < NV * NP) ? a.U[cell * (NV * NP) + r] : a.V[cell * (NV * NP) + (r - NV * NP)];
        }
        cf[lf][s][r] = v;
    }
    __syncthreads();
    if (own < 0) return;
    const int q1 = q % Q, q2 = q / Q;
    // traces: owner at its upper face (side 1), neighbour at its lower face (side 0)
    double UA[NCF], UB[NCF];
#pragma unroll
    for (int i = 0; i < NCF; ++i) UA[i] = UB[i] = 0.0;
#pragma unroll
    for (int s0 = 0; s0 <= K; ++s0)
#pragma unroll
        for (int A = 0; A <= s0; ++A)
#pragma unroll
            for (int B = 0; B <= s0 - A; ++B) {
                const int Cc = s0 - A - B, n = mode3(A, B, Cc);
                const double pa = face_phi<K, Q>(T, d, 1, q1, q2, A, B, Cc);
                const double pb = face_phi<K, Q>(T, d, 0, q1, q2, A, B, Cc);
#pragma unroll
                for (int i = 0; i < NCF; ++i) {
                    UA[i] += cf[lf][0][i * NP + n] * pa;
                    UB[i] += cf[lf][1][i * NP + n] * pb;
                }
            }
#pragma unroll
    for (int i = 0; i < NCF; ++i) {
        UA[i] *= g.scaling;
        UB[i] *= g.scaling;
    }
    double nrm[3] = {0.0, 0.0, 0.0};
    nrm[d] = 1.0;
    const double fac = T.w[q1] * T.w[q2] * g.faceSG[d] * g.scaling;
    double* out = f.buf + ((own * 3 + d) * NCF) * QF + q;
    if constexpr (MODE == MODE_RES) {
        double gA[NV], gB[NV];
#pragma unroll
        for (int e = 0; e < NV; ++e) gA[e] = gB[e] = 0.0;
        double x[3] = {0.0, 0.0, 0.0};
        PhysEuler<3>::inner<double>(a.ph, 0.0, UA, nullptr, UB, nullptr, nrm, x, gA, nullptr, gB, nullptr);
#pragma unroll
        for (int e = 0; e < NV; ++e) out[e * QF] = gA[e] * fac;
    } else {
        // reverse mode: gradient of sum_e f_e (w_IN,e - w_OUT,e) with respect to both traces
        double fb[NV], UAb[NV], UBb[NV];
#pragma unroll
        for (int e = 0; e < NV; ++e) fb[e] = UA[NV + e] - UB[NV + e];
        PhysEuler<3>::inner_adj(a.ph, UA, UB, nrm, fb, UAb, UBb);
#pragma unroll
        for (int e = 0; e < NV; ++e) {
            out[e * QF] = UAb[e] * fac;
            out[(NV + e) * QF] = UBb[e] * fac;
        }
    }
}

// C: projection of the six faces' buffer values onto each cell's test functions, added to out.
template <int K, int Q, int MODE>
__global__ void __launch_bounds__(FaceCfg<K, Q>::CPB_P * NV * FaceCfg<K, Q>::NP)
    k_euler_face_project(const __grid_constant__ FaceArgs f) {
    using C = FaceCfg<K, Q>;
    constexpr int NP = C::NP, QF = C::QF, NCF = (MODE == MODE_VJP) ? 2 * NV : NV, CPB = C::CPB_P;
    const EvalArgs& a = f.a;
    const GridConst& g = a.g;
    const Tables1D& T = a.tab;
    __shared__ double fv[CPB][6][NV][QF];   // the cell's own-side values of its 6 faces
    const int t = threadIdx.x, lc = t / (NV * NP), r = t % (NV * NP), e = r / NP, n = r % NP;
    const long long c = a.cbeg + (long long)blockIdx.x * CPB + lc;
    const bool live = c < a.cend;
    int ijk[3] = {0, 0, 0};
    if (live) cell_ijk(g, c, ijk);
    // stage: faces (d, side 1) owned by c; (d, side 0) owned by the lower neighbour
    for (int i = r; i < 6 * NV * QF; i += NV * NP) {
        const int qq = i % QF, ee = (i / QF) % NV, fc = i / (QF * NV), d = fc / 2, s = fc % 2;
        double v = 0.0;
        if (live) {
            const long long o = s ? c : neighbour(g, ijk, d, 0);
            // residual: +f on the upper face (IN side), -f on the lower face (OUT side);
            // VJP: the owner-side values on the upper face, the neighbour-side ones on the lower
            const long long idx = ((o * 3 + d) * NCF + ((MODE == MODE_VJP && !s) ? NV + ee : ee)) * QF + qq;
            v = f.buf[idx];
            if (MODE == MODE_RES && !s) v = -v;
        }
        fv[lc][fc][ee][qq] = v;
    }
    __syncthreads();
    if (!live) return;
    // test function n = (A, B, Cc)
    int A = 0, B = 0, Cc = 0;
    for (int s0 = 0; s0 <= K; ++s0)
        for (int aa = 0; aa <= s0; ++aa)
            for (int bb = 0; bb <= s0 - aa; ++bb)
                if (mode3(aa, bb, s0 - aa - bb) == n) {
                    A = aa;
                    B = bb;
                    Cc = s0 - aa - bb;
                }
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int qq = 0; qq < QF; ++qq)
                acc += fv[lc][2 * d + s][e][qq] * face_phi<K, Q>(T, d, s, qq % Q, qq / Q, A, B, Cc);
    double* o = a.out + c * (NV * NP) + e * NP + n;
    if constexpr (MODE == MODE_RES) *o += a.alpha * acc;
    else *o += acc;
}

template <int K, int Q>
int launch_faces(bosss_handle* h, int mode, const EvalArgs& a, cudaStream_t s) {
    using C = FaceCfg<K, Q>;
    FaceArgs f{};
    f.a = a;
    f.buf = h->dFace;
    f.mode = mode;
    const long long n = a.cend - a.cbeg;
    const unsigned gridA = (unsigned)((n * 3 + FPB - 1) / FPB);
    const unsigned gridC = (unsigned)((n + C::CPB_P - 1) / C::CPB_P);
    const bool whole = a.cbeg == 0 && a.cend == a.g.J;
    if (mode == MODE_RES) {
        k_euler_faces<K, Q, MODE_RES><<<gridA, C::NT, 0, s>>>(f, 1);
        if (!whole) k_euler_faces<K, Q, MODE_RES><<<gridA, C::NT, 0, s>>>(f, 0);
        k_euler_face_project<K, Q, MODE_RES><<<gridC, C::CPB_P * NV * C::NP, 0, s>>>(f);
    } else {
        k_euler_faces<K, Q, MODE_VJP><<<gridA, C::NT, 0, s>>>(f, 1);
        if (!whole) k_euler_faces<K, Q, MODE_VJP><<<gridA, C::NT, 0, s>>>(f, 0);
        k_euler_face_project<K, Q, MODE_VJP><<<gridC, C::CPB_P * NV * C::NP, 0, s>>>(f);
    }
    CUDA_TRY(cudaGetLastError());
    return BOSSS_OK;
}

}  // namespace

bool faces_once_supported(const bosss_handle* h) {
    if (h->phys != PHYS_EULER || h->D != 3) return false;
    for (int d = 0; d < 3; ++d)
        if (!h->base.g.periodic[d] || h->base.g.gn[d] != h->base.g.n[d] || h->base.g.goff[d] != 0) return false;
    const int K = h->K, Q = h->Q;
    return (K == 3 && Q == 4) || (K == 2 && Q == 3) || (K == 1 && Q == 2) || (K == 4 && Q == 5);
}

int faces_once_alloc(bosss_handle* h) {
    if (h->dFace) return BOSSS_OK;
    const long long QF = (long long)h->Q * h->Q;
    const size_t n = (size_t)h->base.g.J * 3 * 2 * NV * QF;   // VJP: two sides
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMalloc(&h->dFace, sizeof(double) * n));
    return BOSSS_OK;
}

int faces_once_launch(bosss_handle* h, int mode, const EvalArgs& a, cudaStream_t s) {
    if (mode != MODE_RES && mode != MODE_VJP) return fail(BOSSS_ERR_BAD_ARG, "face-once path: residual and VJP");
    int rc = faces_once_alloc(h);
    if (rc) return rc;
    switch (h->K * 10 + h->Q) {
        case 34: return launch_faces<3, 4>(h, mode, a, s);
        case 23: return launch_faces<2, 3>(h, mode, a, s);
        case 12: return launch_faces<1, 2>(h, mode, a, s);
        case 45: return launch_faces<4, 5>(h, mode, a, s);
        default: return fail(BOSSS_ERR_BAD_ARG, "face-once path: no instance for this degree and rule");
    }
}

}  // namespace bosss
