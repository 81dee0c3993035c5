// tc_volume.cu -- volume terms of the 3D Euler residual with the basis contractions on the
// 5th-generation tensor cores (tcgen05, kind::i8), exact to FP64 rounding level.
//
// What it computes (NECQuadratureVolume.EvaluateEx + SaveIntegrationResults,
// NECQuadratureVolume.cs:328-798, for the INonlinearFlux volume term -int F(u) . grad v):
//   u[c,v,q]  = Scaling * sum_n U[c,v,n] phi_n(xi_q)                        (interpolation)
//   F[c,e,d,q] = Euler flux of u[c,:,q] (FP64, PhysEuler::volume, the slab kernel's functor)
//   R[c,e,n]  = detJ Scaling sum_{d,q} F[c,e,d,q] w_q (2/h_d) dphi_n/dxi_d(xi_q)  (projection)
//   out       = beta * out + alpha * R
// The two contractions are the dense products of DGField_Evaluation.cs:100-110 (dgemm) and
// NECQuadratureVolume.cs:689-716 (einsum), [cells*5 x Np] x [Np x Q^3] and
// [cells*5 x 3 Q^3] x [3 Q^3 x Np].
//
// Precision: every FP64 operand row is scaled by a power of two (its largest magnitude
// below 2^E) and split exactly into LEVELS signed 8-bit slices, x = 2^E 2^-6 sum_s a_s 2^-7s
// (|a_s| <= 64, each slice the rounded remainder of the previous one); the constant tables
// are split the same way on the host. The products a_s b_t are exact in the tensor core's
// 32-bit integer accumulators (K <= 192: |sum| < 2^22); products with s + t = L share
// accumulator L, and the LEVELS accumulators are recombined in FP64 (Horner in 2^-7).
// Products with s + t >= LEVELS and the last slices' remainders are dropped: relative to
// (row scale) x (table scale) x K the error is below 2^-48 with LEVELS = 6. The volume terms
// are much larger than the residual they sum to (the nearly constant pressure's volume and
// face integrals cancel), so the residual's relative error is larger than that: 5 levels gave
// 8e-10 at Euler 32^3 k=3, 6 levels stay inside 1e-10. The pointwise Euler flux stays FP64.
//
// Work split: a persistent grid, one CTA (256 threads, 8 warps) per SM owning 512 columns
// of tensor memory; a CTA walks over tiles of TC = 128 / 5 = 25 cells (125 MMA rows).
// Per tile: slice U -> 21 MMAs (M=128, N=64, K=32) -> recombine u into shared memory ->
// one pass of the flux for the row scales -> per direction d: flux + slicing -> 42 MMAs
// (M=128, N=32, K=32) -> recombine R and store. Tensor-core accumulators: stage 1 at
// columns [0, 384), stage 3 at [0, 192) after stage 1 has been drained. One thread issues all MMAs; completion is
// tracked by one mbarrier (tcgen05.commit), every wait bounded (a timeout sets the
// handle's error flag and the tile's outputs are not trusted).
#include <cmath>
#include <cstring>
#include <vector>

#include "handle.h"
#include "tc_sm100.cuh"
#include "tc_volume.h"

namespace bosss {

namespace {

constexpr int LEVELS = 6;        // slices per operand
constexpr int ROWS = 128;        // MMA M
constexpr int THREADS = 256;
constexpr int NV = 5;            // conservative variables (3D Euler)
constexpr int TCELLS = ROWS / NV;
constexpr int QN = 4;            // Gauss nodes per direction
constexpr int NQ = QN * QN * QN; // volume nodes (stage-1 N, stage-3 K per direction)
constexpr int NPK = 32;          // padded basis size (stage-1 K); Np <= 20 (k <= 3)
constexpr int N1 = NQ;           // stage-1 N
constexpr int N3 = 32;           // stage-3 N (padded Np)
constexpr int K3 = 3 * NQ;       // stage-3 K
constexpr int SU = NQ + 1;       // padded row stride of the node values (doubles)
constexpr uint32_t TMEM_COLS = 512;
// accumulator column bases: the projection accumulators reuse the interpolation ones (the
// node values are drained before the first projection MMA is issued)
constexpr uint32_t T1 = 0, T3 = 0;
static_assert(LEVELS * N1 <= (int)TMEM_COLS && LEVELS * N3 <= (int)TMEM_COLS, "tensor memory");

// shared-memory layout (bytes)
constexpr int SZ_B1 = (NPK / 16) * N1 * 16;     // one slice of the interpolation table
constexpr int SZ_B3 = (K3 / 16) * N3 * 16;      // one slice of the projection table
constexpr int SZ_A1 = (NPK / 16) * ROWS * 16;   // one slice of the coefficient tile
constexpr int SZ_A3 = (NQ / 16) * ROWS * 16;    // one slice of one direction's flux tile
constexpr int OFF_B1 = 0;
constexpr int OFF_B3 = OFF_B1 + LEVELS * SZ_B1;
constexpr int OFF_A1 = OFF_B3 + LEVELS * SZ_B3;
constexpr int OFF_A3 = OFF_A1 + LEVELS * SZ_A1;
constexpr int OFF_U = OFF_A3 + LEVELS * SZ_A3;                // node values, FP64 [ROWS][SU]
constexpr int OFF_P1 = OFF_U + ROWS * SU * 8;                 // 2^e1[q]   (double, N1)
constexpr int OFF_P3 = OFF_P1 + N1 * 8;                       // 2^e3[n]   (double, N3)
constexpr int OFF_R1 = OFF_P3 + N3 * 8;                       // row factor of stage 1 (double, ROWS)
constexpr int OFF_R3 = OFF_R1 + ROWS * 8;                     // |F| max bits / row factor (u64/double, ROWS)
constexpr int OFF_I3 = OFF_R3 + ROWS * 8;                     // 2^(6-E3) per row (double, ROWS)
constexpr int OFF_BAR = OFF_I3 + ROWS * 8;                    // mbarrier + tmem slot
constexpr int SMEM_BYTES = OFF_BAR + 16;
static_assert(OFF_A1 % 1024 == 0 && OFF_A3 % 1024 == 0 && OFF_B3 % 1024 == 0, "operand alignment");

constexpr uint32_t WAIT_ITERS = 1u << 22;

__device__ __forceinline__ int row_exponent(double maxabs) {
    // smallest E with maxabs < 2^E (0 for an all-zero row)
    return maxabs > 0.0 ? ilogb(maxabs) + 1 : 0;
}

// LEVELS slices of v * 2^(6-E) (|.| < 64): a_0 = rint(r), a_s = rint(128 (r_{s-1} - a_{s-1}))
__device__ __forceinline__ void slice(double v, double inv, int8_t* a) {
    double r = v * inv;
#pragma unroll
    for (int s = 0; s < LEVELS; ++s) {
        const double q = rint(r);
        a[s] = (int8_t)(int)q;
        r = (r - q) * 128.0;
    }
}

// recombination of the LEVELS accumulators of one entry: sum_L D_L 2^-7L
__device__ __forceinline__ double combine(const int32_t (*D)[16], int j) {
    double acc = (double)D[LEVELS - 1][j];
#pragma unroll
    for (int L = LEVELS - 2; L >= 0; --L) acc = acc * (1.0 / 128.0) + (double)D[L][j];
    return acc;
}

__device__ __forceinline__ void report(int* err) {
    if (err) atomicExch(err, 1);
}

struct TcArgs {
    const int8_t* B1;     // LEVELS slices, shared-memory layout
    const int8_t* B3;
    const double* p1;     // 2^e1[q]
    const double* p3;     // 2^e3[n]
    const double* U;
    double* out;
    double alpha, beta;
    double scaling, detJscaling;
    long long J;          // cells
    int np;               // basis functions per variable
    int* err;             // wait-timeout flag
    PhysParams ph;
};

__global__ void __launch_bounds__(THREADS, 1) tc_volume_kernel(const __grid_constant__ TcArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    int8_t* sB1 = reinterpret_cast<int8_t*>(sm + OFF_B1);
    int8_t* sB3 = reinterpret_cast<int8_t*>(sm + OFF_B3);
    int8_t* sA1 = reinterpret_cast<int8_t*>(sm + OFF_A1);
    int8_t* sA3 = reinterpret_cast<int8_t*>(sm + OFF_A3);
    double* su = reinterpret_cast<double*>(sm + OFF_U);
    double* p1 = reinterpret_cast<double*>(sm + OFF_P1);
    double* p3 = reinterpret_cast<double*>(sm + OFF_P3);
    double* rf1 = reinterpret_cast<double*>(sm + OFF_R1);
    unsigned long long* mx3 = reinterpret_cast<unsigned long long*>(sm + OFF_R3);
    double* rf3 = reinterpret_cast<double*>(sm + OFF_R3);
    double* inv3 = reinterpret_cast<double*>(sm + OFF_I3);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + OFF_BAR + 8);

    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int NP = a.np, NVP = NV * NP;

    // ---- once per CTA: tables into shared memory, tensor memory, barrier
    {
        const int4* s1 = reinterpret_cast<const int4*>(a.B1);
        int4* d1 = reinterpret_cast<int4*>(sB1);
        for (int i = t; i < LEVELS * SZ_B1 / 16; i += THREADS) d1[i] = s1[i];
        const int4* s3 = reinterpret_cast<const int4*>(a.B3);
        int4* d3 = reinterpret_cast<int4*>(sB3);
        for (int i = t; i < LEVELS * SZ_B3 / 16; i += THREADS) d3[i] = s3[i];
        for (int i = t; i < N1; i += THREADS) p1[i] = a.p1[i];
        for (int i = t; i < N3; i += THREADS) p3[i] = a.p3[i];
    }
    if (w == 0) tc::tmem_alloc(tslot, TMEM_COLS);
    if (t == 0) tc::mbar_init(mbar, 1);
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *tslot;
    const uint32_t tlane = tbase + ((uint32_t)(32 * (w & 3)) << 16);   // this warp's lane quarter
    const int half = w >> 2;                                             // column half of the drains
    const int drow = 32 * (w & 3) + lane;                                // row this thread drains
    uint32_t phase = 0;
    bool ok = true;

    const long long ntiles = (a.J + TCELLS - 1) / TCELLS;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long c0 = tile * TCELLS;
        const int ncell = (int)((a.J - c0) < TCELLS ? (a.J - c0) : TCELLS);
        const int nrow = ncell * NV;

        // ---- 1. coefficient rows -> slices (thread = (row, 16-byte K chunk))
        {
            const int r = t >> 1, ch = t & 1;
            double v[16];
            double mx = 0.0;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int n = ch * 16 + i;
                v[i] = (r < nrow && n < NP) ? __ldg(a.U + c0 * NVP + (long long)r * NP + n) : 0.0;
                mx = fmax(mx, fabs(v[i]));
            }
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            const int E = row_exponent(mx);
            const double inv = ldexp(1.0, 6 - E);
            int8_t sl[LEVELS][16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                int8_t s5[LEVELS];
                slice(v[i], inv, s5);
#pragma unroll
                for (int s = 0; s < LEVELS; ++s) sl[s][i] = s5[s];
            }
#pragma unroll
            for (int s = 0; s < LEVELS; ++s)
                *reinterpret_cast<int4*>(sA1 + s * SZ_A1 + ch * ROWS * 16 + r * 16) = *reinterpret_cast<int4*>(sl[s]);
            if (ch == 0) rf1[r] = ldexp(a.scaling, E - 12);
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();

        // ---- 2. interpolation MMAs: accumulator L gets the products with s + t = L
        if (t == 0) {
            tc::fence_after_sync();
            constexpr uint32_t id = tc::idesc_i8(ROWS, N1);
#pragma unroll 1
            for (int L = 0; L < LEVELS; ++L)
                for (int s = 0; s <= L; ++s) {
                    const uint64_t ad = tc::desc_kmajor(tc::smem_u32(sA1 + s * SZ_A1), ROWS * 16, 128);
                    const uint64_t bd = tc::desc_kmajor(tc::smem_u32(sB1 + (L - s) * SZ_B1), N1 * 16, 128);
                    tc::mma_i8(tbase + T1 + L * N1, ad, bd, id, s > 0);
                }
            tc::commit(mbar);
        }
        if (!tc::mbar_wait(mbar, phase, WAIT_ITERS)) { ok = false; report(a.err); }
        phase ^= 1u;
        tc::fence_after_sync();

        // ---- 3. recombine the node values into shared memory (thread = (row, 32 columns))
        {
            const double f = rf1[drow];
#pragma unroll 1
            for (int cc = 0; cc < 2; ++cc) {
                const int col0 = half * 32 + cc * 16;
                int32_t D[LEVELS][16];
#pragma unroll
                for (int L = 0; L < LEVELS; ++L) tc::ld16(tlane + T1 + L * N1 + col0, D[L]);
                tc::ld_wait();
                if (drow < nrow) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) su[drow * SU + col0 + j] = combine(D, j) * f * p1[col0 + j];
                }
            }
        }
        if (t < ROWS) mx3[t] = 0ull;
        tc::fence_before_sync();
        __syncthreads();

        // ---- 4. flux magnitudes per output row (row scales of the projection operand)
        for (int i = t; i < ncell * NQ; i += THREADS) {
            const int c = i / NQ, q = i % NQ;
            double U[NV], fV[NV], fG[NV][3];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                U[v] = su[(c * NV + v) * SU + q];
                fV[v] = 0.0;
                fG[v][0] = fG[v][1] = fG[v][2] = 0.0;
            }
            PhysEuler<3>::volume<double>(a.ph, U, nullptr, nullptr, fV, fG);
#pragma unroll
            for (int e = 0; e < NV; ++e) {
                double m = fmax(fabs(fG[e][0]), fmax(fabs(fG[e][1]), fabs(fG[e][2])));
                // NQ is a multiple of 32: the warp shares the cell
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
                if (lane == 0) atomicMax(&mx3[c * NV + e], (unsigned long long)__double_as_longlong(m));
            }
        }
        __syncthreads();
        if (t < ROWS) {
            const int E = row_exponent(__longlong_as_double((long long)mx3[t]));
            inv3[t] = ldexp(1.0, 6 - E);
            rf3[t] = ldexp(a.detJscaling, E - 12);
        }
        __syncthreads();

        // ---- 5. per direction: flux -> slices -> projection MMAs into the stage-3 accumulators
#pragma unroll 1
        for (int d = 0; d < 3; ++d) {
            // thread item = (cell, 4 consecutive nodes): one 32-bit word per (row, slice)
            for (int i = t; i < ncell * (NQ / 4); i += THREADS) {
                const int c = i / (NQ / 4), q0 = (i % (NQ / 4)) * 4;
                uint32_t word[NV][LEVELS];
#pragma unroll
                for (int e = 0; e < NV; ++e)
#pragma unroll
                    for (int s = 0; s < LEVELS; ++s) word[e][s] = 0u;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    double U[NV], fV[NV], fG[NV][3];
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        U[v] = su[(c * NV + v) * SU + q0 + k];
                        fV[v] = 0.0;
                        fG[v][0] = fG[v][1] = fG[v][2] = 0.0;
                    }
                    PhysEuler<3>::volume<double>(a.ph, U, nullptr, nullptr, fV, fG);
#pragma unroll
                    for (int e = 0; e < NV; ++e) {
                        int8_t s5[LEVELS];
                        slice(fG[e][d], inv3[c * NV + e], s5);
#pragma unroll
                        for (int s = 0; s < LEVELS; ++s) word[e][s] |= ((uint32_t)(uint8_t)s5[s]) << (8 * k);
                    }
                }
                const int ch = q0 >> 4, off = q0 & 15;
#pragma unroll
                for (int e = 0; e < NV; ++e)
#pragma unroll
                    for (int s = 0; s < LEVELS; ++s)
                        *reinterpret_cast<uint32_t*>(sA3 + s * SZ_A3 + ch * ROWS * 16 + (c * NV + e) * 16 + off) =
                            word[e][s];
            }
            tc::fence_proxy_async();
            tc::fence_before_sync();
            __syncthreads();
            if (t == 0) {
                tc::fence_after_sync();
                constexpr uint32_t id = tc::idesc_i8(ROWS, N3);
#pragma unroll 1
                for (int ks = 0; ks < NQ / 32; ++ks)
                    for (int L = 0; L < LEVELS; ++L)
                        for (int s = 0; s <= L; ++s) {
                            const uint64_t ad =
                                tc::desc_kmajor(tc::smem_u32(sA3 + s * SZ_A3 + ks * 2 * ROWS * 16), ROWS * 16, 128);
                            const int chunk = (d * NQ + ks * 32) / 16;
                            const uint64_t bd =
                                tc::desc_kmajor(tc::smem_u32(sB3 + (L - s) * SZ_B3 + chunk * N3 * 16), N3 * 16, 128);
                            tc::mma_i8(tbase + T3 + L * N3, ad, bd, id, d > 0 || ks > 0 || s > 0);
                        }
                tc::commit(mbar);
            }
            // the next direction overwrites the flux slices: wait for these MMAs
            if (!tc::mbar_wait(mbar, phase, WAIT_ITERS)) { ok = false; report(a.err); }
            phase ^= 1u;
            tc::fence_after_sync();
        }

        // ---- 6. recombine R and store (thread = (row, 16 test functions))
        {
            int32_t D[LEVELS][16];
            const int col0 = half * 16;
#pragma unroll
            for (int L = 0; L < LEVELS; ++L) tc::ld16(tlane + T3 + L * N3 + col0, D[L]);
            tc::ld_wait();
            if (drow < nrow && ok) {
                const double f = rf3[drow];
                double* o = a.out + c0 * NVP + (long long)drow * NP;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = col0 + j;
                    if (n < NP) {
                        const double R = combine(D, j) * f * p3[n];
                        o[n] = (a.beta == 0.0) ? a.alpha * R : a.beta * o[n] + a.alpha * R;
                    }
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }
    tc::fence_before_sync();
    __syncthreads();
    if (w == 0) tc::tmem_dealloc(tbase, TMEM_COLS);
}

// ------------------------------------------------------------------ host: tables
void host_slice(double v, double inv, int8_t* s) {
    double r = v * inv;
    for (int i = 0; i < LEVELS; ++i) {
        const double q = std::nearbyint(r);
        s[i] = (int8_t)(int)q;
        r = (r - q) * 128.0;
    }
}

int host_exponent(double maxabs) { return maxabs > 0.0 ? std::ilogb(maxabs) + 1 : 0; }

}  // namespace

struct TcVolume {
    int8_t* B1 = nullptr;
    int8_t* B3 = nullptr;
    double* p1 = nullptr;
    double* p3 = nullptr;
    int* err = nullptr;
    int nsm = 0;
};

bool tc_volume_supported(const bosss_handle* h) {
    return h->phys == PHYS_EULER && h->D == 3 && h->Q == QN && np_of(3, h->K) <= 20;
}

int tc_volume_setup(bosss_handle* h) {
    if (!tc_volume_supported(h))
        return fail(BOSSS_ERR_BAD_ARG, "split-precision path: 3D Euler with DG degree <= 3 and 4 Gauss nodes per "
                                       "direction (quadrature order 6 or 7)");
    const Tables1D& T = h->base.tab;
    const GridConst& g = h->base.g;
    const int K = h->K, NP = np_of(3, K);
    // basis index -> exponents (x, y, z), reference order (mode3)
    std::vector<int> ea(NP), eb(NP), ec(NP);
    for (int s = 0; s <= K; ++s)
        for (int A = 0; A <= s; ++A)
            for (int B = 0; B <= s - A; ++B) {
                const int C = s - A - B, n = mode3(A, B, C);
                ea[n] = A;
                eb[n] = B;
                ec[n] = C;
            }
    // interpolation table phi_n(xi_q), q = (qz*Q + qy)*Q + qx, rows q, K index n
    std::vector<int8_t> B1((size_t)LEVELS * SZ_B1, 0);
    std::vector<double> p1(N1), p3(N3);
    for (int q = 0; q < NQ; ++q) {
        const int qx = q % QN, qy = (q / QN) % QN, qz = q / (QN * QN);
        double row[NPK] = {0}, mx = 0;
        for (int n = 0; n < NP; ++n) {
            row[n] = T.A[qx][ea[n]] * T.A[qy][eb[n]] * T.A[qz][ec[n]];
            mx = std::max(mx, std::fabs(row[n]));
        }
        const int E = host_exponent(mx);
        p1[q] = std::ldexp(1.0, E);
        for (int n = 0; n < NPK; ++n) {
            int8_t s[LEVELS];
            host_slice(row[n], std::ldexp(1.0, 6 - E), s);
            for (int l = 0; l < LEVELS; ++l) B1[(size_t)l * SZ_B1 + (n / 16) * N1 * 16 + q * 16 + (n % 16)] = s[l];
        }
    }
    // projection table w_q (2/h_d) dphi_n/dxi_d(xi_q), rows n, K index d*NQ + q
    std::vector<int8_t> B3((size_t)LEVELS * SZ_B3, 0);
    for (int n = 0; n < N3; ++n) {
        std::vector<double> row(K3, 0.0);
        double mx = 0;
        if (n < NP)
            for (int d = 0; d < 3; ++d)
                for (int q = 0; q < NQ; ++q) {
                    const int qx = q % QN, qy = (q / QN) % QN, qz = q / (QN * QN);
                    const double ax = d == 0 ? T.dA[qx][ea[n]] : T.A[qx][ea[n]];
                    const double ay = d == 1 ? T.dA[qy][eb[n]] : T.A[qy][eb[n]];
                    const double az = d == 2 ? T.dA[qz][ec[n]] : T.A[qz][ec[n]];
                    const double v = T.w[qx] * T.w[qy] * T.w[qz] * g.twoh[d] * ax * ay * az;
                    row[d * NQ + q] = v;
                    mx = std::max(mx, std::fabs(v));
                }
        const int E = host_exponent(mx);
        p3[n] = std::ldexp(1.0, E);
        for (int k = 0; k < K3; ++k) {
            int8_t s[LEVELS];
            host_slice(row[k], std::ldexp(1.0, 6 - E), s);
            for (int l = 0; l < LEVELS; ++l) B3[(size_t)l * SZ_B3 + (k / 16) * N3 * 16 + n * 16 + (k % 16)] = s[l];
        }
    }
    TcVolume* tv = new TcVolume();
    h->tcv = tv;
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMalloc(&tv->B1, B1.size()));
    CUDA_TRY(cudaMalloc(&tv->B3, B3.size()));
    CUDA_TRY(cudaMalloc(&tv->p1, sizeof(double) * N1));
    CUDA_TRY(cudaMalloc(&tv->p3, sizeof(double) * N3));
    CUDA_TRY(cudaMalloc(&tv->err, sizeof(int)));
    CUDA_TRY(cudaMemcpy(tv->B1, B1.data(), B1.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(tv->B3, B3.data(), B3.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(tv->p1, p1.data(), sizeof(double) * N1, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(tv->p3, p3.data(), sizeof(double) * N3, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(tv->err, 0, sizeof(int)));
    CUDA_TRY(cudaDeviceGetAttribute(&tv->nsm, cudaDevAttrMultiProcessorCount, h->device));
    CUDA_TRY(cudaFuncSetAttribute(tc_volume_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    return BOSSS_OK;
}

void tc_volume_destroy(bosss_handle* h) {
    TcVolume* tv = h->tcv;
    if (!tv) return;
    cudaFree(tv->B1);
    cudaFree(tv->B3);
    cudaFree(tv->p1);
    cudaFree(tv->p3);
    cudaFree(tv->err);
    delete tv;
    h->tcv = nullptr;
}

int tc_volume_launch(bosss_handle* h, const double* U, double* out, double alpha, double beta, cudaStream_t s) {
    TcVolume* tv = h->tcv;
    if (!tv) return fail(BOSSS_ERR_BAD_ARG, "split-precision tables missing");
    TcArgs a{};
    a.B1 = tv->B1;
    a.B3 = tv->B3;
    a.p1 = tv->p1;
    a.p3 = tv->p3;
    a.U = U;
    a.out = out;
    a.alpha = alpha;
    a.beta = beta;
    a.scaling = h->base.g.scaling;
    a.detJscaling = h->base.g.detJ * h->base.g.scaling;
    a.J = h->base.g.J;
    a.np = np_of(3, h->K);
    a.err = tv->err;
    a.ph = h->base.ph;
    const long long ntiles = (a.J + TCELLS - 1) / TCELLS;
    const int grid = (int)std::min<long long>(ntiles, tv->nsm);
    if (grid < 1) return BOSSS_OK;
    tc_volume_kernel<<<grid, THREADS, SMEM_BYTES, s>>>(a);
    CUDA_TRY(cudaGetLastError());
    return BOSSS_OK;
}

int tc_volume_check(bosss_handle* h) {
    TcVolume* tv = h->tcv;
    if (!tv) return BOSSS_OK;
    int flag = 0;
    CUDA_TRY(cudaMemcpy(&flag, tv->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(tv->err, 0, sizeof(int));
        return fail(BOSSS_ERR_TIMEOUT, "split-precision volume kernel: a tensor-core completion wait ran out");
    }
    return BOSSS_OK;
}

}  // namespace bosss
